// Learned cost model: a small MLP (F inputs -> 64 ReLU -> 64 ReLU -> O
// outputs, fp32) trained and evaluated with hand-written CUDA kernels.  It
// maps shape features of a conv layer to the predicted log-time of each
// schedule configuration; the autotuner's exhaustive timings are its
// training data and remain the fallback and the yardstick of its picks.  The
// reference has no counterpart (it hard-wires one kernel set per shape,
// src/conv2d.cpp:458-494).
//
// Parameter layout (one flat fp32 array, P = 64F + 64 + 64*64 + 64 + 64O + O):
//   W1[64][F], b1[64], W2[64][64], b2[64], W3[O][64], b3[O].
// Loss: masked mean squared error over (sample, output) pairs with mask 1:
//   L = sum_b sum_o m[b][o] (y[b][o] - t[b][o])^2 / sum m.
//
// Kernels: one CTA (64 threads) per sample runs the forward pass in shared
// memory and, for training, its backward pass, writing that sample's
// gradient row; a second kernel reduces the rows in a fixed order
// (deterministic); a third applies Adam.
#include <cstdint>
#include <cuda_runtime.h>

namespace wino {
namespace mlp {

constexpr int H = 64;      // hidden width
constexpr int FMAX = 16;   // features
constexpr int OMAX = 16;   // outputs

__host__ __device__ inline int nparams(int F, int O) { return H * F + H + H * H + H + O * H + O; }

struct Offsets {
  int w1, b1, w2, b2, w3, b3;
};
__host__ __device__ inline Offsets offsets(int F, int O) {
  Offsets o;
  o.w1 = 0;
  o.b1 = o.w1 + H * F;
  o.w2 = o.b1 + H;
  o.b2 = o.w2 + H * H;
  o.w3 = o.b2 + H;
  o.b3 = o.w3 + O * H;
  return o;
}

// grad_rows == nullptr: forward only (y = predictions).  Otherwise also the
// per-sample gradient of the masked MSE (scaled by 1 / inv_count) into
// grad_rows[b][P] and the per-sample loss into loss_rows[b].
__global__ void __launch_bounds__(H) mlp_sample_kernel(const float* __restrict__ prm,
                                                       const float* __restrict__ x,
                                                       const float* __restrict__ target,
                                                       const float* __restrict__ mask, float* __restrict__ y,
                                                       float* __restrict__ grad_rows,
                                                       float* __restrict__ loss_rows, int F, int O,
                                                       float inv_count) {
  const int b = blockIdx.x;
  const int j = threadIdx.x;
  const Offsets of = offsets(F, O);
  const int P = nparams(F, O);
  __shared__ float xs[FMAX], z1[H], h1[H], z2[H], h2[H], out[OMAX], dout[OMAX], dz2[H], dz1[H];
  if (j < F) xs[j] = x[b * F + j];
  __syncthreads();
  float a = prm[of.b1 + j];
  for (int f = 0; f < F; ++f) a += prm[of.w1 + j * F + f] * xs[f];
  z1[j] = a;
  h1[j] = a > 0.f ? a : 0.f;
  __syncthreads();
  a = prm[of.b2 + j];
  for (int i = 0; i < H; ++i) a += prm[of.w2 + j * H + i] * h1[i];
  z2[j] = a;
  h2[j] = a > 0.f ? a : 0.f;
  __syncthreads();
  if (j < O) {
    float o = prm[of.b3 + j];
    for (int i = 0; i < H; ++i) o += prm[of.w3 + j * H + i] * h2[i];
    out[j] = o;
    if (y) y[b * O + j] = o;
  }
  if (!grad_rows) return;
  __syncthreads();
  if (j < O) {
    const float m = mask[b * O + j];
    const float d = out[j] - target[b * O + j];
    dout[j] = 2.f * m * d * inv_count;
  }
  if (j == 0) {
    float l = 0.f;
    for (int o = 0; o < O; ++o) {
      const float d = out[o] - target[b * O + o];
      l += mask[b * O + o] * d * d;
    }
    loss_rows[b] = l * inv_count;
  }
  __syncthreads();
  float* g = grad_rows + (size_t)b * P;
  // layer 3
  for (int o = 0; o < O; ++o) g[of.w3 + o * H + j] = dout[o] * h2[j];
  if (j < O) g[of.b3 + j] = dout[j];
  float dh2 = 0.f;
  for (int o = 0; o < O; ++o) dh2 += prm[of.w3 + o * H + j] * dout[o];
  dz2[j] = z2[j] > 0.f ? dh2 : 0.f;
  __syncthreads();
  // layer 2: row j of W2
  for (int i = 0; i < H; ++i) g[of.w2 + j * H + i] = dz2[j] * h1[i];
  g[of.b2 + j] = dz2[j];
  float dh1 = 0.f;
  for (int k = 0; k < H; ++k) dh1 += prm[of.w2 + k * H + j] * dz2[k];
  dz1[j] = z1[j] > 0.f ? dh1 : 0.f;
  __syncthreads();
  // layer 1: row j of W1
  for (int f = 0; f < F; ++f) g[of.w1 + j * F + f] = dz1[j] * xs[f];
  g[of.b1 + j] = dz1[j];
}

// grad[p] = sum_b rows[b][p] in sample order; loss = sum_b loss_rows[b].
__global__ void mlp_reduce_kernel(const float* __restrict__ rows, const float* __restrict__ loss_rows,
                                  float* __restrict__ grad, float* __restrict__ loss, int B, int P) {
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p < P) {
    float s = 0.f;
    for (int b = 0; b < B; ++b) s += rows[(size_t)b * P + p];
    grad[p] = s;
  }
  if (p == 0 && loss) {
    float l = 0.f;
    for (int b = 0; b < B; ++b) l += loss_rows[b];
    *loss = l;
  }
}

// Adam (bias-corrected), step t >= 1.
__global__ void mlp_adam_kernel(float* __restrict__ prm, const float* __restrict__ grad,
                                float* __restrict__ m, float* __restrict__ v, int P, float lr, float b1,
                                float b2, float eps, float c1, float c2) {
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= P) return;
  const float g = grad[p];
  const float mm = b1 * m[p] + (1.f - b1) * g;
  const float vv = b2 * v[p] + (1.f - b2) * g * g;
  m[p] = mm;
  v[p] = vv;
  prm[p] -= lr * (mm / c1) / (sqrtf(vv / c2) + eps);
}

}  // namespace mlp
}  // namespace wino

using namespace wino::mlp;

namespace {
int check_dims(int F, int O, int B) {
  return (F >= 1 && F <= FMAX && O >= 1 && O <= OMAX && B >= 1) ? 0 : 1;
}
float mask_count_inv(const float* mask_host_sum) { return *mask_host_sum > 0.f ? 1.f / *mask_host_sum : 0.f; }
}  // namespace

extern "C" {

int wino_mlp_num_params(int F, int O) { return nparams(F, O); }

// Predictions y[B][O] for inputs x[B][F] (device pointers).
int wino_mlp_forward(const float* params, const float* x, float* y, int B, int F, int O, void* stream) {
  if (!params || !x || !y || check_dims(F, O, B)) return 1;
  mlp_sample_kernel<<<B, H, 0, (cudaStream_t)stream>>>(params, x, nullptr, nullptr, y, nullptr, nullptr, F,
                                                        O, 0.f);
  return cudaGetLastError() == cudaSuccess ? 0 : 3;
}

// Gradient of the masked MSE at `params` (device pointers): grad[P], loss[1].
// scratch: B * (P + 1) floats.
int wino_mlp_grad(const float* params, const float* x, const float* target, const float* mask, int B,
                  int F, int O, float mask_count, float* grad, float* loss, float* scratch, void* stream) {
  if (!params || !x || !target || !mask || !grad || !scratch || check_dims(F, O, B)) return 1;
  const int P = nparams(F, O);
  const cudaStream_t s = (cudaStream_t)stream;
  float* rows = scratch;
  float* lrows = scratch + (size_t)B * P;
  mlp_sample_kernel<<<B, H, 0, s>>>(params, x, target, mask, nullptr, rows, lrows, F, O,
                                     mask_count_inv(&mask_count));
  mlp_reduce_kernel<<<(P + 255) / 256, 256, 0, s>>>(rows, lrows, grad, loss, B, P);
  return cudaGetLastError() == cudaSuccess ? 0 : 3;
}

// Full-batch Adam training for `epochs` steps (device pointers; m, v: P
// floats each, zero at step 0; scratch: B * (P + 1) + P + 1 floats).
// loss_history (device, may be null): loss before each step.
int wino_mlp_train(float* params, const float* x, const float* target, const float* mask, int B, int F,
                   int O, float mask_count, int epochs, float lr, float* m, float* v, float* scratch,
                   float* loss_history, void* stream) {
  if (!params || !m || !v || !scratch || epochs < 0) return 1;
  const int P = nparams(F, O);
  const cudaStream_t s = (cudaStream_t)stream;
  float* grad = scratch + (size_t)B * (P + 1);
  float* loss = grad + P;
  const float b1 = 0.9f, b2 = 0.999f, eps = 1e-8f;
  float c1 = 1.f, c2 = 1.f;
  for (int t = 1; t <= epochs; ++t) {
    const int rc = wino_mlp_grad(params, x, target, mask, B, F, O, mask_count, grad,
                                 loss_history ? loss_history + (t - 1) : loss, scratch, stream);
    if (rc) return rc;
    c1 *= b1;
    c2 *= b2;
    mlp_adam_kernel<<<(P + 255) / 256, 256, 0, s>>>(params, grad, m, v, P, lr, b1, b2, eps, 1.f - c1,
                                                    1.f - c2);
  }
  return cudaGetLastError() == cudaSuccess ? 0 : 3;
}

}  // extern "C"
