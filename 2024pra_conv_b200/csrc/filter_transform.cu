// Filter transform U = G g G^T into the tile-major U cache.
//
// Reference: the GgGT* kernels of src/preprocessing.cuh:75-270, which compute
// the same 16 values per (k, c) in fp16 arithmetic and write one of four
// shape-specific layouts, every iteration of the harness.  Here the transform
// runs once per weight tensor, in fp32 with one final rounding, and writes the
// canonical layout of wino_common.cuh so the conv kernels fetch U with bulk
// copies.  One thread per (k, c); threads are numbered in U-cache order so
// each tap's stores from a warp are contiguous.
#include <cuda_runtime.h>
#include <type_traits>
#include "tc_sm100.cuh"
#include "wino_common.cuh"

namespace wino {

template <typename T>
__device__ __forceinline__ T from_f32(float x);
template <>
__device__ __forceinline__ __half from_f32<__half>(float x) { return __float2half_rn(x); }
template <>
__device__ __forceinline__ __nv_bfloat16 from_f32<__nv_bfloat16>(float x) {
  return __float2bfloat16_rn(x);
}

// Linear thread index -> (k, c) in U-cache order (8 c fastest, then 8 k,
// then the two 8-channel halves, then k groups, then 16-channel steps).
__device__ __forceinline__ void uorder_kc(size_t idx, int K, int& k, int& c) {
  const int e = idx & 7;
  const int r = (idx >> 3) & 7;
  const int kc = (idx >> 6) & 1;
  const size_t rest = idx >> 7;
  const int kg = (int)(rest % (size_t)(K >> 3));
  const int cs = (int)(rest / (size_t)(K >> 3));
  k = kg * 8 + r;
  c = cs * 16 + kc * 8 + e;
}

__device__ __forceinline__ void load_filter(const __half* w, int k, int c, int C, float g[9]) {
  const __half* src = w + ((size_t)k * C + c) * 9;
#pragma unroll
  for (int i = 0; i < 9; ++i) g[i] = __half2float(src[i]);
}

// U (fp16 or bf16) for all K x C filters; hi-lo variant writes the residual
// U - round(U) into a second cache when `lo` is non-null.
// layout 0: fused-kernel U cache (u_offset); layout 1: unfused GEMM (u2_offset).
template <typename T>
__global__ void __launch_bounds__(256) filter_transform_kernel(const __half* __restrict__ w,
                                                               T* __restrict__ u, T* __restrict__ lo,
                                                               int K, int C, int layout) {
  const size_t idx = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= (size_t)K * C) return;
  int k, c;
  uorder_kc(idx, K, k, c);
  float g[9], t16[16];
  load_filter(w, k, c, C, g);
  filter_tile(g, t16);
#pragma unroll
  for (int t = 0; t < 16; ++t) {
    const size_t off = layout ? u2_offset(t, k, c, K, C) : u_offset(t, k, c, K, C);
    const T hi = from_f32<T>(t16[t]);
    u[off] = hi;
    if (lo) {
      float r;
      if constexpr (std::is_same<T, __half>::value) r = t16[t] - __half2float(hi);
      else r = t16[t] - __bfloat162float(hi);
      lo[off] = from_f32<T>(r);
    }
  }
}

// Drop-in slot-1 kernel: weight -> transform_filter (fp16 U cache).
__global__ void __launch_bounds__(256) dropin_filter_kernel(KernelParam p) {
  const int K = p.k, C = p.c;
  const size_t idx = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= (size_t)K * C) return;
  int k, c;
  uorder_kc(idx, K, k, c);
  float g[9], t16[16];
  load_filter(static_cast<const __half*>(p.pweight), k, c, C, g);
  filter_tile(g, t16);
  __half* u = static_cast<__half*>(p.transform_filter);
#pragma unroll
  for (int t = 0; t < 16; ++t) u[u_offset(t, k, c, K, C)] = __float2half_rn(t16[t]);
}

// Drop-in slot-1 kernel of the two-stage route: weight -> transform_filter
// in the tap GEMM's U2 layout (u2_offset).
__global__ void __launch_bounds__(256) dropin_filter_u2_kernel(KernelParam p) {
  const int K = p.k, C = p.c;
  const size_t idx = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= (size_t)K * C) return;
  int k, c;
  uorder_kc(idx, K, k, c);
  float g[9], t16[16];
  load_filter(static_cast<const __half*>(p.pweight), k, c, C, g);
  filter_tile(g, t16);
  __half* u = static_cast<__half*>(p.transform_filter);
#pragma unroll
  for (int t = 0; t < 16; ++t) u[u2_offset(t, k, c, K, C)] = __float2half_rn(t16[t]);
}

// ---- fp8 e4m3 -------------------------------------------------------------
// Per-(tap, k) scale su[t][k] = amax_c |U'[t][k][c]| / 448 where
// U'[t][k][c] = U[t][k][c] * sv[c] folds the per-input-channel scale of V
// into the filter (the scales then factor out of the C reduction:
//   M[t][k][tile] = su[t][k] * sum_c q(U'/su)[t][k][c] * q(V/sv)[t][c][tile]).
// One block per (t, k-group of 8); threads loop over c.
__global__ void __launch_bounds__(256) filter_transform_f8_kernel(
    const __half* __restrict__ w, const float* __restrict__ sv, uint8_t* __restrict__ u8,
    float* __restrict__ su, int K, int C) {
  const int t = blockIdx.y;
  const int k = blockIdx.x * 8 + (threadIdx.x >> 5);
  const int lane = threadIdx.x & 31;
  if (k >= K) return;
  float amax = 0.f;
  for (int c = lane; c < C; c += 32) {
    float g[9], t16[16];
    load_filter(w, k, c, C, g);
    filter_tile(g, t16);
    amax = fmaxf(amax, fabsf(t16[t] * sv[c]));
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) amax = fmaxf(amax, __shfl_xor_sync(0xffffffffu, amax, o));
  const float scale = amax > 0.f ? amax / 448.f : 1.f;
  if (lane == 0) su[t * K + k] = scale;
  const float inv = 1.f / scale;
  for (int c = lane; c < C; c += 32) {
    float g[9], t16[16];
    load_filter(w, k, c, C, g);
    filter_tile(g, t16);
    const float x = t16[t] * sv[c] * inv;
    __nv_fp8_e4m3 q(x);
    u8[u8_offset(t, k, c, K, C)] = *reinterpret_cast<uint8_t*>(&q);
  }
}

// fp16 U cache (fused layout, u_offset) -> the same values in the unfused
// GEMM layout (u2_offset): a batch layer routed to the two-stage path
// reuses the caller's fused U cache this way.  One thread per (t, k, c).
__global__ void __launch_bounds__(256) u_to_u2_kernel(const __half* __restrict__ u, __half* __restrict__ u2, int K,
                                                      int C) {
  const size_t idx = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= (size_t)16 * K * C) return;
  const int c = (int)(idx % C);
  const size_t r = idx / C;
  const int k = (int)(r % K), t = (int)(r / K);
  u2[u2_offset(t, k, c, K, C)] = u[u_offset(t, k, c, K, C)];
}

}  // namespace wino

using namespace wino;

extern "C" {

void* wino_dropin_filter_kernel_ptr() { return (void*)dropin_filter_kernel; }
void* wino_dropin_filter_u2_kernel_ptr() { return (void*)dropin_filter_u2_kernel; }

int wino_launch_u_to_u2(const void* u, void* u2, int K, int C, cudaStream_t stream) {
  const size_t n = (size_t)16 * K * C;
  u_to_u2_kernel<<<(unsigned)((n + 255) / 256), 256, 0, stream>>>(static_cast<const __half*>(u),
                                                                   static_cast<__half*>(u2), K, C);
  return (int)cudaGetLastError();
}

int wino_launch_filter_transform(const void* weight, void* ucache, void* ucache_lo, int K, int C,
                                 int bf16, int layout, cudaStream_t stream) {
  const size_t n = (size_t)K * C;
  const unsigned blocks = (unsigned)((n + 255) / 256);
  if (bf16)
    filter_transform_kernel<__nv_bfloat16><<<blocks, 256, 0, stream>>>(
        (const __half*)weight, (__nv_bfloat16*)ucache, (__nv_bfloat16*)ucache_lo, K, C, layout);
  else
    filter_transform_kernel<__half><<<blocks, 256, 0, stream>>>(
        (const __half*)weight, (__half*)ucache, (__half*)ucache_lo, K, C, layout);
  return (int)cudaGetLastError();
}

int wino_launch_filter_transform_f8(const void* weight, const float* sv, void* u8, float* su,
                                    int K, int C, cudaStream_t stream) {
  dim3 grid((K + 7) / 8, 16);
  filter_transform_f8_kernel<<<grid, 256, 0, stream>>>((const __half*)weight, sv, (uint8_t*)u8,
                                                       su, K, C);
  return (int)cudaGetLastError();
}

}  // extern "C"
