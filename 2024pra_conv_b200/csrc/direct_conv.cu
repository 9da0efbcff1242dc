// Direct convolution for the shapes the Winograd path does not take: any
// filter size R x S, stride (u, v), padding (p, q), and channel counts that
// are not multiples of 16.  The reference's getkernelInfo ignores r, s, u, v,
// p, q (src/conv2d.cpp:254-271) and only its six hard-wired shapes work; here
// those shapes go to this kernel behind the same plugin ABI.
//
// Implicit GEMM on CUDA cores: D[k][pixel] = sum_{(c,r,s)} W[k][(c,r,s)] *
// X[(c,r,s)][pixel], pixel = (n, oy, ox) flattened, fp16 operands, fp32
// accumulation, one fp16 rounding of y.  A CTA computes 64 output channels x
// 64 output pixels in steps of 16 (c, r, s) indices: the weight tile is a
// plain copy (KCRS rows are contiguous in (c, r, s)), the input tile is
// gathered with zero padding; each of 256 threads accumulates 4 x 4 outputs.
// This is the general-shape path, not a tensor-core kernel.
#include <cuda_runtime.h>
#include <cuda_fp16.h>
#include "wino_param.h"

namespace wino {

namespace direct {
constexpr int TK = 64, TP = 64, TC = 16;
}

__global__ void __launch_bounds__(256) direct_conv_kernel(KernelParam p) {
  using namespace direct;
  const int N = p.n, C = p.c, H = p.h, W = p.w, K = p.k, R = p.r, S = p.s;
  const int U = p.u, V = p.v, PH = p.p, PW = p.q, OH = p.Oh, OW = p.Ow;
  const __half* X = static_cast<const __half*>(p.pin);
  const __half* Wt = static_cast<const __half*>(p.pweight);
  __half* Y = static_cast<__half*>(p.pout);
  const int CRS = C * R * S;
  const long long npix = (long long)N * OH * OW;
  const int k0 = blockIdx.y * TK;
  const long long pix0 = (long long)blockIdx.x * TP;

  __shared__ float ws[TC][TK + 1];   // [crs][k]
  __shared__ float xs[TC][TP + 1];   // [crs][pixel]
  const int tid = threadIdx.x;
  const int tk = (tid >> 4) * 4, tp = (tid & 15) * 4;   // this thread's 4 x 4 outputs
  float acc[4][4] = {};

  // loader roles: each thread fills 4 entries of each tile per step
  for (int e0 = 0; e0 < CRS; e0 += TC) {
#pragma unroll
    for (int t = 0; t < 4; ++t) {
      const int idx = tid + 256 * t;          // 0 .. 1023 = TC x 64
      const int e = idx / TK, col = idx % TK;
      // weights: k = k0 + col, crs = e0 + e
      const int kk = k0 + col, crs = e0 + e;
      ws[e][col] = (kk < K && crs < CRS) ? __half2float(Wt[(size_t)kk * CRS + crs]) : 0.f;
      // input: pixel = pix0 + col, crs = e0 + e
      float v = 0.f;
      const long long pix = pix0 + col;
      if (crs < CRS && pix < npix) {
        const int c = crs / (R * S);
        const int rs = crs - c * R * S;
        const int r = rs / S, s = rs - r * S;
        const int n = (int)(pix / ((long long)OH * OW));
        const int rem = (int)(pix - (long long)n * OH * OW);
        const int oy = rem / OW, ox = rem - oy * OW;
        const int y = oy * U - PH + r, x = ox * V - PW + s;
        if (y >= 0 && y < H && x >= 0 && x < W)
          v = __half2float(X[(((size_t)n * C + c) * H + y) * W + x]);
      }
      xs[e][col] = v;
    }
    __syncthreads();
#pragma unroll
    for (int e = 0; e < TC; ++e) {
      float a[4], b[4];
#pragma unroll
      for (int i = 0; i < 4; ++i) {
        a[i] = ws[e][tk + i];
        b[i] = xs[e][tp + i];
      }
#pragma unroll
      for (int i = 0; i < 4; ++i)
#pragma unroll
        for (int j = 0; j < 4; ++j) acc[i][j] = fmaf(a[i], b[j], acc[i][j]);
    }
    __syncthreads();
  }
#pragma unroll
  for (int j = 0; j < 4; ++j) {
    const long long pix = pix0 + tp + j;
    if (pix >= npix) continue;
    const int n = (int)(pix / ((long long)OH * OW));
    const int rem = (int)(pix - (long long)n * OH * OW);
#pragma unroll
    for (int i = 0; i < 4; ++i) {
      const int kk = k0 + tk + i;
      if (kk < K) Y[((size_t)n * K + kk) * OH * OW + rem] = __float2half_rn(acc[i][j]);
    }
  }
}

}  // namespace wino

using namespace wino;

extern "C" {

void* wino_direct_kernel_ptr() { return (void*)direct_conv_kernel; }

// Grid of the direct kernel: x = 64-pixel tiles, y = 64-channel tiles.
void wino_direct_grid(int n, int k, int oh, int ow, unsigned* gx, unsigned* gy) {
  const long long npix = (long long)n * oh * ow;
  *gx = (unsigned)((npix + direct::TP - 1) / direct::TP);
  *gy = (unsigned)((k + direct::TK - 1) / direct::TK);
}

int wino_launch_direct(const KernelParam* p, cudaStream_t stream) {
  unsigned gx, gy;
  wino_direct_grid(p->n, p->k, p->Oh, p->Ow, &gx, &gy);
  void* args[] = {const_cast<KernelParam*>(p)};
  return (int)cudaLaunchKernel((void*)direct_conv_kernel, dim3(gx, gy), dim3(256), args, 0, stream);
}

}  // extern "C"
