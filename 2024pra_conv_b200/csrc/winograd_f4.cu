// Winograd F(4x4,3x3): 4x4 output tiles from 6x6 input windows, 36 taps.
//
// The reference has F(2x2,3x3) only (src/preprocessing.cuh:75-424,
// src/matrixmul.cuh:139-556, src/conv2d.cpp:17-250).  F(4x4,3x3) needs 2.25x
// fewer multiplies per output, but its transforms carry coefficients up to 5
// (B), 1/24 (G) and 8 (A), so fp16 operands lose about ten times more
// accuracy than F(2x2).  This path therefore forms U and V in fp32 and stores
// each as fp16 pieces:
//
//   plain : U, V rounded once to fp16                 (c_red = C)
//   hi+lo : hi = fp16(v), lo = fp16(v - hi); the tap GEMM's reduction runs
//           over [V_hi | V_lo | V_hi] x [U_hi | U_hi | U_lo]  (c_red = 3C),
//           i.e. hi*hi + lo*hi + hi*lo accumulated in fp32 by the tensor core
//
// M is kept in fp32 and the output transform runs in fp32 before the single
// fp16 rounding of Y.  Stages (all sm_100a kernels; the GEMM is the unfused
// comparator's tcgen05 tap GEMM with 36 taps and fp32 M):
//
//   f4_filter_transform   W (KCRS)  -> U2 (36 taps, unfused U2 layout)
//   f4_input_transform    X (NCHW)  -> V2 (36 taps, unfused V2 layout), staged
//                         through shared memory into whole-line stores
//   tap_gemm_f32          U2, V2    -> M32[t][k][tile]
//   f4_output_transform   M32       -> Y (N K P Q)
//
// Matrices (Lavin & Gray 2015, points 0, 1, -1, 2, -2, infinity):
//   G  rows [1/4,0,0] [-1/6,-1/6,-1/6] [-1/6,1/6,-1/6] [1/24,1/12,1/6]
//           [1/24,-1/12,1/6] [0,0,1]
//   Bt rows [4,0,-5,0,1,0] [0,-4,-4,1,1,0] [0,4,-4,-1,1,0] [0,-2,-1,2,1,0]
//           [0,2,-1,-2,1,0] [0,4,0,-5,0,1]
//   At rows [1,1,1,1,1,0] [0,1,-1,2,-2,0] [0,1,1,4,4,0] [0,1,-1,8,-8,1]
// Tile (ty, tx) covers outputs 4ty..4ty+3 x 4tx..4tx+3 from input rows
// 4ty-1..4ty+4 and columns 4tx-1..4tx+4, zero outside the image (the pad-1
// window of src/preprocessing.cuh:6-46 with a 4-output step); tap t = 6a + b.
#include <cstdint>
#include <cuda_runtime.h>
#include <cuda_fp16.h>
#include "winoconv.h"
#include "wino_common.cuh"
#include "wino_param.h"

namespace wino {
namespace f4 {

constexpr int TAPS = 36;

__host__ __device__ __forceinline__ int c_red(int C, int hilo) { return hilo ? 3 * C : C; }

// G x (3 values) -> 6 values.
__device__ __forceinline__ void g_col(float x0, float x1, float x2, float o[6]) {
  const float s6 = 1.0f / 6.0f;
  o[0] = 0.25f * x0;
  o[1] = -(x0 + x1 + x2) * s6;
  o[2] = -(x0 - x1 + x2) * s6;
  o[3] = x0 * (1.0f / 24.0f) + x1 * (1.0f / 12.0f) + x2 * s6;
  o[4] = x0 * (1.0f / 24.0f) - x1 * (1.0f / 12.0f) + x2 * s6;
  o[5] = x2;
}

// Bt x (6 values) -> 6 values.
__device__ __forceinline__ void bt_col(const float d[6], float o[6]) {
  o[0] = 4.0f * d[0] - 5.0f * d[2] + d[4];
  o[1] = -4.0f * d[1] - 4.0f * d[2] + d[3] + d[4];
  o[2] = 4.0f * d[1] - 4.0f * d[2] - d[3] + d[4];
  o[3] = -2.0f * d[1] - d[2] + 2.0f * d[3] + d[4];
  o[4] = 2.0f * d[1] - d[2] - 2.0f * d[3] + d[4];
  o[5] = 4.0f * d[1] - 5.0f * d[3] + d[5];
}

// At x (6 values) -> 4 values.
__device__ __forceinline__ void at_col(const float m[6], float o[4]) {
  o[0] = m[0] + m[1] + m[2] + m[3] + m[4];
  o[1] = m[1] - m[2] + 2.0f * (m[3] - m[4]);
  o[2] = m[1] + m[2] + 4.0f * (m[3] + m[4]);
  o[3] = m[1] - m[2] + 8.0f * (m[3] - m[4]) + m[5];
}

// One thread per (k, c): U = G g G^T in fp32 -> fp16 pieces in the U2 layout
// with c_red reduction channels (hi+lo: hi at c and c + C, lo at c + 2C).
__global__ void __launch_bounds__(256) f4_filter_transform(const __half* __restrict__ w,
                                                           __half* __restrict__ u2, int K, int C,
                                                           int hilo) {
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= (long long)K * C) return;
  const int k = (int)(i / C), c = (int)(i - (long long)k * C);
  float g[9];
#pragma unroll
  for (int j = 0; j < 9; ++j) g[j] = __half2float(w[i * 9 + j]);
  float gc[3][6];  // G g: column j of g through G
#pragma unroll
  for (int j = 0; j < 3; ++j) g_col(g[j], g[3 + j], g[6 + j], gc[j]);
  const int CR = c_red(C, hilo);
#pragma unroll
  for (int a = 0; a < 6; ++a) {
    float u[6];
    g_col(gc[0][a], gc[1][a], gc[2][a], u);
#pragma unroll
    for (int b = 0; b < 6; ++b) {
      const int t = 6 * a + b;
      const __half hi = __float2half_rn(u[b]);
      u2[u2_offset(t, k, c, K, CR)] = hi;
      if (hilo) {
        u2[u2_offset(t, k, c + C, K, CR)] = hi;
        u2[u2_offset(t, k, c + 2 * C, K, CR)] = __float2half_rn(u[b] - __half2float(hi));
      }
    }
  }
}

// Input transform.  A CTA covers 64 tiles (half of a 128-tile V2 block) x 8
// channels (half of a 16-channel K-step): exactly one 128-byte chunk of every
// (tap, piece) 4 KB V2 piece per 8 tiles.  Phase 1: each thread forms V for two
// (tile, channel) pairs in fp32 and writes the fp16 pieces into shared-memory
// planes laid out like the V2 chunks (a warp = 8 tiles x 4 channels, so its
// 2-byte stores fill 64 contiguous bytes).  Phase 2: the planes go out as
// 16-byte stores, each warp instruction four whole 128-byte lines.  Tiles
// beyond the batch are written as zeros, so every V2 piece the GEMM reads is
// defined.  grid (2 * tile blocks, C / 8), 256 threads, dynamic shared memory
// 36 KB per piece plane (hi; + lo for hi+lo).
constexpr int IT_THREADS = 256;
constexpr int PLANE = 64 * 8 * 2;          // one tap: 64 tiles x 8 channels fp16

template <bool HILO>
__global__ void __launch_bounds__(IT_THREADS) f4_input_transform(const __half* __restrict__ x,
                                                                 uint8_t* __restrict__ v2, int N,
                                                                 int C, int H, int W, int TP, int TQ,
                                                                 int ntb) {
  extern __shared__ __align__(16) uint8_t sm[];
  uint8_t* const hi_plane = sm;                       // [36][PLANE]
  uint8_t* const lo_plane = sm + TAPS * PLANE;        // [36][PLANE], hi+lo only
  const int tb = blockIdx.x >> 1, gbase = (blockIdx.x & 1) * 8;
  const int oct = blockIdx.y, cs = oct >> 1, h = oct & 1;
  const long long NT = (long long)N * TP * TQ;
  const long long per = (long long)TP * TQ;

#pragma unroll 1
  for (int it = 0; it < 2; ++it) {
    const int p = it * IT_THREADS + threadIdx.x;
    const int tl = p & 7, g = (p >> 5) & 7;
    const int cc8 = ((p >> 8) & 1) * 4 + ((p >> 3) & 3);
    const long long tile = (long long)tb * 128 + (gbase + g) * 8 + tl;
    const int c = oct * 8 + cc8;
    const bool live = tile < NT;
    int n = 0, y0 = 0, x0 = 0;
    if (live) {
      n = (int)(tile / per);
      const int r = (int)(tile - (long long)n * per);
      const int ty = r / TQ, tx = r - ty * TQ;
      y0 = 4 * ty - 1;
      x0 = 4 * tx - 1;
    }
    const __half* xc = x + ((size_t)n * C + c) * H * W;
    // Branch-free window loads: every load reads a clamped in-image address
    // and the value is zeroed where the window leaves the image.
    int xq[6];
    bool qok[6];
#pragma unroll
    for (int q = 0; q < 6; ++q) {
      const int xx = x0 + q;
      qok[q] = xx >= 0 && xx < W;
      xq[q] = min(max(xx, 0), W - 1);
    }
    // f[r][b] = (d B)[r][b], one input row at a time
    float f[6][6];
#pragma unroll
    for (int r = 0; r < 6; ++r) {
      const int y = y0 + r;
      const bool row_ok = live && y >= 0 && y < H;
      const __half* row = xc + (size_t)min(max(y, 0), H - 1) * W;
      float d[6];
#pragma unroll
      for (int q = 0; q < 6; ++q) {
        const float v = __half2float(row[xq[q]]);
        d[q] = (row_ok && qok[q]) ? v : 0.0f;
      }
      bt_col(d, f[r]);
    }
    const int off = g * 128 + cc8 * 16 + tl * 2;
#pragma unroll
    for (int b = 0; b < 6; ++b) {
      float col[6], v[6];
#pragma unroll
      for (int r = 0; r < 6; ++r) col[r] = f[r][b];
      bt_col(col, v);  // v[a] = V[a][b]
#pragma unroll
      for (int a = 0; a < 6; ++a) {
        const int t = 6 * a + b;
        const __half hv = __float2half_rn(v[a]);
        *reinterpret_cast<__half*>(hi_plane + t * PLANE + off) = hv;
        if constexpr (HILO)
          *reinterpret_cast<__half*>(lo_plane + t * PLANE + off) = __float2half_rn(v[a] - __half2float(hv));
      }
    }
  }
  __syncthreads();

  // piece j of tap t: j = 0 hi, 1 lo, 2 hi (reduction order [V_hi | V_lo | V_hi])
  const int CS = C >> 4, CSR = c_red(C, HILO) >> 4;
  constexpr int npiece = HILO ? 3 : 1;
  const int units = TAPS * npiece * (PLANE / 16);
  for (int u = threadIdx.x; u < units; u += IT_THREADS) {
    const int w = u & 63, tj = u >> 6;
    const int t = tj / npiece, j = tj - t * npiece;
    const int g = w >> 3, part = w & 7;
    const uint8_t* src = (j == 1 ? lo_plane : hi_plane) + t * PLANE + g * 128 + part * 16;
    uint8_t* dst = v2 + v2_piece(t, tb, cs + j * CS, ntb, CSR) * 2 + (gbase + g) * 256 + h * 128 + part * 16;
    *reinterpret_cast<uint4*>(dst) = *reinterpret_cast<const uint4*>(src);
  }
}

// grid (ceil(tiles / 256), K): thread = (tile, k); Y tile = At m A in fp32.
// vec: Q % 4 == 0 and Y 8-byte aligned, so each output row of a tile is one
// 8-byte store.
__global__ void __launch_bounds__(256) f4_output_transform(const float* __restrict__ m32,
                                                           __half* __restrict__ y, int K, int P,
                                                           int Q, int TP, int TQ, long long NT,
                                                           long long ntp, int vec) {
  const long long tile = (long long)blockIdx.x * 256 + threadIdx.x;
  const int k = blockIdx.y;
  if (tile >= NT) return;
  float z[4][6];  // z = At m (4 rows x 6 columns)
#pragma unroll
  for (int b = 0; b < 6; ++b) {
    float col[6], o[4];
#pragma unroll
    for (int a = 0; a < 6; ++a) col[a] = m32[((size_t)(6 * a + b) * K + k) * ntp + tile];
    at_col(col, o);
#pragma unroll
    for (int i = 0; i < 4; ++i) z[i][b] = o[i];
  }
  const long long per = (long long)TP * TQ;
  const int n = (int)(tile / per);
  const int r = (int)(tile - (long long)n * per);
  const int ty = r / TQ, tx = r - ty * TQ;
  const int oy = 4 * ty, ox = 4 * tx;
  __half* o = y + (((size_t)n * K + k) * P + oy) * (size_t)Q + ox;
#pragma unroll
  for (int i = 0; i < 4; ++i) {
    if (oy + i >= P) break;
    float yr[4];
    at_col(z[i], yr);
    __half* orow = o + (size_t)i * Q;
    if (vec) {
      const __half2 lo = __floats2half2_rn(yr[0], yr[1]), hi = __floats2half2_rn(yr[2], yr[3]);
      uint2 pk;
      pk.x = *reinterpret_cast<const uint32_t*>(&lo);
      pk.y = *reinterpret_cast<const uint32_t*>(&hi);
      *reinterpret_cast<uint2*>(orow) = pk;
    } else {
#pragma unroll
      for (int j = 0; j < 4; ++j)
        if (ox + j < Q) orow[j] = __float2half_rn(yr[j]);
    }
  }
}

struct Plan {
  int TP, TQ, ntb, CR;
  long long NT, ntp;
  size_t u_bytes, v_bytes, m_bytes;  // each rounded up to 256 bytes
};

inline size_t round256(size_t b) { return (b + 255) / 256 * 256; }

inline Plan plan(int n, int c, int h, int w, int k, int hilo) {
  Plan pl;
  pl.TP = (h + 3) / 4;
  pl.TQ = (w + 3) / 4;
  pl.NT = (long long)n * pl.TP * pl.TQ;
  pl.ntb = (int)((pl.NT + 127) / 128);
  pl.ntp = (long long)pl.ntb * 128;
  pl.CR = c_red(c, hilo);
  pl.u_bytes = round256((size_t)TAPS * k * pl.CR * 2);
  pl.v_bytes = round256((size_t)TAPS * pl.ntp * pl.CR * 2);
  pl.m_bytes = round256((size_t)TAPS * k * pl.ntp * 4);
  return pl;
}

int check(int n, int c, int h, int w, int k, int hilo) {
  if (n < 1 || c < 16 || h < 1 || w < 1 || k < 16) return WINO_EINVAL;
  if (c % 16 || k % 16) return WINO_EUNSUPPORTED;
  if (hilo != 0 && hilo != 1) return WINO_EINVAL;
  if (c > 32767 || h > 32767 || w > 32767 || k > 32767) return WINO_EUNSUPPORTED;
  const Plan pl = plan(n, c, h, w, k, hilo);
  if (pl.ntb > 0x7fffffff / 128 || pl.CR / 16 > 65535) return WINO_EUNSUPPORTED;
  return WINO_OK;
}

}  // namespace f4
}  // namespace wino

using namespace wino;

extern "C" {

size_t wino_f4_filter_bytes(int k, int c, int hilo) {
  return f4::plan(1, c, 1, 1, k, hilo ? 1 : 0).u_bytes;
}

size_t wino_f4_workspace_bytes(int n, int c, int h, int w, int k, int hilo) {
  const f4::Plan pl = f4::plan(n, c, h, w, k, hilo ? 1 : 0);
  return pl.u_bytes + pl.v_bytes + pl.m_bytes;
}

int wino_f4_filter_transform(const void* weight, int k, int c, int hilo, void* workspace,
                             size_t workspace_bytes, void* stream) {
  if (!weight || !workspace) return WINO_EINVAL;
  const int st = f4::check(1, c, 1, 1, k, hilo);
  if (st != WINO_OK) return st;
  if (workspace_bytes < wino_f4_filter_bytes(k, c, hilo)) return WINO_ESCRATCH;
  if ((uintptr_t)workspace & 255) return WINO_EINVAL;
  const long long items = (long long)k * c;
  f4::f4_filter_transform<<<(unsigned)((items + 255) / 256), 256, 0, (cudaStream_t)stream>>>(
      static_cast<const __half*>(weight), static_cast<__half*>(workspace), k, c, hilo);
  return cudaGetLastError() == cudaSuccess ? WINO_OK : WINO_ECUDA;
}

int wino_conv2d_f4(const void* input, void* output, int n, int c, int h, int w, int k, int hilo,
                   void* workspace, size_t workspace_bytes, void* stream) {
  if (!input || !output || !workspace) return WINO_EINVAL;
  const int st = f4::check(n, c, h, w, k, hilo);
  if (st != WINO_OK) return st;
  if (workspace_bytes < wino_f4_workspace_bytes(n, c, h, w, k, hilo)) return WINO_ESCRATCH;
  if ((uintptr_t)workspace & 255) return WINO_EINVAL;
  const f4::Plan pl = f4::plan(n, c, h, w, k, hilo);
  const cudaStream_t s = (cudaStream_t)stream;
  uint8_t* ws = static_cast<uint8_t*>(workspace);
  uint8_t* v2 = ws + pl.u_bytes;
  float* m32 = reinterpret_cast<float*>(ws + pl.u_bytes + pl.v_bytes);
  static const cudaError_t attr = cudaFuncSetAttribute(
      f4::f4_input_transform<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, 2 * f4::TAPS * f4::PLANE);
  if (attr != cudaSuccess) return WINO_ECUDA;
  const dim3 grid(2 * pl.ntb, c / 8);
  if (hilo)
    f4::f4_input_transform<true><<<grid, f4::IT_THREADS, 2 * f4::TAPS * f4::PLANE, s>>>(
        static_cast<const __half*>(input), v2, n, c, h, w, pl.TP, pl.TQ, pl.ntb);
  else
    f4::f4_input_transform<false><<<grid, f4::IT_THREADS, f4::TAPS * f4::PLANE, s>>>(
        static_cast<const __half*>(input), v2, n, c, h, w, pl.TP, pl.TQ, pl.ntb);
  if (cudaGetLastError() != cudaSuccess) return WINO_ECUDA;
  int dev = 0, sms = 148;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  TapGemm tg;
  tg.v2 = v2;
  tg.u2 = ws;
  tg.m = m32;
  tg.taps = f4::TAPS;
  tg.ntb = pl.ntb;
  tg.c_red = pl.CR;
  tg.k = k;
  if (wino_tap_gemm_f32_launch(&tg, sms, stream) != 0) return WINO_ECUDA;
  f4::f4_output_transform<<<dim3((unsigned)((pl.NT + 255) / 256), k), 256, 0, s>>>(
      m32, static_cast<__half*>(output), k, h, w, pl.TP, pl.TQ, pl.NT, pl.ntp,
      (w % 4 == 0 && ((uintptr_t)output & 7) == 0) ? 1 : 0);
  return cudaGetLastError() == cudaSuccess ? WINO_OK : WINO_ECUDA;
}

}  // extern "C"
