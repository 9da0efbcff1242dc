// Shared definitions of the Winograd F(2x2,3x3) kernels: tile geometry,
// the U-cache layout, and the transform matrices.
//
//   G  = [[1,0,0],[1/2,1/2,1/2],[1/2,-1/2,1/2],[0,0,1]]   (reference src/preprocessing.cuh:77-81)
//   Bt = [[1,0,-1,0],[0,1,1,0],[0,-1,1,0],[0,1,0,-1]]    (src/preprocessing.cuh:50-54)
//   At = [[1,1,1,0],[0,1,-1,-1]]                         (src/conv2d.cpp:18-22)
// Tap index t = 4*a + b for row a, column b of the 4x4 Winograd tile, as in
// the reference's G g G^T (preprocessing.cuh:93-108).
//
// Output tile (ty, tx) of image n covers outputs rows 2ty..2ty+1 and columns
// 2tx..2tx+1; its input window is rows 2ty-1..2ty+2, columns 2tx-1..2tx+2,
// zero outside the image (pad = 1).  Tiles are numbered flat over
// (n, ty, tx) with tx fastest; an image has ceil(H/2) * ceil(W/2) tiles.
#pragma once
#include <cstdint>
#include <cuda_fp16.h>
#include <cuda_bf16.h>
#include "wino_param.h"

namespace wino {

// ------------------------------------------------------------ U cache -------
// The transformed filter U[t][k][c] is stored pre-tiled in the canonical
// K-major no-swizzle layout the tensor core reads from shared memory, so a
// CTA fetches the slice it needs with one bulk copy per tap and stage:
//
//   block(cs, t) = U[t][0..K)[16*cs .. 16*cs+16)      (cs = c / 16)
//   blocks ordered (cs, t); inside a block, 8-row groups of k (256 bytes
//   each) hold two 8x8 core matrices (c 0-7, c 8-15) of 8 k-rows x 16 bytes.
//
// fp16/bf16 element offset of (t, k, c) for K output channels:
__host__ __device__ __forceinline__ size_t u_offset(int t, int k, int c, int K) {
  const int cs = c >> 4, cc = c & 15;
  return ((size_t)cs * 16 + t) * (size_t)K * 16 + (size_t)(k >> 3) * 128 + (cc >> 3) * 64 +
         (k & 7) * 8 + (cc & 7);
}

// 8-bit element offset for the fp8 cache: K-steps of 32 channels.
__host__ __device__ __forceinline__ size_t u8_offset(int t, int k, int c, int K) {
  const int cs = c >> 5, cc = c & 31;
  return ((size_t)cs * 16 + t) * (size_t)K * 32 + (size_t)(k >> 3) * 256 + (cc >> 4) * 128 +
         (k & 7) * 16 + (cc & 15);
}

// G g G^T of one 3x3 filter, in fp32 (16 outputs, row-major over the tap).
__host__ __device__ __forceinline__ void filter_tile(const float g[9], float u[16]) {
  float tmp[4][3];
#pragma unroll
  for (int j = 0; j < 3; ++j) {
    tmp[0][j] = g[j];
    tmp[1][j] = 0.5f * (g[j] + g[3 + j] + g[6 + j]);
    tmp[2][j] = 0.5f * (g[j] - g[3 + j] + g[6 + j]);
    tmp[3][j] = g[6 + j];
  }
#pragma unroll
  for (int a = 0; a < 4; ++a) {
    u[4 * a + 0] = tmp[a][0];
    u[4 * a + 1] = 0.5f * (tmp[a][0] + tmp[a][1] + tmp[a][2]);
    u[4 * a + 2] = 0.5f * (tmp[a][0] - tmp[a][1] + tmp[a][2]);
    u[4 * a + 3] = tmp[a][2];
  }
}

__host__ __device__ __forceinline__ int ceil_div(int a, int b) { return (a + b - 1) / b; }

// Precision variants of the GEMM stage.
enum Variant : int { VAR_F16 = 0, VAR_BF16 = 1, VAR_F8 = 2, VAR_F16_HILO = 3 };

}  // namespace wino
