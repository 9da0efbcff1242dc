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
#include <cuda_fp8.h>
#include "wino_param.h"

namespace wino {

// ------------------------------------------------------------ U cache -------
// The transformed filter U[t][k][c] is stored pre-tiled in the canonical
// K-major no-swizzle layout the tensor core reads from shared memory, grouped
// so that one K-step (16 input channels) of one output-channel block is a
// single contiguous piece that a CTA fetches with one bulk copy:
//
//   k-blocks of KB = 128 output channels (the last one may be shorter),
//   inside a k-block: K-steps cs = c / 16, inside a K-step: taps t = 0..15,
//   inside a tap: 8-row groups of k (256 bytes) each holding two 8 x 8 core
//   matrices (channels 0-7 and 8-15 of the step), 8 k-rows x 16 bytes.
//
// A (k-block, K-step) piece holds 16 * kbs * 16 elements (kbs = rows of the
// k-block), taps at a stride of kbs * 16 elements.  Total size 16*K*C.
constexpr int KB = 128;

__host__ __device__ __forceinline__ int kblock_rows(int kb, int K) {
  const int r = K - kb * KB;
  return r < KB ? r : KB;
}

// fp16/bf16 element offset of (t, k, c); C channels, K output channels.
__host__ __device__ __forceinline__ size_t u_offset(int t, int k, int c, int K, int C) {
  const int kb = k / KB, kr = k % KB;
  const int kbs = kblock_rows(kb, K);
  const int cs = c >> 4, cc = c & 15;
  return (size_t)kb * KB * 16 * C + ((size_t)cs * 16 + t) * (size_t)(kbs * 16) + (kr >> 3) * 128 +
         (cc >> 3) * 64 + (kr & 7) * 8 + (cc & 7);
}

// Start (elements) of the (k-block, K-step) piece.
__host__ __device__ __forceinline__ size_t u_piece(int kb, int cs, int K, int C) {
  return (size_t)kb * KB * 16 * C + (size_t)cs * 16 * (size_t)(kblock_rows(kb, K) * 16);
}

// 8-bit cache: K-steps of 32 channels, 8 k-rows x 16 bytes per core matrix.
__host__ __device__ __forceinline__ size_t u8_offset(int t, int k, int c, int K, int C) {
  const int kb = k / KB, kr = k % KB;
  const int kbs = kblock_rows(kb, K);
  const int cs = c >> 5, cc = c & 31;
  return (size_t)kb * KB * 16 * C + ((size_t)cs * 16 + t) * (size_t)(kbs * 32) + (kr >> 3) * 256 +
         (cc >> 4) * 128 + (kr & 7) * 16 + (cc & 15);
}

// ---------------------------------------------- unfused-path layouts -------
// The unfused comparator runs the 16 tap GEMMs as one batched GEMM with
// 128 x 128 output tiles; its operands are laid out so that one pipeline
// stage (up to four 16-channel K-steps) is a single contiguous copy.
//   U2: per tap, k-blocks of KB2 = 128 rows (the last may be shorter), per
//       k-block the K-steps in order, each K-step the canonical K-major
//       layout of wino_common's U cache (8-row groups of two core matrices).
//   V2: per tap, per 128-tile block, per K-step: 16 tile groups of two 8x8
//       MN-major core matrices (8 channels x 8 tiles) = 4 KB.
//   M16: M[t][k][tile] fp16, tiles padded to whole 128-tile blocks.
constexpr int KB2 = 128;
constexpr int TB2 = 128;

__host__ __device__ __forceinline__ int kblock2_rows(int kb, int K) {
  const int r = K - kb * KB2;
  return r < KB2 ? r : KB2;
}

__host__ __device__ __forceinline__ size_t u2_piece(int t, int kb, int cs, int K, int C) {
  return (size_t)t * K * C + (size_t)kb * KB2 * C + (size_t)cs * kblock2_rows(kb, K) * 16;
}

__host__ __device__ __forceinline__ size_t u2_offset(int t, int k, int c, int K, int C) {
  const int kb = k / KB2, kr = k % KB2, cs = c >> 4, cc = c & 15;
  return u2_piece(t, kb, cs, K, C) + (kr >> 3) * 128 + (cc >> 3) * 64 + (kr & 7) * 8 + (cc & 7);
}

__host__ __device__ __forceinline__ size_t v2_piece(int t, int tb, int cs, int nTB, int CS) {
  return (((size_t)t * nTB + tb) * CS + cs) * (size_t)(TB2 * 16);
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
