// Winograd input transform B^T d B for groups of 8 consecutive tiles, in
// packed fp16 arithmetic, shared by the fused kernel (into shared memory)
// and the unfused input-transform kernel (into global memory).
//
// Reference: calculate_transform_pin / prefetch_input / init_mask of
// src/preprocessing.cuh:6-72 (one tile per thread, mask-based padding,
// fp16 arithmetic).  Here a thread forms 8 tiles x 16 taps of one channel:
// the B^T row combination runs on pairs of adjacent input columns, and a
// byte permute regroups them into pairs of adjacent tiles, so each tap's 8
// tiles leave as one 16-byte row of an MN-major core matrix.  Padding is
// handled by zero words outside the image.
#pragma once
#include <cstdint>
#include <cuda_fp16.h>
#include "wino_common.cuh"

namespace wino {

// Problem geometry derived from the kernel argument (pad 1, stride 1).
struct Geometry {
  int N, C, H, W, K, P, Q, TP, TQ;
  long long NT;         // tiles in the batch
  int nTB, nKB, CS;     // tile blocks, k blocks, 16-channel steps
  long long nblocks;
};

__device__ __forceinline__ Geometry make_geometry(const KernelParam& p, int tiles_per_block) {
  Geometry g;
  g.N = p.n; g.C = p.c; g.H = p.h; g.W = p.w; g.K = p.k;
  g.P = p.Oh; g.Q = p.Ow;
  g.TP = (g.P + 1) >> 1; g.TQ = (g.Q + 1) >> 1;
  g.NT = (long long)g.N * g.TP * g.TQ;
  g.nTB = (int)((g.NT + tiles_per_block - 1) / tiles_per_block);
  g.nKB = (g.K + KB - 1) / KB;
  g.CS = g.C >> 4;
  g.nblocks = (long long)g.nTB * g.nKB;
  return g;
}

// ---- input words ------------------------------------------------------------
// A "word" is two horizontally adjacent fp16 inputs (cols 2m, 2m+1) of one row,
// zero outside the image.  Loads are branch-free: an out-of-image word is read
// from a zero word instead of being skipped, so the loads of a task issue
// back to back and their latencies overlap.
static __device__ const uint32_t g_zero_words[4] = {0u, 0u, 0u, 0u};

// `row` points at column 0 of input row y (or anywhere when !row_ok).
__device__ __forceinline__ uint32_t load_word(const __half* row, bool row_ok, int m, int W,
                                             bool w_even) {
  const int c0 = 2 * m;
  if (w_even) {
    const bool ok = row_ok && m >= 0 && c0 < W;
    const unsigned int* p = ok ? reinterpret_cast<const unsigned int*>(row) + m : g_zero_words;
    return __ldg(p);
  }
  const unsigned short* r16 = reinterpret_cast<const unsigned short*>(row);
  const unsigned short* z16 = reinterpret_cast<const unsigned short*>(g_zero_words);
  const bool ok0 = row_ok && c0 >= 0 && c0 < W;
  const bool ok1 = row_ok && c0 + 1 >= 0 && c0 + 1 < W;
  const uint32_t lo = __ldg(ok0 ? r16 + c0 : z16);
  const uint32_t hi = __ldg(ok1 ? r16 + c0 + 1 : z16);
  return lo | (hi << 16);
}

__device__ __forceinline__ uint32_t hadd2(uint32_t a, uint32_t b) {
  __half2 r = __hadd2(*reinterpret_cast<__half2*>(&a), *reinterpret_cast<__half2*>(&b));
  return *reinterpret_cast<uint32_t*>(&r);
}
__device__ __forceinline__ uint32_t hsub2(uint32_t a, uint32_t b) {
  __half2 r = __hsub2(*reinterpret_cast<__half2*>(&a), *reinterpret_cast<__half2*>(&b));
  return *reinterpret_cast<uint32_t*>(&r);
}
// (hi(x), hi(y)) and (lo(x), lo(y)) packed as (low half, high half).
__device__ __forceinline__ uint32_t pk_hi(uint32_t x, uint32_t y) { return __byte_perm(x, y, 0x7632); }
__device__ __forceinline__ uint32_t pk_lo(uint32_t x, uint32_t y) { return __byte_perm(x, y, 0x5410); }

// B^T rows as word operations: e_a = sum_i Bt[a][i] d_i.
__device__ __forceinline__ uint32_t bt_row(int a, uint32_t d0, uint32_t d1, uint32_t d2, uint32_t d3) {
  switch (a) {
    case 0: return hsub2(d0, d2);
    case 1: return hadd2(d1, d2);
    case 2: return hsub2(d2, d1);
    default: return hsub2(d1, d3);
  }
}

// Column half of the transform for one e-row and a pair of tiles whose window
// columns (a0..a3) are given as lane pairs: V[a][b] for b = 0..3.
__device__ __forceinline__ void bt_cols(uint32_t a0, uint32_t a1, uint32_t a2, uint32_t a3,
                                        uint32_t v[4]) {
  v[0] = hsub2(a0, a2);
  v[1] = hadd2(a1, a2);
  v[2] = hsub2(a2, a1);
  v[3] = hsub2(a1, a3);
}

// Produce V for 8 consecutive tiles (tile0 .. tile0+7) of channel c, all 16
// taps: sink(t, w0, w1, w2, w3) receives tap t as four words, each two tiles
// (tile 2i in the low half of w_i, tile 2i+1 in the high half).
// Each e-row a (taps 4a..4a+3) is stored as soon as it is formed.
// Fast path: all 8 tiles in one tile row and W even (word loads).
template <typename Sink>
__device__ __forceinline__ void produce_v8(const __half* __restrict__ X, const Geometry& g,
                                           long long tile0, int c, Sink&& sink) {
  const bool w_even = (g.W & 1) == 0;
  const long long per_img = (long long)g.TP * g.TQ;
  bool fast = false;
  int n0 = 0, ty0 = 0, tx0 = 0;
  if (tile0 + 7 < g.NT) {
    n0 = (int)(tile0 / per_img);
    const int r = (int)(tile0 - (long long)n0 * per_img);
    ty0 = r / g.TQ;
    tx0 = r - ty0 * g.TQ;
    fast = w_even && (tx0 + 7 < g.TQ);
  }
  if (fast) {
    const __half* plane = X + ((size_t)n0 * g.C + c) * (size_t)g.H * g.W;
    uint32_t d[4][10];
#pragma unroll
    for (int i = 0; i < 4; ++i) {
      const int y = 2 * ty0 - 1 + i;
      const bool ok = y >= 0 && y < g.H;
      const __half* row = plane + (size_t)(ok ? y : 0) * g.W;
#pragma unroll
      for (int j = 0; j < 10; ++j) d[i][j] = load_word(row, ok, tx0 - 1 + j, g.W, true);
    }
#pragma unroll
    for (int a = 0; a < 4; ++a) {
      uint32_t e[10];
#pragma unroll
      for (int j = 0; j < 10; ++j) e[j] = bt_row(a, d[0][j], d[1][j], d[2][j], d[3][j]);
      uint32_t out[4][4];
#pragma unroll
      for (int q = 0; q < 4; ++q) {
        const int u = 2 * q;
        uint32_t v[4];
        bt_cols(pk_hi(e[u], e[u + 1]), pk_lo(e[u + 1], e[u + 2]), pk_hi(e[u + 1], e[u + 2]),
                pk_lo(e[u + 2], e[u + 3]), v);
#pragma unroll
        for (int b = 0; b < 4; ++b) out[b][q] = v[b];
      }
#pragma unroll
      for (int b = 0; b < 4; ++b)
        sink(4 * a + b, out[b][0], out[b][1], out[b][2], out[b][3]);
    }
  } else {
    // General path: each tile locates its own window (row or image changes
    // inside the group, odd widths, tiles past the end of the batch).  Per
    // e-row only the two input rows that B^T combines are read; tile
    // coordinates advance incrementally (consecutive tiles step tx, then ty,
    // then the image).
    int n1 = 0, ty1 = 0, tx1 = 0;
    if (tile0 < g.NT) {
      n1 = (int)(tile0 / per_img);
      const int r = (int)(tile0 - (long long)n1 * per_img);
      ty1 = r / g.TQ;
      tx1 = r - ty1 * g.TQ;
    }
#pragma unroll 1
    for (int a = 0; a < 4; ++a) {
      // rows combined by Bt[a]: (0,2), (1,2), (2,1), (1,3) as (plus, minus / plus)
      const int ra = (a == 0) ? 0 : (a == 2 ? 2 : 1);
      const int rb = (a == 0) ? 2 : (a == 3 ? 3 : (a == 1 ? 2 : 1));
      uint32_t ew[8][3];
      int n = n1, ty = ty1, tx = tx1;
#pragma unroll
      for (int s = 0; s < 8; ++s) {
        const bool valid = tile0 + s < g.NT;
        const int ya = 2 * ty - 1 + ra, yb = 2 * ty - 1 + rb;
        const bool oka = valid && ya >= 0 && ya < g.H;
        const bool okb = valid && yb >= 0 && yb < g.H;
        const __half* base = X + ((size_t)(valid ? n : 0) * g.C + c) * (size_t)g.H * g.W;
        const __half* rowa = base + (size_t)(oka ? ya : 0) * g.W;
        const __half* rowb = base + (size_t)(okb ? yb : 0) * g.W;
#pragma unroll
        for (int j = 0; j < 3; ++j) {
          const uint32_t wa = load_word(rowa, oka, tx - 1 + j, g.W, w_even);
          const uint32_t wb = load_word(rowb, okb, tx - 1 + j, g.W, w_even);
          ew[s][j] = (a == 1) ? hadd2(wa, wb) : hsub2(wa, wb);
        }
        if (++tx == g.TQ) {
          tx = 0;
          if (++ty == g.TP) { ty = 0; ++n; }
        }
      }
      uint32_t out[4][4];
#pragma unroll
      for (int q = 0; q < 4; ++q) {
        const int s0 = 2 * q, s1 = 2 * q + 1;
        uint32_t v[4];
        bt_cols(pk_hi(ew[s0][0], ew[s1][0]), pk_lo(ew[s0][1], ew[s1][1]), pk_hi(ew[s0][1], ew[s1][1]),
                pk_lo(ew[s0][2], ew[s1][2]), v);
#pragma unroll
        for (int b = 0; b < 4; ++b) out[b][q] = v[b];
      }
#pragma unroll
      for (int b = 0; b < 4; ++b)
        sink(4 * a + b, out[b][0], out[b][1], out[b][2], out[b][3]);
    }
  }
}

}  // namespace wino
