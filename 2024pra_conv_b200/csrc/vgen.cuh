// Winograd input transform B^T d B in packed fp16 arithmetic (two channels
// or two tiles per 32-bit word), for the fused and unfused kernels.
//
// Reference: calculate_transform_pin / prefetch_input / init_mask of
// src/preprocessing.cuh:6-72 (one tile per thread, mask-based padding, fp16
// arithmetic).  Three producers:
//   produce_v8                 unfused input transform: a thread forms 8
//                              tiles x 16 taps of one channel from NCHW
//                              input (the B^T rows on pairs of adjacent
//                              columns, a byte permute into pairs of adjacent
//                              tiles), each tap's 8 tiles leaving as one
//                              16-byte row of an MN-major core matrix;
//   produce_v_half_xb          fused kernel: one tile, 8 channels, the 8 taps
//                              of two tap rows, from a shared-memory slab of
//                              the channel-blocked XB input (no bounds checks);
//   produce_v_quarter_global   fused kernel without XB: one tile, 4 channels,
//                              16 taps, straight from NCHW input.
// Padding is zero: zero words outside the image, or XB's zero records.
#pragma once
#include <cstdint>
#include <cuda_fp16.h>
#include "wino_common.cuh"
#include "tc_sm100.cuh"

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
__device__ __forceinline__ uint32_t hmul2_u32(uint32_t a, uint32_t b) {
  __half2 r = __hmul2(*reinterpret_cast<__half2*>(&a), *reinterpret_cast<__half2*>(&b));
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

// Words of one input row for a pair of tiles (A, B = A + 1): tile A needs
// words txA-1 .. txA+1, tile B words txB-1 .. txB+1.  When B is A's right
// neighbour those overlap and four loads serve both; when the pair straddles
// a tile-row (or image) boundary B's three words come from its own row.
struct PairRow {
  uint32_t a0, a1, a2, b0, b1, b2;
};

// Location of one tile: input plane of (image, channel), first window row
// and first window word; valid == false for tiles past the batch.
struct TileLoc {
  const __half* plane;
  int y0, m0;
  bool valid;
};

__device__ __forceinline__ PairRow load_pair_row(const TileLoc& A, const TileLoc& B, bool same_row,
                                                 int i, const Geometry& g, bool w_even) {
  PairRow r;
  const int ya = A.y0 + i;
  const bool oka = A.valid && ya >= 0 && ya < g.H;
  const __half* rowa = A.plane + (size_t)(oka ? ya : 0) * g.W;
  r.a0 = load_word(rowa, oka, A.m0, g.W, w_even);
  r.a1 = load_word(rowa, oka, A.m0 + 1, g.W, w_even);
  r.a2 = load_word(rowa, oka, A.m0 + 2, g.W, w_even);
  if (same_row) {
    r.b0 = r.a1;
    r.b1 = r.a2;
    r.b2 = load_word(rowa, oka, A.m0 + 3, g.W, w_even);
  } else {
    const int yb = B.y0 + i;
    const bool okb = B.valid && yb >= 0 && yb < g.H;
    const __half* rowb = B.plane + (size_t)(okb ? yb : 0) * g.W;
    r.b0 = load_word(rowb, okb, B.m0, g.W, w_even);
    r.b1 = load_word(rowb, okb, B.m0 + 1, g.W, w_even);
    r.b2 = load_word(rowb, okb, B.m0 + 2, g.W, w_even);
  }
  return r;
}

// Produce V for 8 consecutive tiles (tile0 .. tile0+7) of channel c, all 16
// taps: sink(t, w0, w1, w2, w3) receives tap t as four words, each two tiles
// (tile 2i in the low half of w_i, tile 2i+1 in the high half).
// If prefetch_c >= 0 the lines the same tiles need for channel prefetch_c are
// brought into L1 first (the producer's next task), so that task's loads hit.
template <typename Sink>
__device__ __forceinline__ void produce_v8(const __half* __restrict__ X, const Geometry& g,
                                           long long tile0, int c, int prefetch_c, Sink&& sink) {
  const bool w_even = (g.W & 1) == 0;
  const long long per_img = (long long)g.TP * g.TQ;
  const size_t plane_elems = (size_t)g.H * g.W;
  int n = 0, ty = 0, tx = 0;
  if (tile0 < g.NT) {
    n = (int)(tile0 / per_img);
    const int r = (int)(tile0 - (long long)n * per_img);
    ty = r / g.TQ;
    tx = r - ty * g.TQ;
  }
  auto loc = [&](long long tile, int nn, int tyy, int txx) {
    TileLoc L;
    L.valid = tile < g.NT;
    L.plane = X + ((size_t)(L.valid ? nn : 0) * g.C + c) * plane_elems;
    L.y0 = 2 * tyy - 1;
    L.m0 = txx - 1;
    return L;
  };
  auto advance = [&](int& nn, int& tyy, int& txx) {
    if (++txx == g.TQ) {
      txx = 0;
      if (++tyy == g.TP) { tyy = 0; ++nn; }
    }
  };
  if (prefetch_c >= 0 && tile0 < g.NT) {
    // the group spans at most a few tile rows: touch each window row once per run
    const ptrdiff_t dc = (ptrdiff_t)(prefetch_c - c) * (ptrdiff_t)plane_elems;
    int pn = n, pty = ty, ptx = tx;
#pragma unroll
    for (int s = 0; s < 8; ++s) {
      const long long tile = tile0 + s;
      if (tile < g.NT && (s == 0 || ptx == 0)) {
        const __half* pl = X + ((size_t)pn * g.C + c) * plane_elems + dc;
#pragma unroll
        for (int i = 0; i < 4; ++i) {
          const int y = 2 * pty - 1 + i;
          if (y >= 0 && y < g.H) prefetch_l1(pl + (size_t)y * g.W + (ptx > 0 ? 2 * ptx - 2 : 0));
        }
      }
      advance(pn, pty, ptx);
    }
  }
  uint32_t out[16][4];
#pragma unroll
  for (int q = 0; q < 4; ++q) {
    const long long ta = tile0 + 2 * q;
    const TileLoc A = loc(ta, n, ty, tx);
    const bool same_row = tx + 1 < g.TQ;
    advance(n, ty, tx);
    const TileLoc B = loc(ta + 1, n, ty, tx);
    advance(n, ty, tx);
    PairRow d[4];
#pragma unroll
    for (int i = 0; i < 4; ++i) d[i] = load_pair_row(A, B, same_row, i, g, w_even);
#pragma unroll
    for (int a = 0; a < 4; ++a) {
      // e-row a of both tiles (B^T across the window rows), on words
      const uint32_t ea0 = bt_row(a, d[0].a0, d[1].a0, d[2].a0, d[3].a0);
      const uint32_t ea1 = bt_row(a, d[0].a1, d[1].a1, d[2].a1, d[3].a1);
      const uint32_t ea2 = bt_row(a, d[0].a2, d[1].a2, d[2].a2, d[3].a2);
      uint32_t eb0, eb1;
      if (same_row) {
        eb0 = ea1;
        eb1 = ea2;
      } else {
        eb0 = bt_row(a, d[0].b0, d[1].b0, d[2].b0, d[3].b0);
        eb1 = bt_row(a, d[0].b1, d[1].b1, d[2].b1, d[3].b1);
      }
      const uint32_t eb2 = bt_row(a, d[0].b2, d[1].b2, d[2].b2, d[3].b2);
      uint32_t v[4];
      bt_cols(pk_hi(ea0, eb0), pk_lo(ea1, eb1), pk_hi(ea1, eb1), pk_lo(ea2, eb2), v);
#pragma unroll
      for (int b = 0; b < 4; ++b) out[4 * a + b][q] = v[b];
    }
  }
#pragma unroll
  for (int t = 0; t < 16; ++t) sink(t, out[t][0], out[t][1], out[t][2], out[t][3]);
}

// ---------------------------------------------------------------------------
// Channel-blocked input ("XB") for the fused kernel's V producers.
//
// A pre-pass (input_layout.cu) rewrites the NCHW input once per call as
// records of one input row of one image and 16 channels:
//   XB[n][c / 16][r][par][hh][e][8]   (fp16)
// r = y + 1 for y = -1 .. 2*TP (xb_rows(H) = 2*TP + 2 rows), par = column
// parity, hh = channel half (channels 8hh .. 8hh+7), e = entry: par 0 entry
// e holds column x = 2e, par 1 entry e holds column x = 2e - 1, e = 0 .. TQ
// (xb_entries(W) = TQ + 1).  Every position outside the image is zero.
// Then the 4 x 4 window of every tile lies inside the record rows and
// entries, so the producers read it without bounds checks, one 16-byte word
// (four channel pairs) per window position; the window columns of
// consecutive tiles of one tile row are consecutive words.  The rows of a
// step's block form one contiguous run per image, which one bulk copy
// brings into a shared-memory slab.
__host__ __device__ __forceinline__ int xb_rows(int H) { return 2 * ((H + 1) >> 1) + 2; }
__host__ __device__ __forceinline__ int xb_entries(int W) { return ((W + 1) >> 1) + 1; }
__host__ __device__ __forceinline__ int xb_row_bytes(int W) { return 64 * xb_entries(W); }
__host__ __device__ __forceinline__ size_t xb_bytes(int N, int C, int H, int W) {
  return (size_t)N * (size_t)(C >> 4) * (size_t)xb_rows(H) * (size_t)xb_row_bytes(W);
}

constexpr int SLAB_MAXSEG = 4;
constexpr int SLAB_BYTES = 16 * 1024;

// Rows of one block's slab: per image it covers (segment) the record rows
// 2*ta .. 2*tb + 3 of its first and last tile rows ta, tb.
struct SlabPlan {
  int nseg, n0, total_rows;
  int ta[SLAB_MAXSEG], rows[SLAB_MAXSEG], row_base[SLAB_MAXSEG];
};

__device__ __forceinline__ SlabPlan slab_plan(const Geometry& g, int tile0, int tiles_per_block) {
  SlabPlan pl;
  const int per_img = g.TP * g.TQ;
  int last = tile0 + tiles_per_block - 1;
  if (last >= (int)g.NT) last = (int)g.NT - 1;
  const int n0 = tile0 / per_img, n1 = last / per_img;
  const int ty0 = (tile0 - n0 * per_img) / g.TQ;
  const int ty1 = (last - n1 * per_img) / g.TQ;
  pl.n0 = n0;
  pl.nseg = n1 - n0 + 1;
  int base = 0;
#pragma unroll
  for (int k = 0; k < SLAB_MAXSEG; ++k) {
    const int ta = (k == 0) ? ty0 : 0;
    const int tb = (k == pl.nseg - 1) ? ty1 : g.TP - 1;
    pl.ta[k] = ta;
    pl.rows[k] = (k < pl.nseg) ? 2 * (tb - ta) + 4 : 0;
    pl.row_base[k] = base;
    base += pl.rows[k];
  }
  pl.total_rows = base;
  return pl;
}

// ncb: XB channel blocks a step stages (16 channels each).
__device__ __forceinline__ bool slab_fits(const Geometry& g, const SlabPlan& pl, int ncb = 1) {
  return pl.nseg <= SLAB_MAXSEG && ncb * pl.total_rows * xb_row_bytes(g.W) <= SLAB_BYTES;
}

// Window origin of one tile; tiles past the end of the batch take the
// coordinates of `fallback_tile` (a valid tile of the same block), so their
// reads stay inside the block's slab.  32-bit: tile counts stay below 2^31
// for any tensor that fits in device memory.
struct TileCoord {
  int n, ty, tx, y0, m0;
  bool valid;
};

__device__ __forceinline__ TileCoord tile_coord(const Geometry& g, int tile, int fallback_tile) {
  TileCoord tc;
  tc.valid = tile < (int)g.NT;
  const int per_img = g.TP * g.TQ;
  const int t = tc.valid ? tile : fallback_tile;
  tc.n = t / per_img;
  const int r = t - tc.n * per_img;
  tc.ty = r / g.TQ;
  tc.tx = r - tc.ty * g.TQ;
  tc.y0 = 2 * tc.ty - 1;
  tc.m0 = tc.tx - 1;
  return tc;
}

// Shared-memory offsets of one tile's window inside a slab, for channel
// half hh: row i of the window at row_off + i * rb; window column j at
// +col_par1 (j = 0), +col_par0 (j = 1), +col_par1 + 16 (j = 2),
// +col_par0 + 16 (j = 3).
struct SlabWindow {
  uint32_t row_off, rb, col_par0, col_par1;
};

__device__ __forceinline__ SlabWindow slab_window(const Geometry& g, const SlabPlan& pl,
                                                  const TileCoord& tc, int hh) {
  SlabWindow sw;
  int k = tc.n - pl.n0;
  k = k < 0 ? 0 : (k >= SLAB_MAXSEG ? SLAB_MAXSEG - 1 : k);
  int ta = pl.ta[0], rbase = pl.row_base[0];
#pragma unroll
  for (int j = 1; j < SLAB_MAXSEG; ++j)
    if (k == j) { ta = pl.ta[j]; rbase = pl.row_base[j]; }
  const int E = xb_entries(g.W);
  sw.rb = (uint32_t)xb_row_bytes(g.W);
  sw.row_off = (uint32_t)(rbase + 2 * (tc.ty - ta)) * sw.rb;
  sw.col_par0 = (uint32_t)((hh * E + tc.tx) * 16);
  sw.col_par1 = (uint32_t)(((2 + hh) * E + tc.tx) * 16);
  return sw;
}

__device__ __forceinline__ void lds_v4(uint32_t addr, uint32_t (&w)[4]) {
  asm volatile("ld.shared.v4.b32 {%0, %1, %2, %3}, [%4];"
               : "=r"(w[0]), "=r"(w[1]), "=r"(w[2]), "=r"(w[3])
               : "r"(addr));
}

// V of one tile for 8 channels (four pairs) and the 8 taps of tap rows
// 2*ar, 2*ar+1 from an XB slab (tap rows 0-1 use window rows 0-2, tap rows
// 2-3 window rows 1-3).  sink(u, w[4]): tap 8*ar + u, channel pairs 0..3.
template <int AR, typename Sink>
__device__ __forceinline__ void produce_v_half_xb(uint32_t slab, const SlabWindow& sw, Sink&& sink) {
  constexpr int ar = AR;
  uint32_t d[3][4][4];  // window row (ar + i), column j, channel pair
#pragma unroll
  for (int i = 0; i < 3; ++i) {
    const uint32_t row = slab + sw.row_off + (uint32_t)(ar + i) * sw.rb;
    lds_v4(row + sw.col_par1, d[i][0]);
    lds_v4(row + sw.col_par0, d[i][1]);
    lds_v4(row + sw.col_par1 + 16, d[i][2]);
    lds_v4(row + sw.col_par0 + 16, d[i][3]);
  }
  uint32_t out[8][4];
#pragma unroll
  for (int p = 0; p < 4; ++p) {
#pragma unroll
    for (int a2 = 0; a2 < 2; ++a2) {
      uint32_t e[4];
#pragma unroll
      for (int j = 0; j < 4; ++j) {
        // rows present: ar + 0..2; B^T row a = 2*ar + a2
        if (AR == 0)
          e[j] = a2 == 0 ? hsub2(d[0][j][p], d[2][j][p]) : hadd2(d[1][j][p], d[2][j][p]);
        else
          e[j] = a2 == 0 ? hsub2(d[1][j][p], d[0][j][p]) : hsub2(d[0][j][p], d[2][j][p]);
      }
      uint32_t v[4];
      bt_cols(e[0], e[1], e[2], e[3], v);
#pragma unroll
      for (int b = 0; b < 4; ++b) out[4 * a2 + b][p] = v[b];
    }
  }
#pragma unroll
  for (int u = 0; u < 8; ++u) sink(u, out[u]);
}

// Same from global memory (fallback for problems whose slab does not fit).
template <typename Sink>
__device__ __forceinline__ void produce_v_quarter_global(const __half* __restrict__ X,
                                                         const Geometry& g, const TileCoord& tc,
                                                         int c, Sink&& sink) {
  const bool w_even = (g.W & 1) == 0;
  const size_t plane_elems = (size_t)g.H * g.W;
  const __half* base = X + ((size_t)tc.n * g.C + c) * plane_elems;
  const int m0 = tc.m0;
  int rowoff[4];
  bool rowok[4];
#pragma unroll
  for (int i = 0; i < 4; ++i) {
    const int y = tc.y0 + i;
    rowok[i] = tc.valid && y >= 0 && y < g.H;
    rowoff[i] = (rowok[i] ? y : 0) * g.W;
  }
  uint32_t out[16][2];
#pragma unroll
  for (int cp = 0; cp < 2; ++cp) {
    const __half* pa = base + (size_t)(2 * cp) * plane_elems;
    const __half* pb = pa + plane_elems;
    uint32_t wa[4][3], wb[4][3];
#pragma unroll
    for (int i = 0; i < 4; ++i)
#pragma unroll
      for (int j = 0; j < 3; ++j) {
        wa[i][j] = load_word(pa + rowoff[i], rowok[i], m0 + j, g.W, w_even);
        wb[i][j] = load_word(pb + rowoff[i], rowok[i], m0 + j, g.W, w_even);
      }
    uint32_t d[4][4];
#pragma unroll
    for (int i = 0; i < 4; ++i) {
      d[i][0] = pk_hi(wa[i][0], wb[i][0]);
      d[i][1] = pk_lo(wa[i][1], wb[i][1]);
      d[i][2] = pk_hi(wa[i][1], wb[i][1]);
      d[i][3] = pk_lo(wa[i][2], wb[i][2]);
    }
#pragma unroll
    for (int a = 0; a < 4; ++a) {
      uint32_t e[4];
#pragma unroll
      for (int j = 0; j < 4; ++j) e[j] = bt_row(a, d[0][j], d[1][j], d[2][j], d[3][j]);
      uint32_t v[4];
      bt_cols(e[0], e[1], e[2], e[3], v);
#pragma unroll
      for (int b = 0; b < 4; ++b) out[4 * a + b][cp] = v[b];
    }
  }
#pragma unroll
  for (int t = 0; t < 16; ++t) sink(t, out[t][0], out[t][1]);
}

}  // namespace wino
