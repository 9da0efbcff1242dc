// Two-stage Winograd F(2x2,3x3): an input pre-pass, full-width tcgen05 tap
// GEMMs writing M, and the output transform as a third kernel.
//
// The single fused kernel (fused_conv.cu) keeps all 16 taps of a tile block
// in TMEM until the output transform, which caps its MMAs at N = 32 tiles.
// This path gives that up for full-width MMAs: the GEMM writes M once, in
// fp16 (16 * K * tiles elements, the size of the reference's mid_result for
// even H, W), and a third kernel applies A^T m A, the stages of the
// reference's pipeline (src/preprocessing.cuh:273-424 writing V to
// transform_pin, src/matrixmul.cuh:139-556 reading it back,
// src/conv2d.cpp:17-250 reading M from mid_result).
//
//   slot 1  dropin_filter_u2_kernel     W -> U2 (unfused GEMM layout), transform_filter
//   slot 2  v2_layout_kernel            X -> V2 (transformed tiles), transform_pin
//   slot 3  twostage_res_kernel_t<1>    V2, U2 -> M (blocked, below), mid_result
//   slot 4  twostage_output_kernel      M -> Y
// for C <= 256; for larger C slot 2 is xb_layout_kernel (X -> XB, the
// channel-blocked input) and slot 3 twostage_stream_kernel (V formed in
// shared memory from XB, U streamed).  The drop-in ABI takes this route
// when M fits mid_result (even H and W) and the pre-pass output fits
// transform_pin; the extension entry point wino_conv2d_twostage runs slots
// 2-4 on any shape.  Build options route C to the producer-fed kernels on
// row-transformed input (XR): twostage_res_kernel_t<0> (WINO_RES_XR_MAX_C)
// and twostage_pair_kernel (WINO_PAIR_MAX_C); both are slower on B200.
//
// M layout (blocked by 128-tile blocks): block tb holds M[t][k][i] for the
// block's ntb = min(128, tiles - 128 tb) tiles, element
//   tb * 16 * K * 128 + (t * K + k) * ntb + i,
// 16 * K * tiles elements in all (no padding).  Rows of a full block are 256
// bytes, so the GEMM epilogue writes and the output transform reads whole
// 16- and 8-byte words.
//
// V is formed with the fused kernel's packed-fp16 operations (rows of B^T d
// first, then columns; every +- sum of two fp16 values rounded once), so the
// GEMM operands are bit-identical to the fused kernel's and to the unfused
// comparator's; with M rounded once to fp16 the output equals the unfused
// comparator's.
//
// twostage_res_kernel_t (C <= 256, the drop-in's GEMM) is described at its
// definition below.
//
// twostage_pair_kernel (build option): a cluster of two CTAs issues
// tcgen05.mma.cta_group::2 of M = 256 output channels x N = 128 tiles x 16
// channels.  A work unit is a PAIR of taps x 256 output channels x 128
// tiles, all C.  The taps of a pair are chosen so that they read common
// input-window words: (a,1)+(a,2) share all four words of their window rows
// and columns, and (0,b)+(1,b), (3,b)+(2,b) for b in {0, 3} share three rows
// and two columns (six words for two taps); over the 16 taps that is 40
// words per tile and 8 channels against 64 for one tap per unit.  Each CTA
// of the pair forms V for 64 of the unit's 128 tiles (the pair MMA reads
// both halves) and keeps its 128 output channels of U for both taps and all
// C resident in shared memory (128 KB, reloaded only when the pair's tap
// pair or k-block changes), so the only L2 traffic of the main loop is the
// window words.  Each (tap pair, k pair) has its own clusters, in number
// proportional to the pair's window words, which take its tile blocks
// round-robin (make_sched below).
//
// twostage_stream_kernel (any C): one CTA per SM, a unit is one tap x 128
// tiles x 256 output channels (two M = 128 MMAs per K-step sharing the tile
// operand), U streamed per stage by bulk copy.
//
// Every wait is bounded; a timeout records an error code that
// wino_twostage_error_read_clear returns.
#include <cuda_runtime.h>
#include <cuda_fp16.h>
#include "tc_sm100.cuh"
#include "wino_common.cuh"
#include "vgen.cuh"

// Load instruction of the tap-pair producers' window words: through L1
// (ld.global.nc) by default, or cached in L2 only (ld.global.cg).
#ifndef WINO_PAIR_LOAD
#define WINO_PAIR_LOAD __ldg
#endif

// Largest C routed to the tap-pair kernel (0: every C takes the streamed-U
// kernel).  The default build routes none: on N128 C256 H=W28 K256 the
// streamed-U kernel's pre-pass + GEMM measure 26.8 + 147.6 us against the
// tap-pair route's 41.0 + 187.6 us.  Tuning builds set
// -DWINO_PAIR_MAX_C=256 (at most 16 * tp::CS_MAX).
#ifndef WINO_PAIR_MAX_C
#define WINO_PAIR_MAX_C 0
#endif
// Largest C routed to the resident-U kernel (C above it, and above
// WINO_PAIR_MAX_C, takes the streamed-U kernel).
#ifndef WINO_RES_MAX_C
#define WINO_RES_MAX_C 256
#endif
// Largest C whose resident-U kernel forms V from row-transformed input
// (XR) in producer warps instead of reading V2 by bulk copy (0: none).
#ifndef WINO_RES_XR_MAX_C
#define WINO_RES_XR_MAX_C 0
#endif

namespace wino {

static __device__ uint32_t g_twostage_err;

namespace ts {

// ---- shared geometry --------------------------------------------------------
struct Geo {
  int K, C, CS, HP, E, TP, TQ, nTB, nKB2, nKP;
  long long NT;
  uint32_t RB;
  size_t cbs;   // bytes between 16-channel record blocks of XB
};

__device__ __forceinline__ Geo geo(const KernelParam& p) {
  Geo g;
  g.K = p.k;
  g.C = p.c;
  g.CS = p.c >> 4;
  g.HP = xb_rows(p.h);
  g.E = xb_entries(p.w);
  g.RB = (uint32_t)xb_row_bytes(p.w);
  g.cbs = (size_t)g.HP * g.RB;
  g.TP = (p.Oh + 1) >> 1;
  g.TQ = (p.Ow + 1) >> 1;
  g.NT = (long long)p.n * g.TP * g.TQ;
  g.nTB = (int)((g.NT + 127) / 128);
  g.nKB2 = (g.K + KB2 - 1) / KB2;
  g.nKP = (g.nKB2 + 1) / 2;
  return g;
}

// Element offset of M[t][k][tile tb*128 + i] in the blocked layout.
__host__ __device__ __forceinline__ size_t m_offset(int tb, int t, int k, int i, int K, long long NT) {
  const long long rem = NT - (long long)tb * 128;
  const int ntb = rem < 128 ? (int)rem : 128;
  return (size_t)tb * 16 * (size_t)K * 128 + ((size_t)t * K + k) * (size_t)ntb + i;
}

// B^T row / column a of the 4-point transform (the fused kernel's bt_row /
// bt_cols: d0-d2, d1+d2, d2-d1, d1-d3) as two indices and the signs s0, s1 of
// s0*x[i0] + s1*x[i1], packed as fp16x2 (+1 = 0x3c00, -1 = 0xbc00).
__host__ __device__ __forceinline__ void bt_pick(int a, int& i0, int& i1, uint32_t& s0, uint32_t& s1) {
  i0 = a == 0 ? 0 : 1;
  i1 = a == 3 ? 3 : 2;
  s0 = a == 2 ? 0xbc00bc00u : 0x3c003c00u;
  s1 = (a == 0 || a == 3) ? 0xbc00bc00u : 0x3c003c00u;
}

// s0*x0 + s1*x1 with one rounding: the product by +-1 is exact, so this is
// bit-identical to the fused kernel's hadd2 / hsub2 whatever the operand order.
__device__ __forceinline__ uint32_t bt_op(uint32_t s0, uint32_t s1, uint32_t x0, uint32_t x1) {
  __half2 r = __hfma2(*reinterpret_cast<__half2*>(&x1), *reinterpret_cast<__half2*>(&s1),
                      __hmul2(*reinterpret_cast<__half2*>(&x0), *reinterpret_cast<__half2*>(&s0)));
  return *reinterpret_cast<uint32_t*>(&r);
}

__device__ __forceinline__ uint4 bt_op4(uint32_t s0, uint32_t s1, const uint4& x0, const uint4& x1) {
  return make_uint4(bt_op(s0, s1, x0.x, x1.x), bt_op(s0, s1, x0.y, x1.y), bt_op(s0, s1, x0.z, x1.z),
                    bt_op(s0, s1, x0.w, x1.w));
}

// Byte offset, inside one (image, 16-channel) XB record block, of the window
// word at window row r (input row 2ty - 1 + r) and window column jc (input
// column 2tx - 1 + jc) of channel half hh: column jc lies in parity
// (jc & 1) ^ 1, entry tx + (jc >> 1).
__device__ __forceinline__ uint32_t win_off(const Geo& g, int ty, int tx, int hh, int r, int jc) {
  return (uint32_t)(2 * ty + r) * g.RB + (uint32_t)(((((jc & 1) ^ 1) * 2 + hh) * g.E + tx + (jc >> 1)) * 16);
}

__device__ __forceinline__ void tile_decode(const Geo& g, long long tile, int& n, int& ty, int& tx) {
  const long long per = (long long)g.TP * g.TQ;
  n = (int)(tile / per);
  const int r = (int)(tile - (long long)n * per);
  ty = r / g.TQ;
  tx = r - ty * g.TQ;
}

}  // namespace ts

// =============================================================================
// Row-transformed input (the tap-pair kernel's pre-pass)
// =============================================================================
// XR: per (image, 16-channel block) the rows rho = 4 ty + a, ty < ceil(H/2),
// a < 4, each row in XB's record format ([parity][channel half][entry][8
// channels], par 0 entry e = column 2e, par 1 entry e = column 2e - 1): row
// (ty, a) holds, per column x in [-1, 2 ceil(W/2)], the tap-row combination
// of the tile row's window,
//   R_a(ty, x) = s0 * X(2ty - 1 + i0, x) + s1 * X(2ty - 1 + i1, x)
// ((i0, i1, s0, s1) = B^T row a), zero rows / columns outside the image, each
// rounded once to fp16: exactly the first (row) step of B^T d B in the fused
// kernel's producers, so V formed from XR by the column step is bit for bit
// the same.  Size N * C/16 * 4 ceil(H/2) * 64 (ceil(W/2) + 1) bytes, about
// twice the input.  One thread per (tile row, entry e): the four window rows
// at columns 2e and 2e + 1 of 16 channels, read once, give the entries of
// all four rows (par 0 entry e, par 1 entry e + 1; the last entry's thread
// also writes the zero column -1).
namespace xr {
__host__ __device__ __forceinline__ int rows(int H) { return 4 * ((H + 1) >> 1); }
__host__ __device__ __forceinline__ size_t bytes(int N, int C, int H, int W) {
  return (size_t)N * (size_t)(C >> 4) * (size_t)rows(H) * (size_t)xb_row_bytes(W);
}
}  // namespace xr

__global__ void __launch_bounds__(256) xr_layout_kernel(KernelParam p) {
  const int C = p.c, H = p.h, W = p.w;
  const int CB = C >> 4, TP = (H + 1) >> 1, E = xb_entries(W);
  const uint32_t items = (uint32_t)p.n * CB * TP * E;
  const unsigned short* X = static_cast<const unsigned short*>(p.pin);
  uint4* XR = static_cast<uint4*>(p.transform_pin);
  const size_t plane = (size_t)H * W;
  const bool w_even = (W & 1) == 0;
  for (uint32_t it = blockIdx.x * blockDim.x + threadIdx.x; it < items; it += gridDim.x * blockDim.x) {
    const uint32_t trow = it / E;                 // (n * CB + cb) * TP + ty
    const int e = (int)(it - trow * E);
    const int ty = (int)(trow % TP);
    const uint32_t ncb = trow / TP;
    const int cb = (int)(ncb % CB), n = (int)(ncb / CB);
    const int x0 = 2 * e;
    const unsigned short* base = X + ((size_t)n * C + 16 * cb) * plane;
    // window rows 0..3 (input rows 2ty - 1 ..), columns (x0, x0 + 1), 16 channels
    uint32_t d[4][16];
#pragma unroll
    for (int r = 0; r < 4; ++r) {
      const int y = 2 * ty - 1 + r;
      const bool rok = y >= 0 && y < H;
      const bool ok0 = rok && x0 < W, ok1 = rok && x0 + 1 < W;
      const unsigned short* src = base + (size_t)(rok ? y : 0) * W + x0;
      if (w_even && ok1) {
#pragma unroll
        for (int i = 0; i < 16; ++i) d[r][i] = *reinterpret_cast<const uint32_t*>(src + i * plane);
      } else {
#pragma unroll
        for (int i = 0; i < 16; ++i)
          d[r][i] = (ok0 ? (uint32_t)src[i * plane] : 0u) | ((ok1 ? (uint32_t)src[i * plane + 1] : 0u) << 16);
      }
    }
    uint4* out = XR + (size_t)trow * 4 * (4 * E);
#pragma unroll
    for (int a = 0; a < 4; ++a) {
      // B^T row a: d0 - d2, d1 + d2, d2 - d1, d1 - d3 (one rounding each)
      uint32_t r[16];
#pragma unroll
      for (int i = 0; i < 16; ++i)
        r[i] = a == 0 ? hsub2(d[0][i], d[2][i]) : a == 1 ? hadd2(d[1][i], d[2][i])
             : a == 2 ? hsub2(d[2][i], d[1][i]) : hsub2(d[1][i], d[3][i]);
      uint4* row = out + a * (4 * E);
#pragma unroll
      for (int hh = 0; hh < 2; ++hh) {
        const uint32_t* q = r + 8 * hh;
        row[hh * E + e] = make_uint4(__byte_perm(q[0], q[1], 0x5410), __byte_perm(q[2], q[3], 0x5410),
                                     __byte_perm(q[4], q[5], 0x5410), __byte_perm(q[6], q[7], 0x5410));
        if (e + 1 < E)
          row[(2 + hh) * E + e + 1] = make_uint4(__byte_perm(q[0], q[1], 0x7632), __byte_perm(q[2], q[3], 0x7632),
                                                 __byte_perm(q[4], q[5], 0x7632), __byte_perm(q[6], q[7], 0x7632));
        else
          row[(2 + hh) * E] = make_uint4(0u, 0u, 0u, 0u);
      }
    }
  }
}

// =============================================================================
// Tap-pair GEMM on CTA pairs (C <= 256)
// =============================================================================
namespace tp {

using namespace ts;

constexpr int SK = 2;                         // K-steps (16 channels) per stage
constexpr int NSTV = 8;                       // V stages
constexpr int VT = 64;                        // tiles per CTA and unit (N / 2)
constexpr int V_TAP = VT * 32;                // 2 KB: one tap, one K-step, 64 tiles x 16 channels
constexpr int V_STAGE = SK * 2 * V_TAP;       // 8 KB
constexpr int CS_MAX = 16;                    // resident U holds up to 16 K-steps (C <= 256)
constexpr int U_STEP = 128 * 32;              // 4 KB: 128 k rows x 16 channels
constexpr int U_TAP = CS_MAX * U_STEP;        // 64 KB
constexpr int U_BYTES = 2 * U_TAP;
constexpr int SMEM_BYTES = U_BYTES + NSTV * V_STAGE + 1024;
// warps 0-3 epilogue (warp w reads TMEM lanes 32 (w % 4) ..), warp 4 lane 0
// U loads (both CTAs) and MMA issue (rank 0), warps 5-12 V producers
constexpr int WARP_E0 = 0, NWARP_E = 4, WARP_MMA = 4, WARP_P0 = 5, NWARP_P = 8;
constexpr int RING = 4;                       // producer register ring (stages of loads)
constexpr int NTHREAD = (WARP_P0 + NWARP_P) * 32;
constexpr int NPAIR = 8;
constexpr uint16_t BOTH = 3;                  // CTA mask of the pair
constexpr uint32_t SLEEP_NS = 32;

struct Shared {
  uint64_t vfull[NSTV], vempty[NSTV];
  uint64_t accfull[2], accempty[2];
  uint64_t ufull, uempty, utx, mmadone;
  uint32_t tmem_base;
  int abort_flag;
};

// Tap pair q: the taps of accumulator slots 0 and 1.  q < 4: (a, 1) and
// (a, 2) of tap row a = q; q >= 4: two tap rows (a0, a1) of tap column b.
__host__ __device__ __forceinline__ void pair_taps(int q, int& t0, int& t1) {
  switch (q) {
    case 0: t0 = 1; t1 = 2; break;     // (0,1) (0,2)
    case 1: t0 = 5; t1 = 6; break;     // (1,1) (1,2)
    case 2: t0 = 9; t1 = 10; break;    // (2,1) (2,2)
    case 3: t0 = 13; t1 = 14; break;   // (3,1) (3,2)
    case 4: t0 = 0; t1 = 4; break;     // (0,0) (1,0)
    case 5: t0 = 12; t1 = 8; break;    // (3,0) (2,0)
    case 6: t0 = 3; t1 = 7; break;     // (0,3) (1,3)
    default: t0 = 15; t1 = 11; break;  // (3,3) (2,3)
  }
}
// Relative cost of a pair's unit (it reads 2 or 4 XR words per tile and
// K-step; the MMA work is the same).
__host__ __device__ __forceinline__ int pair_weight(int q) { return q < 4 ? 2 : 3; }

// Units: u = combo * nTB + tb, combo = q * nKP + kp.  With at least as many
// clusters G as combos, each combo gets a fixed set of n_c >= 1 clusters (one
// each, then the rest in proportion to the pair weights, leftovers by
// largest remainder) and the j-th of them takes the tile blocks j, j + n_c,
// j + 2 n_c, ...: every combo then sweeps the tile blocks at about the same
// pace, so the 8 tap pairs of a tile block read its input rows from L2
// within a short window, and each cluster keeps one U resident throughout.
// With fewer clusters than combos, cluster g takes the combos g, g + G, ...
// whole, one after another.  Unit indices fit 32 bits (the host bounds the
// tile count).
struct Sched {
  int combo;   // the cluster's combo (G >= combos), else its first combo
  int j, s;    // first tile block and tile-block stride (G >= combos)
  int G;
  int cnt;     // units of this cluster
};

__device__ __forceinline__ Sched make_sched(const Geo& g, int cl, int G) {
  Sched sc;
  sc.G = G;
  const int ncombo = NPAIR * g.nKP;
  if (G < ncombo) {
    const int mc = cl < ncombo ? (ncombo - cl + G - 1) / G : 0;
    sc.combo = cl;
    sc.j = 0;
    sc.s = 1;
    sc.cnt = mc * g.nTB;
    return sc;
  }
  const int wsum = g.nKP * (4 * pair_weight(0) + 4 * pair_weight(4));
  const int extra = G - ncombo;  // clusters after one per combo
  // per weight class: floor share and remainder
  const int fa = extra * pair_weight(0) / wsum, ra = extra * pair_weight(0) % wsum;
  const int fb = extra * pair_weight(4) / wsum, rb = extra * pair_weight(4) % wsum;
  const int half = 4 * g.nKP;    // combos per class
  const int left = extra - half * (fa + fb);
  // leftovers: the class with the larger remainder first, in combo order
  const bool b_first = rb >= ra;
  const int first_class_left = left < half ? left : half;
  const int second_class_left = left - first_class_left;
  int start = 0;
  sc.combo = 0;
  sc.j = 0;
  sc.s = 1;
  for (int c = 0; c < ncombo; ++c) {
    const bool isb = (c / g.nKP) >= 4;
    const int rank_in = isb ? c - half : c;   // index within its class
    int n = 1 + (isb ? fb : fa);
    if (isb == b_first ? rank_in < first_class_left : rank_in < second_class_left) ++n;
    if (cl < start + n) {
      sc.combo = c;
      sc.j = cl - start;
      sc.s = n;
      break;
    }
    start += n;
  }
  sc.cnt = sc.j < g.nTB ? (g.nTB - sc.j + sc.s - 1) / sc.s : 0;
  return sc;
}

struct Unit {
  int q, kp, tb;
};

// The i-th unit of a cluster.
__device__ __forceinline__ Unit sched_unit(const Geo& g, const Sched& sc, int i) {
  int combo, tb;
  if (sc.G < NPAIR * g.nKP) {
    const int m = i / g.nTB;
    combo = sc.combo + m * sc.G;
    tb = i - m * g.nTB;
  } else {
    combo = sc.combo;
    tb = sc.j + i * sc.s;
  }
  Unit x;
  x.tb = tb;
  x.q = combo / g.nKP;
  x.kp = combo - x.q * g.nKP;
  return x;
}

// Load side of one unit for a producer thread (tile tl of this CTA's half,
// channel half hh): the 16-byte XR words its
// taps' column step reads.  q < 4: row (ty, a) at columns 2tx (par 0 entry
// tx) and 2tx + 1 (par 1 entry tx + 1); q >= 4: rows (ty, a0), (ty, a1) at
// the two columns of tap column b (b = 0: 2tx - 1, 2tx + 1, par 1 entries
// tx, tx + 1; b = 3: 2tx, 2tx + 2, par 0 entries tx, tx + 1).
struct ProdLoad {
  const uint8_t* rec;  // XR of the tile's image, channel block 0
  uint32_t off[4];
  bool live, four;
};

__device__ __forceinline__ ProdLoad prod_load(const Geo& g, const uint8_t* xr, const Unit& un, int rank,
                                              int tl, int hh) {
  ProdLoad pl;
  const int tile = un.tb * 128 + rank * VT + tl;
  pl.live = tile < (int)g.NT;
  pl.four = un.q >= 4;
  int n = 0, ty = 0, tx = 0;
  if (pl.live) {
    const int per = g.TP * g.TQ;
    n = tile / per;
    const int r = tile - n * per;
    ty = r / g.TQ;
    tx = r - ty * g.TQ;
  }
  int t0, t1;
  pair_taps(un.q, t0, t1);
  const uint32_t RB = g.RB, E = (uint32_t)g.E;
  const uint32_t row0 = (uint32_t)(4 * ty + (t0 >> 2)) * RB, row1 = (uint32_t)(4 * ty + (t1 >> 2)) * RB;
  const uint32_t hb = (uint32_t)(hh * E) * 16;
  if (!pl.four) {
    pl.off[0] = row0 + hb + (uint32_t)tx * 16;                    // column 2tx
    pl.off[1] = row0 + hb + (2 * E + (uint32_t)tx + 1) * 16;      // column 2tx + 1
    pl.off[2] = pl.off[3] = 0;
  } else {
    const uint32_t par = (t0 & 3) == 0 ? 2 * E : 0;              // b = 0: odd columns
    const uint32_t c0 = (par + (uint32_t)tx) * 16, c1 = (par + (uint32_t)tx + 1) * 16;
    pl.off[0] = row0 + hb + c0;
    pl.off[1] = row0 + hb + c1;
    pl.off[2] = row1 + hb + c0;
    pl.off[3] = row1 + hb + c1;
  }
  pl.rec = xr + (size_t)n * g.CS * g.cbs;
  return pl;
}

__device__ __forceinline__ uint4 hadd_4(const uint4& a, const uint4& b) {
  return make_uint4(hadd2(a.x, b.x), hadd2(a.y, b.y), hadd2(a.z, b.z), hadd2(a.w, b.w));
}
__device__ __forceinline__ uint4 hsub_4(const uint4& a, const uint4& b) {
  return make_uint4(hsub2(a.x, b.x), hsub2(a.y, b.y), hsub2(a.z, b.z), hsub2(a.w, b.w));
}

}  // namespace tp

__global__ void __cluster_dims__(2, 1, 1) __launch_bounds__(tp::NTHREAD, 1)
    twostage_pair_kernel(KernelParam p) {
  using namespace tp;
  extern __shared__ __align__(1024) uint8_t smem_raw[];
  __shared__ Shared sh;
  uint8_t* smem = reinterpret_cast<uint8_t*>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
  Geo g = geo(p);
  g.cbs = (size_t)xr::rows(p.h) * g.RB;           // XR record blocks
  const int warp = warp_id(), lane = lane_id();
  const int rank = (int)cluster_ctarank();
  uint32_t* err = &g_twostage_err;
  const Sched sc = make_sched(g, (int)cluster_id_x(), (int)cluster_count_x());
  const int nst = (g.CS + SK - 1) / SK;

  if (threadIdx.x == 0) {
    for (int s = 0; s < NSTV; ++s) {
      mbar_init(&sh.vfull[s], 2 * NWARP_P);
      mbar_init(&sh.vempty[s], 1);
    }
    for (int a = 0; a < 2; ++a) {
      mbar_init(&sh.accfull[a], 1);
      mbar_init(&sh.accempty[a], 2 * NWARP_E);
    }
    mbar_init(&sh.ufull, 1);
    mbar_init(&sh.uempty, 1);
    mbar_init(&sh.utx, 1);
    mbar_init(&sh.mmadone, 1);
    sh.abort_flag = 0;
    fence_barrier_init();
  }
  if (warp == WARP_MMA) { tmem_alloc_pair(&sh.tmem_base, 512); tmem_relinquish_pair(); }
  tc_fence_before();
  // both CTAs' barriers initialised and TMEM allocated before any remote use
  cluster_sync();
  tc_fence_after();
  const uint32_t tmem = sh.tmem_base;
  volatile int* abort_flag = &sh.abort_flag;
  const uint32_t sbase = smem_u32(smem);
  const uint32_t ubase = sbase, vbase = sbase + U_BYTES;
  // rank 0's barriers, as shared::cluster addresses (the pair's MMA side)
  const uint32_t lead_vfull = mapa_shared(smem_u32(&sh.vfull[0]), 0);
  const uint32_t lead_accempty = mapa_shared(smem_u32(&sh.accempty[0]), 0);
  const uint32_t lead_ufull = mapa_shared(smem_u32(&sh.ufull), 0);

  if (warp == WARP_MMA) {
    // ---- U loads and MMA issue.  Each CTA loads its 128 output channels of
    // U for both taps and all C when the unit's (tap pair, k pair) changes;
    // rank 0 also issues every MMA of the pair (per K-step both taps).
    if (lane == 0) {
      const uint8_t* u2 = static_cast<const uint8_t*>(p.transform_filter);
      const uint32_t idesc = instr_desc(256, 128, 0, 0, 0, 0);
      int cq = -1, ckp = -1;
      uint32_t it = 0, ui = 0, nload = 0;
      bool ok = true;
      for (int i = 0; ok && i < sc.cnt && !*abort_flag; ++i, ++ui) {
        const Unit un = sched_unit(g, sc, i);
        if (un.q != cq || un.kp != ckp) {
          if (cq >= 0) {
            // the old U is free once every MMA issued so far has finished
            if (rank == 0) mma_commit_pair(&sh.uempty, BOTH);
            if (!mbar_wait(&sh.uempty, (nload - 1) & 1, abort_flag, err, ERR_WAIT_EMPTY)) break;
          }
          cq = un.q;
          ckp = un.kp;
          int t[2];
          pair_taps(un.q, t[0], t[1]);
          const int kb = 2 * un.kp + rank;
          const int kbs = kb < g.nKB2 ? kblock2_rows(kb, g.K) : 0;
          mbar_arrive_expect_tx(&sh.utx, (uint32_t)(2 * g.CS * kbs * 32));
          for (int s = 0; s < 2 && kbs > 0; ++s) {
            const uint8_t* src = u2 + u2_piece(t[s], kb, 0, g.K, g.C) * 2;
            uint8_t* dst = smem + s * U_TAP;
            if (kbs == 128) {
              bulk_g2s(dst, src, (uint32_t)(g.CS * U_STEP), &sh.utx);
            } else {
              for (int cs = 0; cs < g.CS; ++cs)
                bulk_g2s(dst + cs * U_STEP, src + (size_t)cs * kbs * 32, (uint32_t)(kbs * 32), &sh.utx);
            }
          }
          if (!mbar_wait(&sh.utx, nload & 1, abort_flag, err, ERR_WAIT_FULL)) break;
          if (rank == 1) {
            mbar_arrive_peer(lead_ufull);
          } else if (!mbar_wait_cluster(&sh.ufull, nload & 1, abort_flag, err, ERR_WAIT_FULL)) {
            break;
          }
          ++nload;
        }
        if (rank != 0) continue;
        const int ab = ui & 1;
        if (ui >= 2 &&
            !mbar_wait_cluster(&sh.accempty[ab], ((ui >> 1) - 1) & 1, abort_flag, err, ERR_WAIT_DRAIN))
          break;
        tc_fence_after();
        const uint32_t d = tmem + ab * 256;
        for (int j = 0; j < nst; ++j, ++it) {
          const int st = it % NSTV;
          if (!mbar_wait_cluster(&sh.vfull[st], (it / NSTV) & 1, abort_flag, err, ERR_WAIT_FULL)) {
            ok = false;
            break;
          }
          tc_fence_after();
          const int nk = min(SK, g.CS - j * SK);
          for (int kk = 0; kk < nk; ++kk) {
            const int cs = j * SK + kk;
#pragma unroll
            for (int s = 0; s < 2; ++s)
              mma_f16_pair(d + s * 128, smem_desc(ubase + s * U_TAP + cs * U_STEP, 128, 256),
                           smem_desc(vbase + st * V_STAGE + (kk * 2 + s) * V_TAP, 128, 256), idesc,
                           cs > 0 ? 1u : 0u);
          }
          mma_commit_pair(&sh.vempty[st], BOTH);
        }
        if (ok) mma_commit_pair(&sh.accfull[ab], BOTH);
      }
      if (rank == 0) {
        // every MMA issued (also on an abort) has finished before TMEM is freed
        mma_commit_pair(&sh.mmadone, 1);
        mbar_wait(&sh.mmadone, 0, nullptr, err, ERR_WAIT_ACCUM);
      }
    }
    __syncwarp();
  } else if (warp < WARP_E0 + NWARP_E) {
    // ---- epilogue: TMEM lane = output channel, columns = the unit's tiles
    const int quarter = warp & 3;
    __half* m16 = static_cast<__half*>(p.mid_result);
    const bool m_aligned32 = (reinterpret_cast<uintptr_t>(m16) & 31) == 0;
    uint32_t ui = 0;
    for (int i = 0; i < sc.cnt; ++i, ++ui) {
      const Unit un = sched_unit(g, sc, i);
      const int ab = ui & 1;
      if (!mbar_wait_warp(&sh.accfull[ab], (ui >> 1) & 1, abort_flag, err, ERR_WAIT_ACCUM, SLEEP_NS)) break;
      tc_fence_after();
      int t[2];
      pair_taps(un.q, t[0], t[1]);
      const int k = (2 * un.kp + rank) * 128 + quarter * 32 + lane;
      const long long rem = g.NT - (long long)un.tb * 128;
      const int ntb = rem < 128 ? (int)rem : 128;
      const uint32_t taddr = tmem + ((uint32_t)(quarter * 32) << 16) + ab * 256;
#pragma unroll 1
      for (int s = 0; s < 2; ++s) {
        const int kk = k < g.K ? k : 0;
#pragma unroll 1
        for (int c0 = 0; c0 < 128; c0 += 32) {
          float v[32];
          tmem_ld16(taddr + s * 128 + c0, v);
          tmem_ld16(taddr + s * 128 + c0 + 16, v + 16);
          tmem_ld_wait();
          if (k >= g.K || c0 >= ntb) continue;
          if (ntb == 128) {
            uint32_t h[16];
#pragma unroll
            for (int i2 = 0; i2 < 16; ++i2) {
              const __half2 x = __floats2half2_rn(v[2 * i2], v[2 * i2 + 1]);
              h[i2] = *reinterpret_cast<const uint32_t*>(&x);
            }
            // 32 bytes per lane and store, whole sectors (a full block's rows
            // are 256-byte multiples from a 32-byte aligned mid_result)
            __half* dst = m16 + m_offset(un.tb, t[s], kk, c0, g.K, g.NT);
            if (m_aligned32) {
#pragma unroll
              for (int o = 0; o < 2; ++o) st_global_v8(dst + 16 * o, h + 8 * o);
            } else {
#pragma unroll
              for (int o = 0; o < 4; ++o)
                reinterpret_cast<uint4*>(dst)[o] = make_uint4(h[4 * o], h[4 * o + 1], h[4 * o + 2], h[4 * o + 3]);
            }
          } else {
            __half* row = m16 + m_offset(un.tb, t[s], kk, 0, g.K, g.NT);
#pragma unroll
            for (int i2 = 0; i2 < 32; ++i2)
              if (c0 + i2 < ntb) row[c0 + i2] = __float2half_rn(v[i2]);
          }
        }
      }
      tc_fence_before();
      __syncwarp();
      if (lane == 0) mbar_arrive_peer(lead_accempty + ab * 8);
    }
  } else {
    // ---- V producers: thread = (tile tl of this CTA's 64, channel half hh,
    // K-step kq of each stage); a warp's loads of one word cover 32 tiles'
    // consecutive 16-byte entries.  V of (a, 1), (a, 2) is R(col 2tx) +
    // R(2tx + 1) and R(2tx + 1) - R(2tx); V of (a, b) for b = 0, 3 is R(first
    // column of b) - R(second), one fp16 rounding each.
    const int pw = warp - WARP_P0;
    const int tl = (pw & 1) * 32 + lane, hh = (pw >> 1) & 1, kq = pw >> 2;
    const uint8_t* xr = static_cast<const uint8_t*>(p.transform_pin);
    // The load cursor (lu, lj) runs RING - 1 stages ahead of the consume
    // cursor (cu, cj), the loads of those stages in flight in a register
    // ring; everything a unit needs is worked out when the load cursor enters
    // it.  The consume side keeps, per unit index mod 4 (4 bits each; the
    // cursors are at most RING - 1 units apart), whether the tile exists and
    // whether the pair reads four words.
    int lu = 0, cu = 0, lj = 0, cj = 0;
    uint32_t info = 0;
    ProdLoad pl;
    pl.rec = xr;
    pl.live = false;
    pl.four = false;
    const size_t step_bytes = (size_t)SK * g.cbs;
    uint4 w0[4], w1[4], w2[4], w3[4];
    auto issue = [&](uint4 (&w)[4]) {
      if (lu >= sc.cnt) return;
      if (lj == 0) {
        pl = prod_load(g, xr, sched_unit(g, sc, lu), rank, tl, hh);
        pl.rec += (size_t)kq * g.cbs;
        const uint32_t sh4 = (uint32_t)(lu & 3) * 4;
        info = (info & ~(15u << sh4)) | ((uint32_t)((pl.live ? 1 : 0) | (pl.four ? 2 : 0)) << sh4);
      }
      if (pl.live && lj * SK + kq < g.CS) {
        w[0] = WINO_PAIR_LOAD(reinterpret_cast<const uint4*>(pl.rec + pl.off[0]));
        w[1] = WINO_PAIR_LOAD(reinterpret_cast<const uint4*>(pl.rec + pl.off[1]));
        if (pl.four) {
          w[2] = WINO_PAIR_LOAD(reinterpret_cast<const uint4*>(pl.rec + pl.off[2]));
          w[3] = WINO_PAIR_LOAD(reinterpret_cast<const uint4*>(pl.rec + pl.off[3]));
        }
      }
      pl.rec += step_bytes;
      if (++lj == nst) { lj = 0; ++lu; }
    };
    uint32_t it = 0;
    auto consume = [&](const uint4 (&w)[4]) -> bool {
      const int st = it % NSTV;
      if (it >= NSTV &&
          !mbar_wait_warp(&sh.vempty[st], (it / NSTV - 1) & 1, abort_flag, err, ERR_WAIT_EMPTY, SLEEP_NS))
        return false;
      const uint32_t inf = (info >> ((uint32_t)(cu & 3) * 4)) & 15u;
      if ((inf & 1u) && cj * SK + kq < g.CS) {
        uint4 v0, v1;
        if (inf & 2u) {
          v0 = hsub_4(w[0], w[1]);
          v1 = hsub_4(w[2], w[3]);
        } else {
          v0 = hadd_4(w[0], w[1]);   // b = 1: d1 + d2
          v1 = hsub_4(w[1], w[0]);   // b = 2: d2 - d1
        }
        uint8_t* dst = smem + U_BYTES + st * V_STAGE + (kq * 2) * V_TAP + (tl >> 3) * 256 + hh * 128 +
                       (tl & 7) * 16;
        *reinterpret_cast<uint4*>(dst) = v0;
        *reinterpret_cast<uint4*>(dst + V_TAP) = v1;
      }
      fence_proxy_async_shared();
      __syncwarp();
      if (lane == 0) mbar_arrive_peer(lead_vfull + st * 8);
      ++it;
      if (++cj == nst) { cj = 0; ++cu; }
      return cu < sc.cnt && !*abort_flag;
    };
    static_assert(RING == 4, "the ring below is written out for four slots");
    issue(w0);
    issue(w1);
    issue(w2);
    while (cu < sc.cnt && !*abort_flag) {
      issue(w3);
      if (!consume(w0)) break;
      issue(w0);
      if (!consume(w1)) break;
      issue(w1);
      if (!consume(w2)) break;
      issue(w2);
      if (!consume(w3)) break;
    }
  }
  tc_fence_before();
  __syncthreads();
  // the peer may still read this CTA's shared memory or arrive on its
  // barriers until both CTAs get here
  cluster_sync();
  if (warp == WARP_MMA) {
    tc_fence_after();
    tmem_dealloc_pair(tmem, 512);
  }
}

// =============================================================================
// One-tap GEMM with streamed U (any C)
// =============================================================================
namespace tsk {

using namespace ts;

constexpr int NSTAGE = 4;
constexpr int SK = 4;                         // K-steps (16 channels) per stage
constexpr int KPU = 2;                        // 128-row k-blocks per unit
constexpr int A_STEP = 128 * 16 * 2;          // 4 KB: V of 128 tiles x 16 channels (K-major)
constexpr int B_STEP = KB2 * 16 * 2;          // 4 KB: U of one 128-row k-block
constexpr int STAGE_A = SK * A_STEP;
constexpr int STAGE_B = SK * B_STEP;
constexpr int STAGE_BYTES = STAGE_A + KPU * STAGE_B;
constexpr int SMEM_BYTES = NSTAGE * STAGE_BYTES + 1024;
constexpr int WARP_U = 0, WARP_MMA = 1, WARP_E0 = 2, NWARP_E = 4, WARP_P0 = 6, NWARP_P = 8;
constexpr uint32_t SLEEP_EPI_NS = 32, SLEEP_PROD_NS = 32;
constexpr int NTHREAD = (WARP_P0 + NWARP_P) * 32;

struct Shared {
  uint64_t full[NSTAGE], empty[NSTAGE];
  uint64_t accfull[2], accempty[2];
  uint64_t mmadone;
  uint32_t tmem_base;
  int abort_flag;
};

__device__ __forceinline__ long long nunits(const Geo& g) { return 16LL * g.nTB * ((g.nKB2 + KPU - 1) / KPU); }

// Unit u -> tap t (fastest), k-block pair, tile block; kbs[i] = rows of the
// pair's i-th k-block (0 when absent).
__device__ __forceinline__ void unit_coords(const Geo& g, long long u, int& t, int& tb, int& kb,
                                            int (&kbs)[KPU]) {
  const int nKP = (g.nKB2 + KPU - 1) / KPU;
  t = (int)(u & 15);
  const long long r = u >> 4;
  const int kp = (int)(r % nKP);
  tb = (int)(r / nKP);
  kb = kp * KPU;
#pragma unroll
  for (int i = 0; i < KPU; ++i) kbs[i] = kb + i < g.nKB2 ? kblock2_rows(kb + i, g.K) : 0;
}

struct ProdUnit {
  const uint8_t* xn;
  uint32_t o[4];
  uint32_t sa0, sa1, sb0, sb1;
  bool live;
};

__device__ __forceinline__ ProdUnit prod_unit(const Geo& g, const uint8_t* xb, int t, int tb, int tl, int hh) {
  ProdUnit pu;
  const long long tile = (long long)tb * 128 + tl;
  pu.live = tile < g.NT;
  int n = 0, ty = 0, tx = 0;
  if (pu.live) tile_decode(g, tile, n, ty, tx);
  int i0, i1, j0, j1;
  bt_pick(t >> 2, i0, i1, pu.sa0, pu.sa1);
  bt_pick(t & 3, j0, j1, pu.sb0, pu.sb1);
  pu.o[0] = win_off(g, ty, tx, hh, i0, j0);
  pu.o[1] = win_off(g, ty, tx, hh, i0, j1);
  pu.o[2] = win_off(g, ty, tx, hh, i1, j0);
  pu.o[3] = win_off(g, ty, tx, hh, i1, j1);
  pu.xn = xb + (size_t)n * g.CS * g.cbs;
  return pu;
}

}  // namespace tsk

__global__ void __launch_bounds__(tsk::NTHREAD, 1) twostage_stream_kernel(KernelParam p) {
  using namespace tsk;
  extern __shared__ __align__(1024) uint8_t smem_raw[];
  __shared__ Shared sh;
  uint8_t* smem = reinterpret_cast<uint8_t*>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
  const Geo g = geo(p);
  const int warp = warp_id(), lane = lane_id();
  uint32_t* err = &g_twostage_err;
  const long long NU = nunits(g);
  const int nst = (g.CS + SK - 1) / SK;

  if (threadIdx.x == 0) {
    for (int s = 0; s < NSTAGE; ++s) {
      mbar_init(&sh.full[s], 1 + NWARP_P);
      mbar_init(&sh.empty[s], 1);
    }
    for (int a = 0; a < 2; ++a) {
      mbar_init(&sh.accfull[a], 1);
      mbar_init(&sh.accempty[a], NWARP_E);
    }
    mbar_init(&sh.mmadone, 1);
    sh.abort_flag = 0;
    fence_barrier_init();
  }
  if (warp == WARP_MMA) { tmem_alloc(&sh.tmem_base, 512); tmem_relinquish(); }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = sh.tmem_base;
  volatile int* abort_flag = &sh.abort_flag;
  const uint32_t sbase = smem_u32(smem);

  if (warp == WARP_U) {
    if (lane == 0) {
      const uint8_t* u2 = static_cast<const uint8_t*>(p.transform_filter);
      uint32_t it = 0;
      bool ok = true;
      for (long long u = blockIdx.x; ok && u < NU && !*abort_flag; u += gridDim.x) {
        int t, tb, kb, kbs[KPU];
        unit_coords(g, u, t, tb, kb, kbs);
        for (int j = 0; j < nst; ++j, ++it) {
          const int st = it % NSTAGE;
          if (it >= NSTAGE &&
              !mbar_wait(&sh.empty[st], (it / NSTAGE - 1) & 1, abort_flag, err, ERR_WAIT_EMPTY)) {
            ok = false;
            break;
          }
          const int nk = min(SK, g.CS - j * SK);
          uint32_t tx = 0;
#pragma unroll
          for (int i = 0; i < KPU; ++i) tx += nk * kbs[i] * 32;
          mbar_arrive_expect_tx(&sh.full[st], tx);
#pragma unroll
          for (int i = 0; i < KPU; ++i)
            if (kbs[i])
              bulk_g2s(smem + st * STAGE_BYTES + STAGE_A + i * STAGE_B,
                       u2 + u2_piece(t, kb + i, j * SK, g.K, p.c) * 2, nk * kbs[i] * 32, &sh.full[st]);
        }
      }
      if (*abort_flag) __nanosleep(20000);
    }
    __syncwarp();
  } else if (warp == WARP_MMA) {
    if (lane == 0) {
      uint32_t it = 0, ui = 0;
      bool ok = true;
      for (long long u = blockIdx.x; ok && u < NU && !*abort_flag; u += gridDim.x, ++ui) {
        int t, tb, kb, kbs[KPU];
        unit_coords(g, u, t, tb, kb, kbs);
        uint32_t idesc[KPU];
#pragma unroll
        for (int i = 0; i < KPU; ++i) idesc[i] = instr_desc(128, kbs[i] ? kbs[i] : 16, 0, 0, 0, 0);
        const int ab = ui & 1;
        if (ui >= 2 && !mbar_wait(&sh.accempty[ab], ((ui >> 1) - 1) & 1, abort_flag, err, ERR_WAIT_DRAIN))
          break;
        tc_fence_after();
        const uint32_t d = tmem + ab * (KPU * 128);
        for (int j = 0; j < nst; ++j, ++it) {
          const int st = it % NSTAGE;
          if (!mbar_wait(&sh.full[st], (it / NSTAGE) & 1, abort_flag, err, ERR_WAIT_FULL)) {
            ok = false;
            break;
          }
          tc_fence_after();
          const int nk = min(SK, g.CS - j * SK);
          const uint32_t a0 = sbase + st * STAGE_BYTES;
          for (int kk = 0; kk < nk; ++kk) {
            const uint64_t adesc = smem_desc(a0 + kk * A_STEP, 128, 256);
#pragma unroll
            for (int i = 0; i < KPU; ++i)
              if (kbs[i])
                mma_f16(d + i * 128, adesc, smem_desc(a0 + STAGE_A + i * STAGE_B + kk * kbs[i] * 32, 128, 256),
                        idesc[i], (j > 0 || kk > 0) ? 1u : 0u);
          }
          mma_commit(&sh.empty[st]);
        }
        if (ok) mma_commit(&sh.accfull[ab]);
      }
      // every MMA issued (also on an abort) has finished before TMEM is freed
      mma_commit(&sh.mmadone);
      mbar_wait(&sh.mmadone, 0, nullptr, err, ERR_WAIT_ACCUM);
    }
    __syncwarp();
  } else if (warp < WARP_E0 + NWARP_E) {
    // epilogue: TMEM lanes 32*quarter .. +31 = tiles of the block
    const int quarter = warp & 3;
    __half* m16 = static_cast<__half*>(p.mid_result);
    uint32_t ui = 0;
    for (long long u = blockIdx.x; u < NU; u += gridDim.x, ++ui) {
      int t, tb, kb, kbs[KPU];
      unit_coords(g, u, t, tb, kb, kbs);
      const int ab = ui & 1;
      if (!mbar_wait_warp(&sh.accfull[ab], (ui >> 1) & 1, abort_flag, err, ERR_WAIT_ACCUM, SLEEP_EPI_NS)) break;
      tc_fence_after();
      const int i = quarter * 32 + lane;   // tile within the block
      const bool live = (long long)tb * 128 + i < g.NT;
      const uint32_t taddr = tmem + ((uint32_t)(quarter * 32) << 16) + ab * (KPU * 128);
      // rows of the block are ntb elements apart: one base pointer per unit
      const long long rem = g.NT - (long long)tb * 128;
      const int ntb = rem < 128 ? (int)rem : 128;
      __half* mrow = m16 + m_offset(tb, t, kb * KB2, i, g.K, g.NT);
      for (int cc = 0; cc < KPU * 128; cc += 32) {
        const int kbi = cc >> 7, c0 = cc & 127;
        if (c0 >= kbs[kbi]) continue;
        // K is a multiple of 16: the second half exists when c0 + 16 < rows
        const bool two = c0 + 16 < kbs[kbi];
        float v[32];
        tmem_ld16(taddr + cc, v);
        if (two) tmem_ld16(taddr + cc + 16, v + 16);
        tmem_ld_wait();
        if (live) {
          __half* dst = mrow + (size_t)cc * ntb;
#pragma unroll
          for (int jj = 0; jj < 16; ++jj) dst[(size_t)jj * ntb] = __float2half_rn(v[jj]);
          if (two) {
#pragma unroll
            for (int jj = 16; jj < 32; ++jj) dst[(size_t)jj * ntb] = __float2half_rn(v[jj]);
          }
        }
      }
      tc_fence_before();
      __syncwarp();
      if (lane == 0) mbar_arrive(&sh.accempty[ab]);
    }
  } else {
    // V producers: thread = (tile tl of the unit's 128-tile block, channel half hh).
    const int pw = warp - WARP_P0;
    const int tl = (pw & 3) * 32 + lane, hh = pw >> 2;
    const uint8_t* xb = static_cast<const uint8_t*>(p.transform_pin);
    uint32_t it = 0;
    bool ok = true;
    for (long long u = blockIdx.x; ok && u < NU && !*abort_flag; u += gridDim.x) {
      int t, tb, kb, kbs[KPU];
      unit_coords(g, u, t, tb, kb, kbs);
      const ProdUnit pu = prod_unit(g, xb, t, tb, tl, hh);
      for (int j = 0; j < nst; ++j, ++it) {
        const int st = it % NSTAGE;
        const int nk = min(SK, g.CS - j * SK);
        // the window loads go out before the wait for a free stage: only the
        // shared-memory stores below need it
        uint4 d[SK][4];
#pragma unroll
        for (int kk = 0; kk < SK; ++kk) {
          if (pu.live && kk < nk) {
            const uint8_t* rec = pu.xn + (size_t)(j * SK + kk) * g.cbs;
#pragma unroll
            for (int w = 0; w < 4; ++w) d[kk][w] = __ldg(reinterpret_cast<const uint4*>(rec + pu.o[w]));
          } else {
#pragma unroll
            for (int w = 0; w < 4; ++w) d[kk][w] = make_uint4(0u, 0u, 0u, 0u);
          }
        }
        if (it >= NSTAGE &&
            !mbar_wait_warp(&sh.empty[st], (it / NSTAGE - 1) & 1, abort_flag, err, ERR_WAIT_EMPTY,
                            SLEEP_PROD_NS)) {
          ok = false;
          break;
        }
        uint8_t* adst = smem + st * STAGE_BYTES + (tl >> 3) * 256 + hh * 128 + (tl & 7) * 16;
#pragma unroll
        for (int kk = 0; kk < SK; ++kk) {
          if (kk < nk) {
            // rows first (e_jc = sa0*d[i0][jc] + sa1*d[i1][jc]), then columns
            *reinterpret_cast<uint4*>(adst + kk * A_STEP) =
                bt_op4(pu.sb0, pu.sb1, bt_op4(pu.sa0, pu.sa1, d[kk][0], d[kk][2]),
                       bt_op4(pu.sa0, pu.sa1, d[kk][1], d[kk][3]));
          }
        }
        fence_proxy_async_shared();
        __syncwarp();
        if (lane == 0) mbar_arrive(&sh.full[st]);
      }
    }
  }
  tc_fence_before();
  __syncthreads();
  if (warp == WARP_MMA) {
    tc_fence_after();
    tmem_dealloc(tmem, 512);
  }
}

// =============================================================================
// One-tap GEMM with resident U on row-transformed input (C <= 256)
// =============================================================================
// The streamed-U kernel's unit (one tap x 128 tiles x two 128-row k-blocks,
// two M = 128 MMAs per K-step sharing the tile operand), with the two
// per-unit streams it pays for removed:
//  - U: each CTA serves one (tap, k pair) "combo" and keeps that combo's U
//    (both k-blocks, all C: at most 128 KB) in shared memory, loaded once;
//    the CTAs of a combo take its tile blocks round-robin (j, j + s, ...),
//    so all combos sweep the tile blocks at the same pace and the input rows
//    of a tile block are read by its 16 taps from L2 within a short window.
//  - input words: V of tap (a, b) is one fp16 add / subtract of two XR words
//    (the row step already applied by the pre-pass), 2 loads per V word
//    instead of the 4 window words of XB.
// Each producer thread keeps RING - 1 stages of window loads in flight in a
// register ring while it stores one.
namespace trs {

using namespace ts;

#ifndef WINO_RES_NSTAGE
#define WINO_RES_NSTAGE 5
#endif
// Load instruction of the producers' window words (__ldg: through L1).
#ifndef WINO_RES_LOAD
#define WINO_RES_LOAD __ldg
#endif
constexpr int NSTAGE = WINO_RES_NSTAGE;
constexpr int SK = 4;                         // K-steps (16 channels) per stage
constexpr int KPU = 2;                        // 128-row k-blocks per unit
constexpr int CS_MAX = 16;                    // resident U holds up to 16 K-steps (C <= 256)
constexpr int A_STEP = 128 * 16 * 2;          // 4 KB: V of 128 tiles x 16 channels
constexpr int STAGE_A = SK * A_STEP;          // 16 KB
// U of the unit's k pair, K-step major: K-step cs holds its 256 k rows (the
// two k-blocks' row groups back to back) at cs * U_CS, so one N = 256 MMA
// reads both k-blocks
constexpr int U_CS = KPU * KB2 * 16 * 2;      // 8 KB
constexpr int U_BYTES = CS_MAX * U_CS;        // 128 KB
constexpr int SMEM_BYTES = U_BYTES + NSTAGE * STAGE_A + 1024;
// Four warpgroups: warps 0-3 epilogue (warp w reads TMEM lanes 32 w ..),
// warp 4 lane 0 U loads and MMA issue (warps 5-7 idle), warps 8-15 V
// producers.  The block launches with 128 registers a thread (512 threads,
// the whole register file); the epilogue and MMA warpgroups then give
// registers up to the producers, whose window-load ring they hold:
// 128 x 104 + 128 x 56 + 256 x 176 = 65536.
constexpr int WARP_E0 = 0, NWARP_E = 4, WARP_MMA = 4, WARP_LOAD = 5, WARP_P0 = 8, NWARP_P = 8;
constexpr int NTHREAD = (WARP_P0 + NWARP_P) * 32;
constexpr int NTHREAD_V = WARP_P0 * 32;       // bulk-copy-fed variant: no producer warps
constexpr int REGS_LAUNCH = 128, REGS_EPI = 104, REGS_MMA = 56, REGS_PROD = 176;
static_assert(128 * REGS_EPI + 128 * REGS_MMA + 256 * REGS_PROD == NTHREAD * REGS_LAUNCH,
              "the warpgroups' register limits add up to the launch allocation");
static_assert(NTHREAD * REGS_LAUNCH == 65536, "the block holds the whole register file");
constexpr uint32_t SLEEP_NS = 32;
// producer register ring: stages of window loads held in registers (the
// loads of RING - 1 stages are in flight while one stage is stored)
#ifndef WINO_RES_RING
#define WINO_RES_RING 4
#endif
constexpr int RING = WINO_RES_RING;
static_assert(RING >= 2 && RING <= 4, "ring of two to four stages");

struct Shared {
  uint64_t full[NSTAGE], empty[NSTAGE];
  uint64_t accfull[2], accempty[2];
  uint64_t ufull, uempty, mmadone;
  uint32_t tmem_base;
  int abort_flag;
};

// Combos: c = t * nKP + kp.  With at least as many CTAs G as combos, combo c
// gets s = G / ncombo CTAs (one more for the first G % ncombo combos) and its
// j-th CTA takes the tile blocks j, j + s, ...; with fewer, CTA g takes the
// combos g, g + G, ... whole, one after another.  Unit indices fit 32 bits
// (the host bounds the tile count).
struct Sched {
  int combo, j, s, G, cnt;
};

__device__ __forceinline__ Sched make_sched(int ncombo, int nTB, int cl, int G) {
  Sched sc;
  sc.G = G;
  if (G < ncombo) {
    const int mc = cl < ncombo ? (ncombo - cl + G - 1) / G : 0;
    sc.combo = cl;
    sc.j = 0;
    sc.s = 1;
    sc.cnt = mc * nTB;
    return sc;
  }
  const int base = G / ncombo, extra = G - base * ncombo;
  const int big = extra * (base + 1);
  if (cl < big) {
    sc.combo = cl / (base + 1);
    sc.j = cl - sc.combo * (base + 1);
    sc.s = base + 1;
  } else {
    const int r = cl - big;
    sc.combo = extra + r / base;
    sc.j = r - (r / base) * base;
    sc.s = base;
  }
  sc.cnt = sc.j < nTB ? (nTB - sc.j + sc.s - 1) / sc.s : 0;
  return sc;
}

struct Unit {
  int combo, t, kp, tb;
};

// Tile blocks are taken in decreasing order: the pre-pass writes them in
// increasing order, so the most recently written, still in L2, come first.
__device__ __forceinline__ Unit sched_unit(const Geo& g, const Sched& sc, int i) {
  Unit x;
  const int ncombo = 16 * g.nKP;
  int r;
  if (sc.G < ncombo) {
    const int m = i / g.nTB;
    x.combo = sc.combo + m * sc.G;
    r = i - m * g.nTB;
  } else {
    x.combo = sc.combo;
    r = sc.j + i * sc.s;
  }
  x.tb = g.nTB - 1 - r;
  x.t = x.combo / g.nKP;
  x.kp = x.combo - x.t * g.nKP;
  return x;
}

// Producer side of one unit for thread (tile tl, channel half hh): V of tap
// (a, b) is x op y of the XR words at byte offsets ox, oy of row (ty, a):
//   b = 0: R(2tx - 1) - R(2tx + 1)    (par 1 entries tx, tx + 1)
//   b = 1: R(2tx) + R(2tx + 1)        (par 0 entry tx, par 1 entry tx + 1)
//   b = 2: R(2tx + 1) - R(2tx)
//   b = 3: R(2tx) - R(2tx + 2)        (par 0 entries tx, tx + 1)
// (the B^T columns d0 - d2, d1 + d2, d2 - d1, d1 - d3 over the window
// columns 2tx - 1 ..), one fp16 rounding as in the fused kernel.
struct Prod {
  const uint8_t* rec;  // XR of the tile's image, channel block 0
  uint32_t ox, oy;
  bool live, add;
};

__device__ __forceinline__ Prod prod(const Geo& g, const uint8_t* xr, int t, int tb, int tl, int hh) {
  Prod pr;
  const int tile = tb * 128 + tl;
  pr.live = tile < (int)g.NT;
  int n = 0, ty = 0, tx = 0;
  if (pr.live) {
    const int per = g.TP * g.TQ;
    n = tile / per;
    const int r = tile - n * per;
    ty = r / g.TQ;
    tx = r - ty * g.TQ;
  }
  const int a = t >> 2, b = t & 3;
  const uint32_t E = (uint32_t)g.E;
  const uint32_t row = (uint32_t)(4 * ty + a) * g.RB + (uint32_t)(hh * E) * 16;
  const uint32_t p0 = row + (uint32_t)tx * 16, p1 = row + (2 * E + (uint32_t)tx) * 16;
  switch (b) {
    case 0: pr.ox = p1; pr.oy = p1 + 16; break;
    case 1: pr.ox = p0; pr.oy = p1 + 16; break;
    case 2: pr.ox = p1 + 16; pr.oy = p0; break;
    default: pr.ox = p0; pr.oy = p0 + 16; break;
  }
  pr.add = b == 1;
  pr.rec = xr + (size_t)n * g.CS * g.cbs;
  return pr;
}

}  // namespace trs

// TMAV false: V formed by the producer warps from XR (transform_pin).
// TMAV true: V read by bulk copy from the transformed tiles V2 in
// transform_pin (v2_layout_kernel); warp 5 lane 0 issues the copies and no
// producer warps run.
// F8 (with TMAV): the fp8 hi+lo variant.  V2 and U hold e4m3 hi and lo
// terms (x = hi + lo to about 8 bits), 32 channels per K-step, the two terms
// of a K-step back to back (so a K-step's two pieces take the place of two
// fp16 K-steps' pieces: loader and stages are unchanged); per K-step three
// kind::f8f6f4 MMAs accumulate hi.hi + lo.hi + hi.lo; the per-input-channel
// V scale is folded into U, and the epilogue multiplies by the per-(tap,
// output channel) U scale su (p.pweight, fp32 [16][K]) before rounding M.
// F8 = 1: single e4m3 terms (one MMA per K-step, one byte per tile and
// channel, a K-step of 32 channels per piece).
template <bool TMAV, int F8 = 0>
__global__ void __launch_bounds__(TMAV ? trs::NTHREAD_V : trs::NTHREAD, 1) twostage_res_kernel_t(KernelParam p) {
  static_assert(F8 == 0 || TMAV, "the fp8 variants read V2 by bulk copy");
  constexpr int TERMS = F8 == 1 ? 1 : 2;        // bytes per tile and channel in V2 and U
  using namespace trs;
  extern __shared__ __align__(1024) uint8_t smem_raw[];
  __shared__ Shared sh;
  uint8_t* smem = reinterpret_cast<uint8_t*>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
  Geo g = geo(p);
  g.cbs = (size_t)xr::rows(p.h) * g.RB;           // XR record blocks
  const int warp = warp_id(), lane = lane_id();
  uint32_t* err = &g_twostage_err;
  const Sched sc = make_sched(16 * g.nKP, g.nTB, (int)blockIdx.x, (int)gridDim.x);
  // pieces of rows x 32 bytes per unit: 16-channel steps (fp16), K-step
  // terms (fp8 hi+lo: two per 32 channels), K-steps (single fp8)
  const int npc = F8 == 1 ? g.C / 32 : g.CS;
  const int nst = (npc + SK - 1) / SK;

  if (threadIdx.x == 0) {
    for (int s = 0; s < NSTAGE; ++s) {
      mbar_init(&sh.full[s], TMAV ? 1 : NWARP_P);
      mbar_init(&sh.empty[s], 1);
    }
    for (int a = 0; a < 2; ++a) {
      mbar_init(&sh.accfull[a], 1);
      mbar_init(&sh.accempty[a], NWARP_E);
    }
    mbar_init(&sh.ufull, 1);
    mbar_init(&sh.uempty, 1);
    mbar_init(&sh.mmadone, 1);
    sh.abort_flag = 0;
    fence_barrier_init();
  }
  if (warp == WARP_MMA) { tmem_alloc(&sh.tmem_base, 512); tmem_relinquish(); }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = sh.tmem_base;
  volatile int* abort_flag = &sh.abort_flag;
  const uint32_t sbase = smem_u32(smem);
  // each role sets its warpgroup's register limit first thing in its branch
  if (warp >= WARP_MMA && warp < WARP_P0) {
    if constexpr (!TMAV) regs_dec<REGS_MMA>();
    if (TMAV && warp == WARP_LOAD && lane == 0) {
      // V2 loader: stage j of a unit is K-steps j*SK .. of the unit's tile
      // block and tap; a full block's pieces (4 KB each) are contiguous, a
      // partial block's pieces (rows * 32 bytes) go one by one to their
      // 4 KB slots
      const uint8_t* v2 = static_cast<const uint8_t*>(p.transform_pin);
      const int NT8 = ((int)g.NT + 7) & ~7;
      uint32_t it = 0;
      for (int i = 0; i < sc.cnt && !*abort_flag; ++i) {
        const Unit un = sched_unit(g, sc, i);
        const int rows = min(128, NT8 - un.tb * 128);
        // TERMS bytes per tile and channel: fp16 or the fp8 hi and lo terms (2), single fp8 (1)
        const uint8_t* src = v2 + ((size_t)un.t * NT8 + (size_t)un.tb * 128) * g.C * TERMS;
        bool ok = true;
        for (int j = 0; j < nst; ++j, ++it) {
          const int st = it % NSTAGE;
          if (it >= NSTAGE &&
              !mbar_wait(&sh.empty[st], (it / NSTAGE - 1) & 1, abort_flag, err, ERR_WAIT_EMPTY)) {
            ok = false;
            break;
          }
          const int nk = min(SK, npc - j * SK);
          const uint32_t piece = (uint32_t)(rows * 32);
          mbar_arrive_expect_tx(&sh.full[st], (uint32_t)nk * piece);
          uint8_t* dst = smem + U_BYTES + st * STAGE_A;
          const uint8_t* sp = src + (size_t)j * SK * piece;
          if (rows == 128) {
            bulk_g2s(dst, sp, (uint32_t)nk * piece, &sh.full[st]);
          } else {
            for (int kk = 0; kk < nk; ++kk) bulk_g2s(dst + kk * A_STEP, sp + (size_t)kk * piece, piece, &sh.full[st]);
          }
        }
        if (!ok) break;
      }
      // copies still in flight land before the CTA leaves (on an abort the
      // MMA side may not have waited for them)
      for (uint32_t s2 = it > (uint32_t)NSTAGE ? it - NSTAGE : 0; s2 < it; ++s2)
        mbar_wait(&sh.full[s2 % NSTAGE], (s2 / NSTAGE) & 1, nullptr, err, ERR_WAIT_FULL);
    }
    if (warp == WARP_MMA && lane == 0) {
      const uint8_t* u2 = static_cast<const uint8_t*>(p.transform_filter);
      int cur = -1;
      uint32_t it = 0, nload = 0;
      bool ok = true;
      for (int i = 0; ok && i < sc.cnt && !*abort_flag; ++i) {
        const Unit un = sched_unit(g, sc, i);
        const int kb = un.kp * KPU;
        int kbs[KPU];
#pragma unroll
        for (int q = 0; q < KPU; ++q) kbs[q] = kb + q < g.nKB2 ? kblock2_rows(kb + q, g.K) : 0;
        if (un.combo != cur) {
          if (cur >= 0) {
            // the old U is free once every MMA issued so far has finished
            mma_commit(&sh.uempty);
            if (!mbar_wait(&sh.uempty, (nload - 1) & 1, abort_flag, err, ERR_WAIT_EMPTY)) break;
          }
          cur = un.combo;
          uint32_t bytes = 0;
#pragma unroll
          for (int q = 0; q < KPU; ++q) bytes += (uint32_t)(kbs[q] * g.C * TERMS);
          mbar_arrive_expect_tx(&sh.ufull, bytes);
          if constexpr (F8 != 0) {
            // the combo's [K-step][term][rows x 32 B] block is contiguous
            bulk_g2s(smem, u2 + ((size_t)un.t * g.K + (size_t)un.kp * 2 * KB2) * g.C * TERMS, bytes, &sh.ufull);
          } else {
            for (int cs = 0; cs < g.CS; ++cs)
#pragma unroll
              for (int q = 0; q < KPU; ++q)
                if (kbs[q])
                  bulk_g2s(smem + cs * U_CS + q * (KB2 * 32), u2 + u2_piece(un.t, kb + q, cs, g.K, g.C) * 2,
                           (uint32_t)(kbs[q] * 32), &sh.ufull);
          }
          if (!mbar_wait(&sh.ufull, nload & 1, abort_flag, err, ERR_WAIT_FULL)) break;
          ++nload;
        }
        // one MMA per K-step: M = 128 tiles, N = the k pair's rows (<= 256);
        // V2 and the producers' V share the K-major tile-operand layout
        const uint32_t idesc = instr_desc(128, (uint32_t)(kbs[0] + kbs[1]), 0, 0, 0, 0);
        const int ab = i & 1;
        if (i >= 2 && !mbar_wait(&sh.accempty[ab], ((i >> 1) - 1) & 1, abort_flag, err, ERR_WAIT_DRAIN)) break;
        tc_fence_after();
        const uint32_t d = tmem + ab * (KPU * 128);
        // descriptors advance by adding the byte step >> 4 to the address field
        const uint64_t bdesc0 = smem_desc(sbase, 128, 256);
        for (int j = 0; j < nst; ++j, ++it) {
          const int st = it % NSTAGE;
          if (!mbar_wait(&sh.full[st], (it / NSTAGE) & 1, abort_flag, err, ERR_WAIT_FULL)) {
            ok = false;
            break;
          }
          tc_fence_after();
          const int nk = min(SK, npc - j * SK);
          const uint64_t adesc = smem_desc(sbase + U_BYTES + st * STAGE_A, 128, 256);
          if constexpr (F8 == 1) {
            const uint32_t step = (uint32_t)(kbs[0] + kbs[1]) * 32 >> 4;   // one K-step of U
            for (int kk = 0; kk < nk; ++kk)
              mma_f8(d, adesc + (uint64_t)(kk * (A_STEP >> 4)), bdesc0 + (uint64_t)(j * SK + kk) * step, idesc,
                     (j > 0 || kk > 0) ? 1u : 0u);
            mma_commit(&sh.empty[st]);
            continue;
          }
          if constexpr (F8 == 2) {
            // nk pieces = nk / 2 K-steps of 32 channels, each hi then lo
            const uint32_t rk = (uint32_t)(kbs[0] + kbs[1]);
            const uint32_t term = rk * 32 >> 4;        // descriptor step between the terms of U
            for (int kk = 0; kk < nk / 2; ++kk) {
              const int cs32 = j * (SK / 2) + kk;
              const uint64_t ah = adesc + (uint64_t)(2 * kk * (A_STEP >> 4)), al = ah + (uint64_t)(A_STEP >> 4);
              const uint64_t bh = bdesc0 + (uint64_t)(2 * cs32) * term, bl = bh + term;
              mma_f8(d, ah, bh, idesc, (j > 0 || kk > 0) ? 1u : 0u);
              mma_f8(d, al, bh, idesc, 1u);
              mma_f8(d, ah, bl, idesc, 1u);
            }
            mma_commit(&sh.empty[st]);
            continue;
          }
          const uint64_t bdesc = bdesc0 + (uint64_t)(j * SK * (U_CS >> 4));
          if (nk == SK) {
#pragma unroll
            for (int kk = 0; kk < SK; ++kk)
              mma_f16(d, adesc + (uint64_t)(kk * (A_STEP >> 4)), bdesc + (uint64_t)(kk * (U_CS >> 4)), idesc,
                      (j > 0 || kk > 0) ? 1u : 0u);
          } else {
            for (int kk = 0; kk < nk; ++kk)
              mma_f16(d, adesc + (uint64_t)(kk * (A_STEP >> 4)), bdesc + (uint64_t)(kk * (U_CS >> 4)), idesc,
                      (j > 0 || kk > 0) ? 1u : 0u);
          }
          mma_commit(&sh.empty[st]);
        }
        if (ok) mma_commit(&sh.accfull[ab]);
      }
      // every MMA issued (also on an abort) has finished before TMEM is freed
      mma_commit(&sh.mmadone);
      mbar_wait(&sh.mmadone, 0, nullptr, err, ERR_WAIT_ACCUM);
    }
    __syncwarp();
  } else if (warp < WARP_E0 + NWARP_E) {
    if constexpr (!TMAV) regs_dec<REGS_EPI>();
    // epilogue: TMEM lanes 32*quarter .. +31 = tiles of the block
    const int quarter = warp & 3;
    __half* m16 = static_cast<__half*>(p.mid_result);
    for (int ui = 0; ui < sc.cnt; ++ui) {
      const Unit un = sched_unit(g, sc, ui);
      const int kb = un.kp * KPU;
      const int ab = ui & 1;
      if (!mbar_wait_warp(&sh.accfull[ab], (ui >> 1) & 1, abort_flag, err, ERR_WAIT_ACCUM, SLEEP_NS)) break;
      tc_fence_after();
      const int i = quarter * 32 + lane;   // tile within the block
      const bool live = (long long)un.tb * 128 + i < g.NT;
      const uint32_t taddr = tmem + ((uint32_t)(quarter * 32) << 16) + ab * (KPU * 128);
      const long long rem = g.NT - (long long)un.tb * 128;
      const int ntb = rem < 128 ? (int)rem : 128;
      __half* mrow = m16 + m_offset(un.tb, un.t, kb * KB2, i, g.K, g.NT);
      // the unit's k rows (columns of D): a multiple of 16, at most 256
      int nrows = 0;
#pragma unroll
      for (int q = 0; q < KPU; ++q) nrows += kb + q < g.nKB2 ? kblock2_rows(kb + q, g.K) : 0;
      // 32-column chunks, the TMEM load of the next chunk in flight while
      // the current one is converted and stored
      auto ld = [&](int cc, float* v) {
        tmem_ld16(taddr + cc, v);
        if (cc + 16 < nrows) tmem_ld16(taddr + cc + 16, v + 16);
      };
      // fp8: M = su[t][k] * D (one fp32 product, then the fp16 rounding)
      const float* sur = F8 != 0 ? static_cast<const float*>(p.pweight) + (size_t)un.t * g.K + kb * KB2 : nullptr;
      auto st = [&](int cc, const float* v) {
        if (!live) return;
        __half* dst = mrow + (size_t)cc * ntb;
        float sc[32];
        if constexpr (F8 != 0) {
          // the chunk's 32 scales (the same for every lane), 16-byte loads
          const float4* s4 = reinterpret_cast<const float4*>(sur + cc);
#pragma unroll
          for (int q = 0; q < 8; ++q) {
            if (q >= 4 && cc + 16 >= nrows) break;
            const float4 f = __ldg(s4 + q);
            sc[4 * q] = f.x; sc[4 * q + 1] = f.y; sc[4 * q + 2] = f.z; sc[4 * q + 3] = f.w;
          }
        }
#pragma unroll
        for (int jj = 0; jj < 16; ++jj) dst[(size_t)jj * ntb] = __float2half_rn(F8 != 0 ? v[jj] * sc[jj] : v[jj]);
        if (cc + 16 < nrows) {
#pragma unroll
          for (int jj = 16; jj < 32; ++jj) dst[(size_t)jj * ntb] = __float2half_rn(F8 != 0 ? v[jj] * sc[jj] : v[jj]);
        }
      };
      float va[32], vb[32];
      ld(0, va);
      tmem_ld_wait();
      for (int cc = 0; cc < nrows; cc += 64) {
        if (cc + 32 < nrows) ld(cc + 32, vb);
        st(cc, va);
        tmem_ld_wait();
        if (cc + 32 >= nrows) break;
        if (cc + 64 < nrows) ld(cc + 64, va);
        st(cc + 32, vb);
        tmem_ld_wait();
      }
      tc_fence_before();
      __syncwarp();
      if (lane == 0) mbar_arrive(&sh.accempty[ab]);
    }
  } else if constexpr (!TMAV) {
    regs_inc<REGS_PROD>();
    // V producers: thread = (tile tl of the unit's 128-tile block, channel
    // half hh).  The load cursor (lu, lj) runs up to RING stages ahead of
    // the consume cursor (cu, cj); the consume side keeps per unit index
    // mod 8 (2 bits each) whether the tile exists and whether its tap adds.
    const int pw = warp - WARP_P0;
    const int tl = (pw & 3) * 32 + lane, hh = pw >> 2;
    const uint8_t* xr = static_cast<const uint8_t*>(p.transform_pin);
    int lu = 0, lj = 0, cu = 0, cj = 0;
    uint32_t info = 0;
    Prod pr;
    pr.rec = xr;
    pr.ox = pr.oy = 0;
    pr.live = pr.add = false;
    const size_t step_bytes = (size_t)SK * g.cbs;
    const uint8_t* rec = xr;
    uint4 w0[SK][2], w1[SK][2], w2[SK][2], w3[SK][2];
    auto issue = [&](uint4 (&w)[SK][2]) {
      if (lu >= sc.cnt) return;
      if (lj == 0) {
        const Unit un = sched_unit(g, sc, lu);
        pr = prod(g, xr, un.t, un.tb, tl, hh);
        rec = pr.rec;
        const uint32_t sh2 = (uint32_t)(lu & 7) * 2;
        info = (info & ~(3u << sh2)) | ((uint32_t)((pr.live ? 1 : 0) | (pr.add ? 2 : 0)) << sh2);
      }
#pragma unroll
      for (int kk = 0; kk < SK; ++kk) {
        if (pr.live && lj * SK + kk < g.CS) {
          const uint8_t* r = rec + (size_t)kk * g.cbs;
          w[kk][0] = WINO_RES_LOAD(reinterpret_cast<const uint4*>(r + pr.ox));
          w[kk][1] = WINO_RES_LOAD(reinterpret_cast<const uint4*>(r + pr.oy));
        }
      }
      rec += step_bytes;
      if (++lj == nst) { lj = 0; ++lu; }
    };
    uint32_t it = 0;
    auto consume = [&](const uint4 (&w)[SK][2]) -> bool {
      const int st = it % NSTAGE;
      if (it >= NSTAGE &&
          !mbar_wait_warp(&sh.empty[st], (it / NSTAGE - 1) & 1, abort_flag, err, ERR_WAIT_EMPTY, SLEEP_NS))
        return false;
      const uint32_t inf = (info >> ((uint32_t)(cu & 7) * 2)) & 3u;
      uint8_t* adst = smem + U_BYTES + st * STAGE_A + (tl >> 3) * 256 + hh * 128 + (tl & 7) * 16;
#pragma unroll
      for (int kk = 0; kk < SK; ++kk) {
        if (cj * SK + kk < g.CS) {
          uint4 v = make_uint4(0u, 0u, 0u, 0u);
          if (inf & 1u) v = (inf & 2u) ? tp::hadd_4(w[kk][0], w[kk][1]) : tp::hsub_4(w[kk][0], w[kk][1]);
          *reinterpret_cast<uint4*>(adst + kk * A_STEP) = v;
        }
      }
      fence_proxy_async_shared();
      __syncwarp();
      if (lane == 0) mbar_arrive(&sh.full[st]);
      ++it;
      if (++cj == nst) { cj = 0; ++cu; }
      return cu < sc.cnt && !*abort_flag;
    };
    if (sc.cnt > 0) {
      if constexpr (RING == 4) {
        issue(w0);
        issue(w1);
        issue(w2);
        while (true) {
          issue(w3);
          if (!consume(w0)) break;
          issue(w0);
          if (!consume(w1)) break;
          issue(w1);
          if (!consume(w2)) break;
          issue(w2);
          if (!consume(w3)) break;
        }
      } else if constexpr (RING == 3) {
        issue(w0);
        issue(w1);
        while (true) {
          issue(w2);
          if (!consume(w0)) break;
          issue(w0);
          if (!consume(w1)) break;
          issue(w1);
          if (!consume(w2)) break;
        }
      } else {
        issue(w0);
        while (true) {
          issue(w1);
          if (!consume(w0)) break;
          issue(w0);
          if (!consume(w1)) break;
        }
      }
    }
  }
  tc_fence_before();
  __syncthreads();
  if (warp == WARP_MMA) {
    tc_fence_after();
    tmem_dealloc(tmem, 512);
  }
}

// =============================================================================
// Transformed input tiles V2 (pre-pass of the bulk-copy-fed GEMM)
// =============================================================================
// V2 holds V[t][tile][c] in tile blocks of 128 tiles, without padding beyond
// the tile count rounded up to 8 (NT8): block tb of tap t starts at element
// (t * NT8 + 128 tb) * C, its K-step cs at + cs * rows * 16 (rows =
// min(128, NT8 - 128 tb)); inside a K-step the K-major core-matrix
// interleave of the GEMM's tile operand puts tile i, channel c at byte
// (i >> 3) * 256 + (c >> 3) * 128 + (i & 7) * 16 + (c & 7) * 2.  16 * NT8 *
// C fp16 in all: the reference's transform_pin holds exactly V for even
// H = W and tiles a multiple of 8.  Values as the fused kernel's producers
// and the unfused comparator's input transform (B^T rows first, then
// columns; every +- sum of two fp16 values rounded once), which the
// reference computes at src/preprocessing.cuh:273-424.
//
// Thread = (tile, channel half): lanes are consecutive tiles, so each
// window-row load of a warp (4 bytes: columns 2x, 2x + 1) is one contiguous
// run per tile row; two channels go through the transform together as the
// halves of fp16x2 values, which is also how they sit in a V2 word, and each
// tap's 8 channels leave as one 16-byte store.  Item = (tile block, K-step),
// 256 threads, grid-stride over items.  W odd (4-byte words would be
// misaligned) reads single elements instead.
namespace v2t {
constexpr int SMEM_BYTES = 0;
}  // namespace v2t

#ifndef WINO_V2_MINB
#define WINO_V2_MINB 2
#endif
__global__ void __launch_bounds__(256, WINO_V2_MINB) v2_layout_kernel(KernelParam p) {
  const int C = p.c, H = p.h, W = p.w;
  const int TP = (p.Oh + 1) >> 1, TQ = (p.Ow + 1) >> 1;
  const int NT = p.n * TP * TQ;                  // < 2^30 (host bound)
  const int NT8 = (NT + 7) & ~7;
  const int CS = C >> 4, nTB = (NT8 + 127) >> 7;
  const int items = nTB * CS;
  const int il = threadIdx.x & 127, hh = threadIdx.x >> 7;
  const unsigned short* X = static_cast<const unsigned short*>(p.pin);
  uint8_t* v2 = static_cast<uint8_t*>(p.transform_pin);
  const size_t plane = (size_t)H * W;
  const size_t tap_bytes = (size_t)NT8 * C * 2;
  const bool w_even = (W & 1) == 0;
  // W % 4 == 0 and an 8-byte aligned input: the window row's words at
  // columns 2tx - 2 and 2tx (or 2tx and 2tx + 2) form one aligned 8-byte word
  const bool w4 = (W & 3) == 0 && (reinterpret_cast<uintptr_t>(X) & 7) == 0;
  for (int item = blockIdx.x; item < items; item += gridDim.x) {
    const int tb = item / CS, cs = item - tb * CS;
    const int rows = min(128, NT8 - tb * 128);
    // threads past the block's rows compute zeros and store nothing
    const bool inblk = il < rows;
    const int tile = tb * 128 + il;
    const bool live = inblk && tile < NT;
    int n = 0, ty = 0, tx = 0;
    if (live) {
      const int per = TP * TQ;
      n = tile / per;
      const int r = tile - n * per;
      ty = r / TQ;
      tx = r - ty * TQ;
    }
    const int y0 = 2 * ty - 1, x0 = 2 * tx;      // window rows y0 .., columns x0 - 1 .. x0 + 2
    const unsigned short* base = X + ((size_t)n * C + cs * 16 + hh * 8) * plane;
    uint32_t vt[16][4];                          // [tap][channel pair]
#pragma unroll
    for (int cp = 0; cp < 4; ++cp) {
      // col[r][j] = (channel 2cp, channel 2cp + 1) at row y0 + r, column x0 - 1 + j
      uint32_t col[4][4];
#pragma unroll
      for (int r = 0; r < 4; ++r) {
        const int y = y0 + r;
        const bool rok = live && y >= 0 && y < H;
        uint32_t a[2][3];                        // channel, word (columns x0-2.., x0.., x0+2..)
#pragma unroll
        for (int ch = 0; ch < 2; ++ch) {
          const unsigned short* row = base + (size_t)(2 * cp + ch) * plane + (size_t)(rok ? y : 0) * W;
          if (w4) {
            // odd tx: [2tx-2, 2tx+1] aligned + [2tx+2, 2tx+3]; even tx: [2tx, 2tx+3]
            // aligned + [2tx-2, 2tx-1] -- two loads, the 8-byte one shared by
            // a pair of lanes; the aligned word never crosses the row end
            const bool odd = (tx & 1) != 0;
            const int xa = odd ? x0 - 2 : x0, xb = odd ? x0 + 2 : x0 - 2;
            const uint2 wa = rok ? *reinterpret_cast<const uint2*>(row + xa) : make_uint2(0u, 0u);
            const uint32_t wb = (rok && xb >= 0 && xb < W) ? *reinterpret_cast<const uint32_t*>(row + xb) : 0u;
            a[ch][0] = odd ? wa.x : wb;
            a[ch][1] = odd ? wa.y : wa.x;
            a[ch][2] = odd ? wb : wa.y;
          } else if (w_even) {
#pragma unroll
            for (int q = 0; q < 3; ++q) {
              const int x = x0 - 2 + 2 * q;
              a[ch][q] = (rok && x >= 0 && x < W) ? *reinterpret_cast<const uint32_t*>(row + x) : 0u;
            }
          } else {
#pragma unroll
            for (int q = 0; q < 3; ++q) {
              const int x = x0 - 2 + 2 * q;
              const uint32_t lo = (rok && x >= 0 && x < W) ? row[x] : 0u;
              const uint32_t hi = (rok && x + 1 >= 0 && x + 1 < W) ? row[x + 1] : 0u;
              a[ch][q] = lo | (hi << 16);
            }
          }
        }
        col[r][0] = __byte_perm(a[0][0], a[1][0], 0x7632);   // column x0 - 1
        col[r][1] = __byte_perm(a[0][1], a[1][1], 0x5410);   // x0
        col[r][2] = __byte_perm(a[0][1], a[1][1], 0x7632);   // x0 + 1
        col[r][3] = __byte_perm(a[0][2], a[1][2], 0x5410);   // x0 + 2
      }
      // rows of B^T d (d0 - d2, d1 + d2, d2 - d1, d1 - d3), then the same on columns
      uint32_t e[4][4];
#pragma unroll
      for (int j = 0; j < 4; ++j) {
        e[0][j] = hsub2(col[0][j], col[2][j]);
        e[1][j] = hadd2(col[1][j], col[2][j]);
        e[2][j] = hsub2(col[2][j], col[1][j]);
        e[3][j] = hsub2(col[1][j], col[3][j]);
      }
#pragma unroll
      for (int a = 0; a < 4; ++a) {
        vt[4 * a + 0][cp] = hsub2(e[a][0], e[a][2]);
        vt[4 * a + 1][cp] = hadd2(e[a][1], e[a][2]);
        vt[4 * a + 2][cp] = hsub2(e[a][2], e[a][1]);
        vt[4 * a + 3][cp] = hsub2(e[a][1], e[a][3]);
      }
    }
    if (!inblk) continue;
    uint8_t* out = v2 + ((size_t)tb * 128 * C + (size_t)cs * rows * 16) * 2 + (il >> 3) * 256 + hh * 128 +
                   (il & 7) * 16;
#pragma unroll
    for (int t = 0; t < 16; ++t)
      *reinterpret_cast<uint4*>(out + (size_t)t * tap_bytes) = make_uint4(vt[t][0], vt[t][1], vt[t][2], vt[t][3]);
  }
}

// =============================================================================
// fp8 hi+lo two-stage variant: channel scales, U and V2 in e4m3 hi + lo
// =============================================================================
// x = hi + lo with hi = e4m3(x) and lo = e4m3(x - hi) keeps about 8 bits of
// x; the tap GEMM accumulates U_hi V_hi + U_lo V_hi + U_hi V_lo (the dropped
// U_lo V_lo is ~2^-8 of a product), so the fp8 tensor path reaches the
// accuracy of fp16 operands.  Scales as the fused fp8 variant's: per input
// channel inv_c = fp16(min(448 / (4 max|x_c|), 65504)) (|V| <= 4 max|x_c|),
// V' = fp16(V) * inv_c; U'[t][k][c] = U * (1 / inv_c), su[t][k] = max_c |U'|
// / 448, U'' = U' / su; M = su * sum_c U'' V'.  The reference has no fp8
// path (src/matrixmul.cuh:28-35 is fp16).

// per-channel max |x| as fp16 magnitude bits (monotonic as unsigned);
// amax must be zero on entry.  Grid (C, image groups): a CTA reduces its
// channel over images g, g + gridDim.y, ... (16-byte loads when the planes
// are 16-byte aligned, hw % 8 == 0) and issues one atomicMax.
__global__ void __launch_bounds__(128) f8_amax_kernel(const unsigned short* __restrict__ x, unsigned* amax, int n,
                                                      int c, int hw) {
  __shared__ unsigned wmax[4];
  const int ch = blockIdx.x;
  const bool vec = (hw & 7) == 0 && (reinterpret_cast<uintptr_t>(x) & 15) == 0;
  unsigned m = 0;
  for (int img = blockIdx.y; img < n; img += gridDim.y) {
    const unsigned short* src = x + ((size_t)img * c + ch) * hw;
    if (vec) {
      const uint4* s4 = reinterpret_cast<const uint4*>(src);
      for (int i = threadIdx.x; i < hw / 8; i += blockDim.x) {
        const uint4 v = __ldg(s4 + i);
        const uint32_t w[4] = {v.x, v.y, v.z, v.w};
#pragma unroll
        for (int j = 0; j < 4; ++j) m = max(m, max(w[j] & 0x7fffu, (w[j] >> 16) & 0x7fffu));
      }
    } else {
      for (int i = threadIdx.x; i < hw; i += blockDim.x) m = max(m, (unsigned)(src[i] & 0x7fffu));
    }
  }
  for (int o = 16; o > 0; o >>= 1) m = max(m, __shfl_xor_sync(0xffffffffu, m, o));
  if ((threadIdx.x & 31) == 0) wmax[threadIdx.x >> 5] = m;
  __syncthreads();
  if (threadIdx.x == 0) {
    m = max(max(wmax[0], wmax[1]), max(wmax[2], wmax[3]));
    if (m) atomicMax(amax + ch, m);
  }
}

__device__ __forceinline__ float f8_inv_scale(unsigned amax_bits) {
  const float a = __half2float(__ushort_as_half((unsigned short)amax_bits));
  return a > 0.f ? __half2float(__float2half_rn(fminf(448.f / (4.f * a), 65504.f))) : 1.f;
}

// two fp16 -> two e4m3 (round to nearest, saturating) and back
__device__ __forceinline__ uint32_t e4m3x2_of_h2(uint32_t h2) {
  unsigned short r;
  asm("cvt.rn.satfinite.e4m3x2.f16x2 %0, %1;" : "=h"(r) : "r"(h2));
  return r;
}
__device__ __forceinline__ uint32_t h2_of_e4m3x2(uint32_t e2) {
  uint32_t r;
  asm("cvt.rn.f16x2.e4m3x2 %0, %1;" : "=r"(r) : "h"((unsigned short)e2));
  return r;
}

// e4m3 hi and lo of an fp32 value
__device__ __forceinline__ void f8_split(float v, uint8_t& hi, uint8_t& lo) {
  const __nv_fp8_e4m3 h(v);
  const float hf = static_cast<float>(h);
  const __nv_fp8_e4m3 l(v - hf);
  hi = h.__x;
  lo = l.__x;
}

// U (fp16, unfused GEMM layout) -> U8 [t][k pair][K-step of 32][term][rows x
// 32 bytes in the K-major core-matrix interleave] and su[t][k].  Warp per
// (tap, output channel): lanes stride over the channels, the row maximum by
// shuffles; inv_c is recomputed from amax.
__global__ void __launch_bounds__(256) f8_u_kernel(const __half* __restrict__ u2, const unsigned* __restrict__ amax,
                                                   uint8_t* u8, float* su, int K, int C, int terms) {
  const int row = (int)((blockIdx.x * blockDim.x + threadIdx.x) >> 5), lane = threadIdx.x & 31;
  if (row >= 16 * K) return;                     // whole warps leave together
  const int t = row / K, k = row - t * K;
  auto uval = [&](int c) { return __half2float(u2[u2_offset(t, k, c, K, C)]) / f8_inv_scale(amax[c]); };
  float m = 0.f;
  for (int c = lane; c < C; c += 32) m = fmaxf(m, fabsf(uval(c)));
  for (int o = 16; o > 0; o >>= 1) m = fmaxf(m, __shfl_xor_sync(0xffffffffu, m, o));
  const float s = m > 0.f ? m / 448.f : 1.f;
  if (lane == 0) su[row] = s;
  const int kp = k / (2 * KB2), r = k - kp * 2 * KB2;          // row within the k pair
  const int rk = min(2 * KB2, K - kp * 2 * KB2);                // rows of the k pair
  uint8_t* blk = u8 + ((size_t)t * K + (size_t)kp * 2 * KB2) * C * terms;
  for (int c = lane; c < C; c += 32) {
    uint8_t hi, lo;
    f8_split(uval(c) / s, hi, lo);
    const int c32 = c >> 5, cc = c & 31;
    const size_t off = (size_t)(r >> 3) * 256 + (cc >> 4) * 128 + (r & 7) * 16 + (cc & 15);
    blk[((size_t)c32 * terms + 0) * rk * 32 + off] = hi;
    if (terms == 2) blk[((size_t)c32 * 2 + 1) * rk * 32 + off] = lo;
  }
}

// V2 in e4m3 hi + lo: as v2_layout_kernel, then V' = fp16(V) * inv_c (fp16
// product, as the fused fp8 variant) split into e4m3 hi and lo.  Per tap the
// tile block's K-steps of 32 channels hold [hi | lo] pieces of rows x 32
// bytes; inside a piece tile i, channel c (of 32) at byte (i >> 3) * 256 +
// (c >> 4) * 128 + (i & 7) * 16 + (c & 15).  Item = (tile block, 16-channel
// half of a K-step); thread = (tile, 8 channels).
template <int TERMS>
__global__ void __launch_bounds__(256, 2) v2f8_layout_kernel(KernelParam p) {
  const int C = p.c, H = p.h, W = p.w;
  const int TP = (p.Oh + 1) >> 1, TQ = (p.Ow + 1) >> 1;
  const int NT = p.n * TP * TQ;
  const int NT8 = (NT + 7) & ~7;
  const int CS = C >> 4, nTB = (NT8 + 127) >> 7;
  const int items = nTB * CS;
  const int il = threadIdx.x & 127, hh = threadIdx.x >> 7;
  const unsigned short* X = static_cast<const unsigned short*>(p.pin);
  const unsigned* amax = static_cast<const unsigned*>(p.mid_result);
  uint8_t* v2 = static_cast<uint8_t*>(p.transform_pin);
  const size_t plane = (size_t)H * W;
  const size_t tap_bytes = (size_t)NT8 * C * TERMS;   // bytes per tile and channel: the terms
  const bool w_even = (W & 1) == 0;
  for (int item = blockIdx.x; item < items; item += gridDim.x) {
    const int tb = item / CS, cs = item - tb * CS;
    const int rows = min(128, NT8 - tb * 128);
    if (il >= rows) continue;
    const int tile = tb * 128 + il;
    const bool live = tile < NT;
    int n = 0, ty = 0, tx = 0;
    if (live) {
      const int per = TP * TQ;
      n = tile / per;
      const int r = tile - n * per;
      ty = r / TQ;
      tx = r - ty * TQ;
    }
    const int y0 = 2 * ty - 1, x0 = 2 * tx;
    const int c0 = cs * 16 + hh * 8;
    const unsigned short* base = X + ((size_t)n * C + c0) * plane;
    uint32_t inv2[4];                            // (inv_c, inv_c+1) as fp16x2
#pragma unroll
    for (int cp = 0; cp < 4; ++cp) {
      const __half2 iv = __floats2half2_rn(f8_inv_scale(amax[c0 + 2 * cp]), f8_inv_scale(amax[c0 + 2 * cp + 1]));
      inv2[cp] = *reinterpret_cast<const uint32_t*>(&iv);
    }
    uint32_t vt[16][4];
#pragma unroll
    for (int cp = 0; cp < 4; ++cp) {
      uint32_t col[4][4];
#pragma unroll
      for (int r = 0; r < 4; ++r) {
        const int y = y0 + r;
        const bool rok = live && y >= 0 && y < H;
        uint32_t a[2][3];
#pragma unroll
        for (int ch = 0; ch < 2; ++ch) {
          const unsigned short* row = base + (size_t)(2 * cp + ch) * plane + (size_t)(rok ? y : 0) * W;
          if (w_even) {
#pragma unroll
            for (int q = 0; q < 3; ++q) {
              const int x = x0 - 2 + 2 * q;
              a[ch][q] = (rok && x >= 0 && x < W) ? *reinterpret_cast<const uint32_t*>(row + x) : 0u;
            }
          } else {
#pragma unroll
            for (int q = 0; q < 3; ++q) {
              const int x = x0 - 2 + 2 * q;
              const uint32_t lo = (rok && x >= 0 && x < W) ? row[x] : 0u;
              const uint32_t hi = (rok && x + 1 >= 0 && x + 1 < W) ? row[x + 1] : 0u;
              a[ch][q] = lo | (hi << 16);
            }
          }
        }
        col[r][0] = __byte_perm(a[0][0], a[1][0], 0x7632);
        col[r][1] = __byte_perm(a[0][1], a[1][1], 0x5410);
        col[r][2] = __byte_perm(a[0][1], a[1][1], 0x7632);
        col[r][3] = __byte_perm(a[0][2], a[1][2], 0x5410);
      }
      uint32_t e[4][4];
#pragma unroll
      for (int j = 0; j < 4; ++j) {
        e[0][j] = hsub2(col[0][j], col[2][j]);
        e[1][j] = hadd2(col[1][j], col[2][j]);
        e[2][j] = hsub2(col[2][j], col[1][j]);
        e[3][j] = hsub2(col[1][j], col[3][j]);
      }
#pragma unroll
      for (int a = 0; a < 4; ++a) {
        vt[4 * a + 0][cp] = hsub2(e[a][0], e[a][2]);
        vt[4 * a + 1][cp] = hadd2(e[a][1], e[a][2]);
        vt[4 * a + 2][cp] = hsub2(e[a][2], e[a][1]);
        vt[4 * a + 3][cp] = hsub2(e[a][1], e[a][3]);
      }
    }
    // K-step cs >> 1 of 32 channels, this thread's 8 channels at (cs & 1) * 16 + hh * 8
    const int rws = rows * 32;                   // bytes of one piece
    uint8_t* out = v2 + (size_t)tb * 128 * C * TERMS + (size_t)(cs >> 1) * TERMS * rws + (il >> 3) * 256 + (cs & 1) * 128 +
                   (il & 7) * 16 + hh * 8;
#pragma unroll
    for (int t = 0; t < 16; ++t) {
      // V' = fp16(V * inv); hi = e4m3(V'); lo = e4m3(V' - hi), the fp16
      // difference exact (hi is V' rounded to 4 significant bits)
      uint32_t hw[2], lw[2];
#pragma unroll
      for (int q = 0; q < 2; ++q) {
        uint32_t hp[2], lp[2];
#pragma unroll
        for (int u = 0; u < 2; ++u) {
          const uint32_t w = hmul2_u32(vt[t][2 * q + u], inv2[2 * q + u]);
          hp[u] = e4m3x2_of_h2(w);
          lp[u] = TERMS == 2 ? e4m3x2_of_h2(hsub2(w, h2_of_e4m3x2(hp[u]))) : 0u;
        }
        hw[q] = hp[0] | (hp[1] << 16);
        lw[q] = lp[0] | (lp[1] << 16);
      }
      *reinterpret_cast<uint2*>(out + (size_t)t * tap_bytes) = make_uint2(hw[0], hw[1]);
      if (TERMS == 2) *reinterpret_cast<uint2*>(out + (size_t)t * tap_bytes + rws) = make_uint2(lw[0], lw[1]);
    }
  }
}

// =============================================================================
// Output transform
// =============================================================================
// Persistent: work item = (tile block tb, 8 output channels kg), item i =
// tb * (K / 8) + kg, CTA b takes items b, b + grid, ...: the tile blocks in
// increasing order, the GEMM's last-written (still in L2) first.  An item's 16
// taps x 8 channels of the blocked M (16 contiguous runs of 8 * ntb fp16)
// come in by bulk copy into one of NBUF shared-memory buffers (two by
// default, with three CTAs per SM), each refilled as soon as it is free, so
// the next item's copy is in flight while one is transformed and the bytes
// in flight do not depend on registers.
// Thread = (channel kl, 4 tiles g4 .. g4+3 of the block): it reads its 16
// taps from shared memory (a warp's 8-byte reads are contiguous),
// accumulates z = A^T m in fp32 tap by tap in the order of the comparator's
// output transform (so the result is bit-identical to it), forms y = z A and
// stores it with one fp16 rounding; two tiles of one tile row starting at an
// even tile column share one 8-byte store per output row (63.5 -> 56.3 us on
// N128 C256 H28 K256 against a 4-byte store per tile and row).  K is a
// multiple of 16 and mid_result 16-byte aligned, so every copy starts on a
// 16-byte boundary and moves a multiple of 16 bytes.
#ifndef WINO_OT_KG
#define WINO_OT_KG 8
#endif
#ifndef WINO_OT_NBUF
#define WINO_OT_NBUF 2
#endif
#ifndef WINO_OT_MINB
#define WINO_OT_MINB 3
#endif
// Tuning knobs (defaults measured fastest on N128 C256 H28 K256): output
// channels per item, shared-memory buffers, resident CTAs per SM -- two 32 KB
// buffers and three CTAs per SM take 47 us against 55 for three buffers and
// two CTAs.
namespace ot {
constexpr int KG = WINO_OT_KG;                // output channels per item (one warp each)
constexpr int TT = 4;                         // tiles per thread
constexpr int NBUF = WINO_OT_NBUF;
constexpr int NTHREAD = 32 * KG;
constexpr int BUF_BYTES = 16 * KG * 128 * 2;  // 32 KB for 8 channels
constexpr int SMEM_BYTES = NBUF * BUF_BYTES + 128;
}

__global__ void __launch_bounds__(ot::NTHREAD, WINO_OT_MINB) twostage_output_kernel(KernelParam p) {
  using namespace ts;
  extern __shared__ __align__(128) uint8_t osm[];
  __shared__ uint64_t full[ot::NBUF];
  const int K = p.k, P = p.Oh, Q = p.Ow;
  const int TP = (P + 1) >> 1, TQ = (Q + 1) >> 1;
  const long long NT = (long long)p.n * TP * TQ;
  const int nTB = (int)((NT + 127) / 128);
  const int nKG = K / ot::KG;
  const int nitems = nTB * nKG;
  const __half* m16 = static_cast<const __half*>(p.mid_result);
  if (threadIdx.x == 0) {
    for (int b = 0; b < ot::NBUF; ++b) mbar_init(&full[b], 1);
    fence_barrier_init();
  }
  __syncthreads();
  // issue the copies of `item` into buffer `buf` (warp 0)
  auto fetch = [&](int item, int buf) {
    const int tb = item / nKG, k0 = (item - tb * nKG) * ot::KG;
    const long long rem = NT - (long long)tb * 128;
    const int ntb = rem < 128 ? (int)rem : 128;
    const uint32_t run = (uint32_t)(ot::KG * ntb * 2);
    if (threadIdx.x == 0) mbar_arrive_expect_tx(&full[buf], 16 * run);
    __syncwarp();
    if (threadIdx.x < 16)
      bulk_g2s(osm + buf * ot::BUF_BYTES + threadIdx.x * run,
               m16 + m_offset(tb, threadIdx.x, k0, 0, K, NT), run, &full[buf]);
  };
  if (threadIdx.x < 32)
    for (int b = 0; b < ot::NBUF; ++b)
      if ((int)blockIdx.x + b * (int)gridDim.x < nitems) fetch(blockIdx.x + b * gridDim.x, b);
  const int kl = threadIdx.x >> 5, g4 = (threadIdx.x & 31) * ot::TT;
  const int per_img = TP * TQ;
  const bool pair_ok = (Q & 1) == 0 && (reinterpret_cast<uintptr_t>(p.pout) & 3) == 0;
  // rows of a multiple of 4 elements from an 8-byte aligned output: tile
  // pairs starting at an even tile column write 8-byte words
  const bool pair8_ok = (Q & 3) == 0 && (reinterpret_cast<uintptr_t>(p.pout) & 7) == 0;
  __half* out = static_cast<__half*>(p.pout);
  int j = 0;
  for (int item = blockIdx.x; item < nitems; item += gridDim.x, ++j) {
    const int buf = j % ot::NBUF;
    const int tb = item / nKG, k = (item - tb * nKG) * ot::KG + kl;
    const long long rem = NT - (long long)tb * 128;
    const int ntb = rem < 128 ? (int)rem : 128;
    const uint32_t run = (uint32_t)(ot::KG * ntb * 2);
    // the copies complete within microseconds; a wait past the bound leaves
    // the error word set and the rest of the output unwritten
    if (!mbar_wait(&full[buf], (j / ot::NBUF) & 1, nullptr, &g_twostage_err, ERR_WAIT_FULL)) break;
    if (g4 < ntb) {
      const __half* ms = reinterpret_cast<const __half*>(osm + buf * ot::BUF_BYTES);
      // z[r][b] = sum_a At[r][a] m[4a+b], accumulated in tap order a = 0..3
      float z[ot::TT][2][4];
#pragma unroll
      for (int t = 0; t < 16; ++t) {
        const int a = t >> 2, b = t & 3;
        const __half* src = ms + (size_t)t * (run / 2) + kl * ntb + g4;
        float v[ot::TT];
        if (ntb == 128) {
          const uint2 w = *reinterpret_cast<const uint2*>(src);
          const float2 f0 = __half22float2(*reinterpret_cast<const __half2*>(&w.x));
          const float2 f1 = __half22float2(*reinterpret_cast<const __half2*>(&w.y));
          v[0] = f0.x; v[1] = f0.y; v[2] = f1.x; v[3] = f1.y;
        } else {
#pragma unroll
          for (int i = 0; i < ot::TT; ++i) v[i] = g4 + i < ntb ? __half2float(src[i]) : 0.f;
        }
#pragma unroll
        for (int i = 0; i < ot::TT; ++i) {
          if (a == 0) z[i][0][b] = v[i];
          if (a == 1) { z[i][0][b] = z[i][0][b] + v[i]; z[i][1][b] = v[i]; }
          if (a == 2) { z[i][0][b] = z[i][0][b] + v[i]; z[i][1][b] = z[i][1][b] - v[i]; }
          if (a == 3) z[i][1][b] = z[i][1][b] - v[i];
        }
      }
      // the first tile's (n, ty, tx), then step along the tile row
      const int tile0 = tb * 128 + g4;            // tiles < 2^30 (host check)
      int n = tile0 / per_img;
      int ty = (tile0 - n * per_img) / TQ;
      int tx = tile0 - n * per_img - ty * TQ;
      bool skip = false;                          // tile written with the previous one
#pragma unroll
      for (int i = 0; i < ot::TT; ++i) {
        if (g4 + i >= ntb) break;
        if (i > 0 && ++tx == TQ) {
          tx = 0;
          if (++ty == TP) { ty = 0; ++n; }
        }
        if (skip) { skip = false; continue; }
        float y[4];
#pragma unroll
        for (int r = 0; r < 2; ++r) {
          y[2 * r + 0] = z[i][r][0] + z[i][r][1] + z[i][r][2];
          y[2 * r + 1] = z[i][r][1] - z[i][r][2] - z[i][r][3];
        }
        const int oy = 2 * ty, ox = 2 * tx;
        __half* o = out + (((size_t)n * K + k) * P + oy) * (size_t)Q + ox;
        const bool two_cols = ox + 1 < Q, two_rows = oy + 1 < P;
        // this tile and the next in one tile row, 8-byte aligned: one 8-byte
        // store per output row for both
        if (i + 1 < ot::TT && g4 + i + 1 < ntb && tx + 1 < TQ && (tx & 1) == 0 && pair8_ok) {
          float y1[4];
#pragma unroll
          for (int r = 0; r < 2; ++r) {
            y1[2 * r + 0] = z[i + 1][r][0] + z[i + 1][r][1] + z[i + 1][r][2];
            y1[2 * r + 1] = z[i + 1][r][1] - z[i + 1][r][2] - z[i + 1][r][3];
          }
#pragma unroll
          for (int r = 0; r < 2; ++r) {
            if (oy + r >= P) break;
            const __half2 a = __floats2half2_rn(y[2 * r], y[2 * r + 1]);
            const __half2 b = __floats2half2_rn(y1[2 * r], y1[2 * r + 1]);
            *reinterpret_cast<uint2*>(o + (size_t)r * Q) =
                make_uint2(*reinterpret_cast<const uint32_t*>(&a), *reinterpret_cast<const uint32_t*>(&b));
          }
          skip = true;
          continue;
        }
        if (two_cols && pair_ok) {
          *reinterpret_cast<__half2*>(o) = __floats2half2_rn(y[0], y[1]);
          if (two_rows) *reinterpret_cast<__half2*>(o + Q) = __floats2half2_rn(y[2], y[3]);
        } else {
          o[0] = __float2half_rn(y[0]);
          if (two_cols) o[1] = __float2half_rn(y[1]);
          if (two_rows) {
            o[Q] = __float2half_rn(y[2]);
            if (two_cols) o[Q + 1] = __float2half_rn(y[3]);
          }
        }
      }
    }
    __syncthreads();   // every thread is done with the buffer
    const int next = item + ot::NBUF * (int)gridDim.x;
    if (threadIdx.x < 32 && next < nitems) fetch(next, buf);
  }
}

}  // namespace wino

using namespace wino;

extern "C" {

// The GEMM kernel for C input channels: the tap-pair kernel keeps U resident
// for up to 256 channels, the streamed-U kernel takes any C.
static_assert(WINO_PAIR_MAX_C <= 16 * tp::CS_MAX, "the tap-pair kernel keeps U for at most 256 channels");
static_assert(WINO_RES_MAX_C <= 16 * trs::CS_MAX, "the resident-U kernel keeps U for at most 256 channels");
enum GemmKind { GEMM_STREAM = 0, GEMM_RES = 1, GEMM_PAIR = 2, GEMM_RESV = 3 };
static GemmKind gemm_kind(int c) {
  if (c <= WINO_PAIR_MAX_C) return GEMM_PAIR;
  if (c <= WINO_RES_XR_MAX_C) return GEMM_RES;
  if (c <= WINO_RES_MAX_C) return GEMM_RESV;
  return GEMM_STREAM;
}
static bool use_xr(int c) { return gemm_kind(c) == GEMM_RES || gemm_kind(c) == GEMM_PAIR; }
static bool use_v2(int c) { return gemm_kind(c) == GEMM_RESV; }
static long long tiles8(int n, int h, int w) { return ((long long)n * ((h + 1) / 2) * ((w + 1) / 2) + 7) / 8 * 8; }

void* wino_twostage_gemm_kernel_ptr_for(int c) {
  switch (gemm_kind(c)) {
    case GEMM_PAIR: return (void*)twostage_pair_kernel;
    case GEMM_RES: return (void*)twostage_res_kernel_t<false>;
    case GEMM_RESV: return (void*)twostage_res_kernel_t<true>;
    default: return (void*)twostage_stream_kernel;
  }
}
void* wino_twostage_pair_kernel_ptr() { return (void*)twostage_pair_kernel; }
void* wino_twostage_res_kernel_ptr() { return (void*)twostage_res_kernel_t<false>; }
void* wino_twostage_resv_kernel_ptr() { return (void*)twostage_res_kernel_t<true>; }
void* wino_twostage_stream_kernel_ptr() { return (void*)twostage_stream_kernel; }
void* wino_twostage_output_kernel_ptr() { return (void*)twostage_output_kernel; }
int wino_twostage_threads_for(int c) {
  switch (gemm_kind(c)) {
    case GEMM_PAIR: return tp::NTHREAD;
    case GEMM_RES: return trs::NTHREAD;
    case GEMM_RESV: return trs::NTHREAD_V;
    default: return tsk::NTHREAD;
  }
}
int wino_twostage_smem_bytes_for(int c) {
  switch (gemm_kind(c)) {
    case GEMM_PAIR: return tp::SMEM_BYTES;
    case GEMM_RES:
    case GEMM_RESV: return trs::SMEM_BYTES;
    default: return tsk::SMEM_BYTES;
  }
}

int wino_twostage_output_smem_bytes() { return ot::SMEM_BYTES; }
int wino_twostage_output_threads() { return ot::NTHREAD; }

int wino_twostage_prepare() {
  if (cudaFuncSetAttribute(twostage_output_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                           ot::SMEM_BYTES) != cudaSuccess)
    return 1;
  if (cudaFuncSetAttribute(twostage_stream_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                           tsk::SMEM_BYTES) != cudaSuccess)
    return 1;
  if (cudaFuncSetAttribute(twostage_res_kernel_t<false>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                           trs::SMEM_BYTES) != cudaSuccess ||
      cudaFuncSetAttribute(twostage_res_kernel_t<true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                           trs::SMEM_BYTES) != cudaSuccess ||
      cudaFuncSetAttribute(twostage_res_kernel_t<true, 1>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                           trs::SMEM_BYTES) != cudaSuccess ||
      cudaFuncSetAttribute(twostage_res_kernel_t<true, 2>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                           trs::SMEM_BYTES) != cudaSuccess)
    return 1;
  // the resident-U kernel's warpgroups split exactly the registers it is
  // launched with; any other launch count would leave an increase waiting
  cudaFuncAttributes fa{};
  if (cudaFuncGetAttributes(&fa, twostage_res_kernel_t<false>) != cudaSuccess || fa.numRegs != trs::REGS_LAUNCH)
    return 1;
  return (int)cudaFuncSetAttribute(twostage_pair_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                   tp::SMEM_BYTES);
}

// The two-stage pre-pass: row-transformed records (XR) for the resident-U
// and tap-pair kernels, channel-blocked records (XB) for the streamed-U
// kernel.
size_t wino_xb_bytes(int n, int c, int h, int w);
unsigned wino_xb_layout_grid(int n, int c, int h, int w);
void* wino_xb_layout_kernel_ptr();

size_t wino_twostage_prepass_bytes(int n, int c, int h, int w) {
  if (use_v2(c)) return (size_t)16 * (size_t)tiles8(n, h, w) * (size_t)c * 2;
  return use_xr(c) ? xr::bytes(n, c, h, w) : wino_xb_bytes(n, c, h, w);
}
long long wino_twostage_prepass_items(int n, int c, int h, int w) {
  if (use_v2(c)) return (tiles8(n, h, w) + 127) / 128 * (c >> 4);
  const long long rows = use_xr(c) ? xr::rows(h) : xb_rows(h);
  return (long long)n * (c >> 4) * rows * xb_entries(w);
}
void* wino_twostage_prepass_kernel_ptr_for(int c) {
  if (use_v2(c)) return (void*)v2_layout_kernel;
  return use_xr(c) ? (void*)xr_layout_kernel : wino_xb_layout_kernel_ptr();
}
unsigned wino_twostage_prepass_grid(int n, int c, int h, int w) {
  if (use_v2(c)) {
    // the resident CTAs (WINO_V2_MINB per SM), grid-stride over the items
    const long long items = wino_twostage_prepass_items(n, c, h, w);
    const long long cap = 148LL * WINO_V2_MINB;
    return (unsigned)(items < cap ? (items > 0 ? items : 1) : cap);
  }
  if (!use_xr(c)) return wino_xb_layout_grid(n, c, h, w);
  const long long blocks = (wino_twostage_prepass_items(n, c, h, w) / 4 + 255) / 256;
  const long long cap = 148LL * 64;
  return (unsigned)(blocks < cap ? (blocks > 0 ? blocks : 1) : cap);
}
int wino_twostage_prepass_smem_bytes(int c) { return use_v2(c) ? v2t::SMEM_BYTES : 0; }
int wino_launch_twostage_prepass(const KernelParam* p, cudaStream_t stream) {
  void* args[] = {const_cast<KernelParam*>(p)};
  return (int)cudaLaunchKernel(wino_twostage_prepass_kernel_ptr_for(p->c),
                               dim3(wino_twostage_prepass_grid(p->n, p->c, p->h, p->w)), dim3(256), args,
                               (size_t)wino_twostage_prepass_smem_bytes(p->c), stream);
}

// Tiles and the M16 bytes of a shape (no padding).
long long wino_twostage_tiles(int n, int h, int w) { return (long long)n * ((h + 1) / 2) * ((w + 1) / 2); }
size_t wino_twostage_m_bytes(int n, int h, int w, int k) {
  return (size_t)16 * (size_t)k * (size_t)wino_twostage_tiles(n, h, w) * 2;
}

// Element offset of M[t][kk][tile] in the blocked M layout (for callers that
// read mid_result).
size_t wino_twostage_m_offset(int n, int h, int w, int k, int t, int kk, long long tile) {
  const long long NT = wino_twostage_tiles(n, h, w);
  return ts::m_offset((int)(tile / 128), t, kk, (int)(tile % 128), k, NT);
}

// GEMM grid: one CTA per SM up to the work available; the tap-pair kernel
// runs clusters of two CTAs (an even grid).
unsigned wino_twostage_gemm_grid(int n, int c, int h, int w, int k, int sms) {
  const long long ntb = (wino_twostage_tiles(n, h, w) + 127) / 128;
  const long long nkb = (k + KB2 - 1) / KB2;
  if (gemm_kind(c) == GEMM_PAIR) {
    const long long units = (long long)tp::NPAIR * ntb * ((nkb + 1) / 2);
    const long long clusters = sms / 2;
    return (unsigned)(2 * (units < clusters ? units : clusters));
  }
  static_assert(tsk::KPU == trs::KPU, "both one-tap kernels take two k-blocks per unit");
  const long long units = 16LL * ntb * ((nkb + tsk::KPU - 1) / tsk::KPU);
  return (unsigned)(units < sms ? units : sms);
}

// Output transform grid: the resident persistent CTAs (WINO_OT_MINB per SM)
// up to the work items.
void wino_twostage_output_grid(int n, int h, int w, int k, int sms, unsigned* gx, unsigned* gy) {
  const long long items = (wino_twostage_tiles(n, h, w) + 127) / 128 * (k / ot::KG);
  const long long cap = (long long)WINO_OT_MINB * sms;
  *gx = (unsigned)(items < cap ? items : cap);
  *gy = 1;
}

// fp8 two-stage path (extension API); hilo 1: e4m3 hi + lo terms, 0: single
// e4m3 terms.  Workspace, each part 256-byte aligned: channel maxima (C
// u32), su (16 K fp32), U8 (16 K C x terms bytes), V2 (16 x tiles rounded up
// to 8 x C x terms bytes), M16 (16 K tiles fp16).
static size_t al256(size_t b) { return (b + 255) / 256 * 256; }
static bool f8_ok(int n, int c, int h, int w, int k, int hilo) {
  return (hilo == 0 || hilo == 1) && n >= 1 && h >= 1 && w >= 1 && k >= 16 && k % 16 == 0 && c >= 32 &&
         c % 32 == 0 && c <= 256 && k <= 32767 && n <= 32767 && h <= 32767 && w <= 32767 &&
         wino_twostage_tiles(n, h, w) < (1LL << 30) &&
         (long long)n * (c >> 4) * ((tiles8(n, h, w) + 127) / 128) < (1LL << 31);
}
size_t wino_twostage_f8_workspace_bytes(int n, int c, int h, int w, int k, int hilo) {
  if (!f8_ok(n, c, h, w, k, hilo)) return 0;
  const size_t terms = hilo ? 2 : 1;
  return al256((size_t)c * 4) + al256((size_t)16 * k * 4) + al256((size_t)16 * k * c * terms) +
         al256((size_t)16 * tiles8(n, h, w) * c * terms) + wino_twostage_m_bytes(n, h, w, k);
}
void* wino_twostage_f8_kernel_ptr(int hilo) {
  return hilo ? (void*)twostage_res_kernel_t<true, 2> : (void*)twostage_res_kernel_t<true, 1>;
}
int wino_conv2d_twostage_f8(const void* x, const void* ucache2, void* workspace, void* y, int n, int c, int h,
                            int w, int k, int hilo, void* stream) {
  if (!x || !ucache2 || !workspace || !y) return 1;                  // WINO_EINVAL
  if ((reinterpret_cast<uintptr_t>(workspace) & 255) != 0) return 1;
  if (!f8_ok(n, c, h, w, k, hilo)) return 2;                         // WINO_EUNSUPPORTED
  if (wino_twostage_prepare() != 0) return 3;                         // WINO_ECUDA
  const int terms = hilo ? 2 : 1;
  uint8_t* ws = static_cast<uint8_t*>(workspace);
  unsigned* amax = reinterpret_cast<unsigned*>(ws);
  float* su = reinterpret_cast<float*>(ws + al256((size_t)c * 4));
  uint8_t* u8 = reinterpret_cast<uint8_t*>(su) + al256((size_t)16 * k * 4);
  uint8_t* v2 = u8 + al256((size_t)16 * k * c * terms);
  uint8_t* m16 = v2 + al256((size_t)16 * tiles8(n, h, w) * c * terms);
  const cudaStream_t s = (cudaStream_t)stream;
  int dev = 0, sms = 148;
  if (cudaGetDevice(&dev) != cudaSuccess ||
      cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess)
    return 3;
  KernelParam p{};
  p.pin = const_cast<void*>(x);
  p.pout = y;
  p.n = (short)n; p.c = (short)c; p.h = (short)h; p.w = (short)w; p.k = (short)k;
  p.r = 3; p.s = 3; p.u = 1; p.v = 1; p.p = 1; p.q = 1; p.Oh = (short)h; p.Ow = (short)w;
  if (cudaMemsetAsync(amax, 0, (size_t)c * 4, s) != cudaSuccess) return 3;
  {
    // enough CTAs to cover the GPU several times, at most one per image
    int groups = (32 * sms + c - 1) / c;
    if (groups > n) groups = n;
    f8_amax_kernel<<<dim3(c, groups), 128, 0, s>>>(static_cast<const unsigned short*>(x), amax, n, c, h * w);
  }
  f8_u_kernel<<<(16 * k * 32 + 255) / 256, 256, 0, s>>>(static_cast<const __half*>(ucache2), amax, u8, su, k, c,
                                                         terms);
  // V2: the channel maxima come in through mid_result
  p.transform_pin = v2;
  p.mid_result = amax;
  {
    const long long items = (tiles8(n, h, w) + 127) / 128 * (c >> 4);
    const long long cap = 2LL * sms;
    const unsigned grid = (unsigned)(items < cap ? items : cap);
    if (hilo) v2f8_layout_kernel<2><<<grid, 256, 0, s>>>(p);
    else v2f8_layout_kernel<1><<<grid, 256, 0, s>>>(p);
  }
  // tap GEMM: U8 resident, su through pweight, M into the workspace
  p.transform_filter = u8;
  p.pweight = su;
  p.mid_result = m16;
  {
    void* args[] = {&p};
    if (cudaLaunchKernel(wino_twostage_f8_kernel_ptr(hilo), dim3(wino_twostage_gemm_grid(n, c, h, w, k, sms)),
                         dim3(trs::NTHREAD_V), args, (size_t)trs::SMEM_BYTES, s) != cudaSuccess)
      return 3;
    unsigned ox, oy;
    wino_twostage_output_grid(n, h, w, k, sms, &ox, &oy);
    if (cudaLaunchKernel((void*)twostage_output_kernel, dim3(ox, oy), dim3(ot::NTHREAD), args,
                         (size_t)ot::SMEM_BYTES, s) != cudaSuccess)
      return 3;
  }
  return cudaGetLastError() == cudaSuccess ? 0 : 3;
}

uint32_t wino_twostage_error_read_clear() {
  uint32_t v = 0, z = 0;
  cudaMemcpyFromSymbol(&v, g_twostage_err, sizeof(v));
  cudaMemcpyToSymbol(g_twostage_err, &z, sizeof(z));
  return v;
}

}  // extern "C"
