// Two-stage Winograd F(2x2,3x3): input transform fused into the tap GEMM,
// output transform as a second kernel.
//
// The single fused kernel (fused_conv.cu) keeps all 16 taps of a tile block
// in TMEM until the output transform, which caps its MMAs at N = 32 tiles.
// This path gives that up for full-width MMAs: a work unit is one tap x 128
// tiles x 256 output channels (two M=128 N<=128 MMAs per K-step sharing the
// tile operand); its V operand is formed in shared memory by producer warps
// straight from the channel-blocked input (XB, written by the input
// pre-pass, L2-resident), so V never reaches HBM; M goes out as fp16 (16 * K
// * tiles elements, the size of the reference's mid_result for even H, W)
// and a second kernel applies A^T m A.  Against the reference's pipeline
// (src/preprocessing.cuh:273-424 writing V to transform_pin,
// src/matrixmul.cuh:139-556 reading it back, src/conv2d.cpp:17-250 reading
// M from mid_result) it drops the V round trip.
//
//   slot 1  dropin_filter_u2_kernel   W -> U2 (unfused GEMM layout), transform_filter
//   slot 2  xb_layout_kernel          X -> XB, transform_pin
//   slot 3  twostage_gemm_kernel      XB, U2 -> M16[t][k][tile], mid_result
//   slot 4  twostage_output_kernel    M16 -> Y
// (the drop-in ABI's route when M fits mid_result, i.e. even H and W; the
// extension entry point wino_conv2d_twostage runs slots 2-4 on any shape).
//
// V is formed with the fused kernel's packed-fp16 operations in the same
// order (rows of B^T d first, then columns), so the GEMM operands are
// bit-identical to the fused kernel's and to the unfused comparator's; with
// M rounded once to fp16 the output equals the unfused comparator's.
//
// Warp roles of the GEMM (448 threads, one CTA per SM): warp 0 lane 0 issues
// the U bulk copies, warp 1 lane 0 the MMAs, warps 2-5 drain TMEM into M16,
// warps 6-13 produce V (one thread per tile and 8-channel half; the 16
// window loads of a stage are in flight together before any arithmetic).
// Work units run tap-fastest, so the 16 taps of a tile block are in flight
// on neighbouring CTAs together and read the same XB rows from L2.  Every
// wait is bounded.
//
// The producers bound the GEMM: each stage's window loads (4 x 16 bytes per
// tile, channel half and K-step, 64 KB per stage) come back from L2 after
// 1.5-2.5 k cycles under load, and each producer has one stage of loads in
// flight.
#include <cuda_runtime.h>
#include <cuda_fp16.h>
#include "tc_sm100.cuh"
#include "wino_common.cuh"
#include "vgen.cuh"

namespace wino {

static __device__ uint32_t g_twostage_err;

namespace ts {

constexpr int NSTAGE = 4;
constexpr int SK = 4;                         // K-steps (16 channels each) per stage
constexpr int KPU = 2;                        // 128-row k-blocks per unit
constexpr int A_STEP = 128 * 16 * 2;          // 4 KB: V of 128 tiles x 16 channels (K-major)
constexpr int B_STEP = KB2 * 16 * 2;          // 4 KB: U of one 128-row k-block
constexpr int STAGE_A = SK * A_STEP;
constexpr int STAGE_B = SK * B_STEP;
constexpr int STAGE_BYTES = STAGE_A + KPU * STAGE_B;
constexpr int SMEM_BYTES = NSTAGE * STAGE_BYTES + 1024;
constexpr int WARP_U = 0, WARP_MMA = 1, WARP_E0 = 2, NWARP_E = 4, WARP_P0 = 6, NWARP_P = 8;
// Back-off of the waiting warps (after 8 polls), so that spinning epilogue
// and producer warps do not take issue slots from the working ones.
constexpr uint32_t SLEEP_EPI_NS = 32, SLEEP_PROD_NS = 32;
constexpr int NTHREAD = (WARP_P0 + NWARP_P) * 32;

struct Shared {
  uint64_t full[NSTAGE], empty[NSTAGE];
  uint64_t accfull[2], accempty[2];
  uint32_t tmem_base;
  int abort_flag;
};

struct Geo {
  int K, CS, HP, E, TP, TQ, nTB, nKB2, nKP, nst;
  long long NT, nunits;
  uint32_t RB;
};

__device__ __forceinline__ Geo geo(const KernelParam& p) {
  Geo g;
  g.K = p.k;
  g.CS = p.c >> 4;
  g.HP = xb_rows(p.h);
  g.E = xb_entries(p.w);
  g.RB = (uint32_t)xb_row_bytes(p.w);
  g.TP = (p.Oh + 1) >> 1;
  g.TQ = (p.Ow + 1) >> 1;
  g.NT = (long long)p.n * g.TP * g.TQ;
  g.nTB = (int)((g.NT + 127) / 128);
  g.nKB2 = (g.K + KB2 - 1) / KB2;
  g.nKP = (g.nKB2 + KPU - 1) / KPU;
  g.nunits = 16LL * g.nTB * g.nKP;
  g.nst = (g.CS + SK - 1) / SK;
  return g;
}

// Unit u -> tap t (fastest), k-block pair, tile block; kbs[i] = rows of the
// pair's i-th k-block (0 when absent).
__device__ __forceinline__ void unit_coords(const Geo& g, long long u, int& t, int& tb, int& kb,
                                            int (&kbs)[KPU]) {
  t = (int)(u & 15);
  const long long r = u >> 4;
  const int kp = (int)(r % g.nKP);
  tb = (int)(r / g.nKP);
  kb = kp * KPU;
#pragma unroll
  for (int i = 0; i < KPU; ++i) kbs[i] = kb + i < g.nKB2 ? kblock2_rows(kb + i, g.K) : 0;
}

// B^T row / column a of the 4-point transform (the fused kernel's bt_row /
// bt_cols: d0-d2, d1+d2, d2-d1, d1-d3) as two indices and the signs s0, s1 of
// s0*x[i0] + s1*x[i1], packed as fp16x2 (+1 = 0x3c00, -1 = 0xbc00).
__device__ __forceinline__ void bt_pick(int a, int& i0, int& i1, uint32_t& s0, uint32_t& s1) {
  i0 = a == 0 ? 0 : 1;
  i1 = a == 3 ? 3 : 2;
  s0 = a == 2 ? 0xbc00bc00u : 0x3c003c00u;
  s1 = (a == 0 || a == 3) ? 0xbc00bc00u : 0x3c003c00u;
}

// s0*x0 + s1*x1 with one rounding: the product by +-1 is exact, so this is
// bit-identical to the fused kernel's hadd2 / hsub2.
__device__ __forceinline__ uint32_t bt_op(uint32_t s0, uint32_t s1, uint32_t x0, uint32_t x1) {
  __half2 r = __hfma2(*reinterpret_cast<__half2*>(&x1), *reinterpret_cast<__half2*>(&s1),
                      __hmul2(*reinterpret_cast<__half2*>(&x0), *reinterpret_cast<__half2*>(&s0)));
  return *reinterpret_cast<uint32_t*>(&r);
}

// Loading side of one work unit for a producer thread.
struct ProdUnit {
  const uint8_t* xn;          // XB of the tile's image, channel block 0
  uint32_t o[4];              // window positions (i0,j0) (i0,j1) (i1,j0) (i1,j1)
  uint32_t sa0, sa1, sb0, sb1;
  bool live;
};

__device__ __forceinline__ ProdUnit prod_unit(const Geo& g, const uint8_t* xb, int t, int tb, int tl,
                                              int hh) {
  ProdUnit pu;
  const long long tile = (long long)tb * 128 + tl;
  pu.live = tile < g.NT;
  int n = 0, ty = 0, tx = 0;
  if (pu.live) {
    const long long per = (long long)g.TP * g.TQ;
    n = (int)(tile / per);
    const int r = (int)(tile - (long long)n * per);
    ty = r / g.TQ;
    tx = r - ty * g.TQ;
  }
  int i0, i1, j0, j1;
  bt_pick(t >> 2, i0, i1, pu.sa0, pu.sa1);
  bt_pick(t & 3, j0, j1, pu.sb0, pu.sb1);
  // byte offsets in an XB record block (n, cb) of the window positions (row
  // 2ty + i, column 2tx - 1 + jc) of channel half hh: column jc lies in
  // parity (jc & 1) ^ 1, entry tx + (jc >> 1)
  const uint32_t rbase = (uint32_t)(2 * ty) * g.RB;
  auto col_off = [&](int jc) {
    return (uint32_t)(((((jc & 1) ^ 1) * 2 + hh) * g.E + tx + (jc >> 1)) * 16);
  };
  pu.o[0] = rbase + i0 * g.RB + col_off(j0);
  pu.o[1] = rbase + i0 * g.RB + col_off(j1);
  pu.o[2] = rbase + i1 * g.RB + col_off(j0);
  pu.o[3] = rbase + i1 * g.RB + col_off(j1);
  pu.xn = xb + (size_t)n * g.CS * g.HP * g.RB;
  return pu;
}

}  // namespace ts

__global__ void __launch_bounds__(ts::NTHREAD, 1) twostage_gemm_kernel(KernelParam p) {
  using namespace ts;
  extern __shared__ __align__(1024) uint8_t smem_raw[];
  __shared__ Shared sh;
  uint8_t* smem = reinterpret_cast<uint8_t*>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
  const Geo g = geo(p);
  const int warp = warp_id(), lane = lane_id();
  uint32_t* err = &g_twostage_err;

  if (threadIdx.x == 0) {
    for (int s = 0; s < NSTAGE; ++s) {
      mbar_init(&sh.full[s], 1 + NWARP_P);
      mbar_init(&sh.empty[s], 1);
    }
    for (int a = 0; a < 2; ++a) {
      mbar_init(&sh.accfull[a], 1);
      mbar_init(&sh.accempty[a], NWARP_E);
    }
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
      for (long long u = blockIdx.x; ok && u < g.nunits && !*abort_flag; u += gridDim.x) {
        int t, tb, kb, kbs[KPU];
        unit_coords(g, u, t, tb, kb, kbs);
        for (int j = 0; j < g.nst; ++j, ++it) {
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
      for (long long u = blockIdx.x; ok && u < g.nunits && !*abort_flag; u += gridDim.x, ++ui) {
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
        for (int j = 0; j < g.nst; ++j, ++it) {
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
    }
    __syncwarp();
  } else if (warp < WARP_E0 + NWARP_E) {
    // epilogue: TMEM lanes 32*quarter .. +31 = tiles of the block
    const int quarter = warp & 3;
    __half* m16 = static_cast<__half*>(p.mid_result);
    const size_t NT = (size_t)g.NT;
    uint32_t ui = 0;
    for (long long u = blockIdx.x; u < g.nunits; u += gridDim.x, ++ui) {
      int t, tb, kb, kbs[KPU];
      unit_coords(g, u, t, tb, kb, kbs);
      const int ab = ui & 1;
      if (!mbar_wait_warp(&sh.accfull[ab], (ui >> 1) & 1, abort_flag, err, ERR_WAIT_ACCUM, SLEEP_EPI_NS)) break;
      tc_fence_after();
      const size_t tile = (size_t)tb * 128 + quarter * 32 + lane;
      const bool live = tile < NT;
      const uint32_t taddr = tmem + ((uint32_t)(quarter * 32) << 16) + ab * (KPU * 128);
      for (int cc = 0; cc < KPU * 128; cc += 16) {
        const int i = cc >> 7, c0 = cc & 127;
        if (c0 >= kbs[i]) continue;
        float v[16];
        tmem_ld16(taddr + cc, v);
        tmem_ld_wait();
        if (live) {
          __half* dst = m16 + ((size_t)t * g.K + (size_t)(kb + i) * KB2 + c0) * NT + tile;
#pragma unroll
          for (int jj = 0; jj < 16; ++jj) dst[(size_t)jj * NT] = __float2half_rn(v[jj]);
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
    const size_t cb_stride = (size_t)g.HP * g.RB;
    uint32_t it = 0;
    bool ok = true;
    for (long long u = blockIdx.x; ok && u < g.nunits && !*abort_flag; u += gridDim.x) {
      int t, tb, kb, kbs[KPU];
      unit_coords(g, u, t, tb, kb, kbs);
      const ProdUnit pu = prod_unit(g, xb, t, tb, tl, hh);
      for (int j = 0; j < g.nst; ++j, ++it) {
        const int st = it % NSTAGE;
        const int nk = min(SK, g.CS - j * SK);
        // the window loads go out before the wait for a free stage: only the
        // shared-memory stores below need it
        uint4 d[SK][4];
#pragma unroll
        for (int kk = 0; kk < SK; ++kk) {
          if (pu.live && kk < nk) {
            const uint8_t* rec = pu.xn + (size_t)(j * SK + kk) * cb_stride;
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
            const uint4 a0 = d[kk][0], a1 = d[kk][1], b0 = d[kk][2], b1 = d[kk][3];
            uint4 v;
            v.x = bt_op(pu.sb0, pu.sb1, bt_op(pu.sa0, pu.sa1, a0.x, b0.x), bt_op(pu.sa0, pu.sa1, a1.x, b1.x));
            v.y = bt_op(pu.sb0, pu.sb1, bt_op(pu.sa0, pu.sa1, a0.y, b0.y), bt_op(pu.sa0, pu.sa1, a1.y, b1.y));
            v.z = bt_op(pu.sb0, pu.sb1, bt_op(pu.sa0, pu.sa1, a0.z, b0.z), bt_op(pu.sa0, pu.sa1, a1.z, b1.z));
            v.w = bt_op(pu.sb0, pu.sb1, bt_op(pu.sa0, pu.sa1, a0.w, b0.w), bt_op(pu.sa0, pu.sa1, a1.w, b1.w));
            *reinterpret_cast<uint4*>(adst + kk * A_STEP) = v;
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

// Output transform: thread = (2 consecutive tiles, k) reading the 16 taps of
// M16 (tile stride = the number of tiles) as one fp16 pair each when the
// tile count is even; Y tile = A^T m A in fp32, one fp16 rounding.
// grid (ceil(tiles / 512), K).
constexpr int OT_TILES = 2;

__global__ void __launch_bounds__(256) twostage_output_kernel(KernelParam p) {
  const int K = p.k, P = p.Oh, Q = p.Ow;
  const int TP = (P + 1) >> 1, TQ = (Q + 1) >> 1;
  const long long NT = (long long)p.n * TP * TQ;
  const long long tile0 = ((long long)blockIdx.x * 256 + threadIdx.x) * OT_TILES;
  const int k = blockIdx.y;
  if (tile0 >= NT) return;
  const int nt = NT - tile0 < OT_TILES ? (int)(NT - tile0) : OT_TILES;
  const __half* m16 = static_cast<const __half*>(p.mid_result);
  const bool vec = (NT & 1) == 0 && (reinterpret_cast<uintptr_t>(m16) & 3) == 0;
  float m[16][OT_TILES];
#pragma unroll
  for (int t = 0; t < 16; ++t) {
    const __half* src = m16 + ((size_t)t * K + k) * (size_t)NT + tile0;
    if (vec) {
      const float2 v = __half22float2(*reinterpret_cast<const __half2*>(src));
      m[t][0] = v.x;
      m[t][1] = v.y;
    } else {
      m[t][0] = __half2float(src[0]);
      m[t][1] = nt > 1 ? __half2float(src[1]) : 0.f;
    }
  }
  const long long per_img = (long long)TP * TQ;
  const bool pair_ok = (Q & 1) == 0 && (reinterpret_cast<uintptr_t>(p.pout) & 3) == 0;
  // both tiles in one tile row with 8-byte aligned output rows: the four
  // columns of each output row go out as one 8-byte store
  float yy[OT_TILES][4];
  int n0 = 0, ty0 = 0, tx0 = 0;
  {
    const int r0 = (int)(tile0 - (long long)(tile0 / per_img) * per_img);
    n0 = (int)(tile0 / per_img);
    ty0 = r0 / TQ;
    tx0 = r0 - ty0 * TQ;
  }
  const bool row_pair = nt == 2 && tx0 + 1 < TQ && (Q & 3) == 0 && (tx0 & 1) == 0 &&
                        (reinterpret_cast<uintptr_t>(p.pout) & 7) == 0;
#pragma unroll
  for (int j = 0; j < OT_TILES; ++j) {
    if (j >= nt) break;
    float z[2][4];
#pragma unroll
    for (int b = 0; b < 4; ++b) {
      z[0][b] = m[b][j] + m[4 + b][j] + m[8 + b][j];
      z[1][b] = m[4 + b][j] - m[8 + b][j] - m[12 + b][j];
    }
    float* y = yy[j];
#pragma unroll
    for (int i = 0; i < 2; ++i) {
      y[2 * i + 0] = z[i][0] + z[i][1] + z[i][2];
      y[2 * i + 1] = z[i][1] - z[i][2] - z[i][3];
    }
    if (row_pair) continue;
    const long long tile = tile0 + j;
    const int n = (int)(tile / per_img);
    const int r = (int)(tile - (long long)n * per_img);
    const int ty = r / TQ, tx = r - ty * TQ;
    const int oy = 2 * ty, ox = 2 * tx;
    __half* o = static_cast<__half*>(p.pout) + (((size_t)n * K + k) * P + oy) * (size_t)Q + ox;
    const bool two_cols = ox + 1 < Q, two_rows = oy + 1 < P;
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
  if (row_pair) {
    const int oy = 2 * ty0, ox = 2 * tx0;
    __half* o = static_cast<__half*>(p.pout) + (((size_t)n0 * K + k) * P + oy) * (size_t)Q + ox;
#pragma unroll
    for (int i = 0; i < 2; ++i) {
      if (oy + i >= P) break;
      const __half2 a = __floats2half2_rn(yy[0][2 * i], yy[0][2 * i + 1]);
      const __half2 b = __floats2half2_rn(yy[1][2 * i], yy[1][2 * i + 1]);
      uint2 pk;
      pk.x = *reinterpret_cast<const uint32_t*>(&a);
      pk.y = *reinterpret_cast<const uint32_t*>(&b);
      *reinterpret_cast<uint2*>(o + (size_t)i * Q) = pk;
    }
  }
}

}  // namespace wino

using namespace wino;

extern "C" {

void* wino_twostage_gemm_kernel_ptr() { return (void*)twostage_gemm_kernel; }
void* wino_twostage_output_kernel_ptr() { return (void*)twostage_output_kernel; }
int wino_twostage_threads() { return ts::NTHREAD; }
int wino_twostage_smem_bytes() { return ts::SMEM_BYTES; }

int wino_twostage_prepare() {
  return (int)cudaFuncSetAttribute(twostage_gemm_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                   ts::SMEM_BYTES);
}

// Tiles and the M16 bytes of a shape (tile stride = tiles, no padding).
long long wino_twostage_tiles(int n, int h, int w) { return (long long)n * ((h + 1) / 2) * ((w + 1) / 2); }
size_t wino_twostage_m_bytes(int n, int h, int w, int k) {
  return (size_t)16 * (size_t)k * (size_t)wino_twostage_tiles(n, h, w) * 2;
}

// GEMM grid: one CTA per SM up to the number of work units.
unsigned wino_twostage_gemm_grid(int n, int h, int w, int k, int sms) {
  const long long ntb = (wino_twostage_tiles(n, h, w) + 127) / 128;
  const long long nkp = ((k + KB2 - 1) / KB2 + ts::KPU - 1) / ts::KPU;
  const long long units = 16LL * ntb * nkp;
  return (unsigned)(units < sms ? units : sms);
}

void wino_twostage_output_grid(int n, int h, int w, int k, unsigned* gx, unsigned* gy) {
  *gx = (unsigned)((wino_twostage_tiles(n, h, w) + 256 * OT_TILES - 1) / (256 * OT_TILES));
  *gy = (unsigned)k;
}

uint32_t wino_twostage_error_read_clear() {
  uint32_t v = 0, z = 0;
  cudaMemcpyFromSymbol(&v, g_twostage_err, sizeof(v));
  cudaMemcpyToSymbol(g_twostage_err, &z, sizeof(z));
  return v;
}

}  // extern "C"
