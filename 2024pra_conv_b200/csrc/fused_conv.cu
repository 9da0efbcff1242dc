// Fused Winograd F(2x2,3x3) conv2d for sm_100a: input transform, the 16
// per-tap channel GEMMs on tcgen05 tensor cores, and the output transform in
// one persistent kernel.  Only the NCHW input, the cached U and the NKPQ
// output touch global memory.
//
// Reference path replaced (reference files):
//   input transform  B^T d B    src/preprocessing.cuh:273-424 (BTdB1/2/3)
//   16 tap GEMMs                src/matrixmul.cuh:139-556 (matrixMul1/3/4/5/6)
//   output transform A^T m A    src/conv2d.cpp:17-250 (store, store1..5)
// which there run as three kernels with V and M round-tripping through HBM.
//
// Work unit ("block"): 128 output channels x 32 consecutive Winograd tiles.
// Per tap t the tensor core computes
//     M_t[k][tile] = sum_c U_t[k][c] * V_t[c][tile]
// as a 128 x 32 x 16 MMA per 16-channel step (A = U from the U cache, B = V
// produced on chip, both K-major), accumulating in TMEM: lane = output channel, columns
// t*32 .. t*32+31 = tiles (16 taps x 32 = all 512 columns).  All 16 taps of
// a (k, tile) pair live in one thread's lane, so the output transform is
// per-thread register arithmetic.  With output channels on the 128-row side
// each V element feeds 128 channels, which keeps the CUDA-core input
// transform small next to the MMAs.
//
// Pipelines (shared memory, 225 KB): U in four 32 KB slots, each holding
// 8 taps of a step (a step's two halves, two steps in flight); V in three
// 16 KB slots, one per step; two 16 KB input slabs; 16 KB of epilogue store
// staging.  The MMA thread commits once per step (each tcgen05.commit stalls
// the MMA pipe for ~90 cycles on this part) to a "step done" barrier that
// releases that step's U slots and V slot together.
//
// Precision variants of the GEMM stage (template parameter VAR):
//   VAR_F16       fp16 U and V (the drop-in path), 16 channels per step;
//   VAR_BF16      bf16 U and V: V formed in fp16 then rounded to bf16;
//   VAR_F8        fp8 e4m3 U and V, 32 channels per step (kind::f8f6f4,
//                 K = 32): V is scaled per input channel (1 / sv[c]) before
//                 rounding, sv folded into the cached U, and U carries a
//                 per-(tap, output channel) scale su[t][k] that the
//                 epilogue applies;
//   VAR_F16_HILO  fp16 V against U = U_hi + U_lo (two fp16 caches): every
//                 tap GEMM runs twice into the same accumulator, four U
//                 pieces per step.
//
// Warp roles (15 warps):
//   warp 0       TMEM allocation; one thread issues the MMAs
//   warp 4       lanes 0 and 1 bulk-copy the two U halves of a step (one
//                copy in flight per issuing thread, so two threads)
//   warps 1,2,3,5 V producers, all four on every step: producer q forms channel
//                half q&1 (8 channels) of tap rows 2(q>>1), 2(q>>1)+1 (8
//                taps) of the step's V for all 32 tiles (lane = tile):
//                B^T d B in packed fp16 straight into the K-major operand
//                (8 tiles x 8 channels per core matrix, one 16-byte row per
//                lane and tap).  They read the step's slab, or, without an
//                XB workspace or when a block's rows exceed a slab, the NCHW
//                input directly.
//   warps 7-14   epilogue: drain TMEM one tap half at a time (the block's
//                last MMAs commit each half separately, and each drained half
//                goes back to the MMA thread at once, so the drain overlaps
//                the MMAs on both sides), A^T m A in fp32, fp16 NKPQ stores.
//   warp 6       stager: with an XB workspace (p.transform_pin, written by
//                the pre-pass of input_layout.cu) bulk-copies each step's
//                input rows into a slab, up to two steps ahead (one copy
//                per image the block touches, issued from separate lanes).
#include <cuda_runtime.h>
#include "tc_sm100.cuh"
#include "wino_common.cuh"
#include "vgen.cuh"
#include "wino_batch.h"

// Back-off (ns) between polls of a waiting warp once its wait is long:
// producers, stager, epilogue.
#ifndef WINO_SLEEP_PROD
#define WINO_SLEEP_PROD 32
#endif
#ifndef WINO_SLEEP_STAGE
#define WINO_SLEEP_STAGE 64
#endif
#ifndef WINO_SLEEP_EPI
#define WINO_SLEEP_EPI 64
#endif

namespace wino {

static __device__ uint32_t g_fused_err;


namespace fused {

constexpr int TILES = 32;              // MMA N: tiles per block
constexpr int NTAP = 16;
constexpr int V_TAP_BYTES = TILES * 32;              // 1 KB per tap per step (32 B per tile)
constexpr int V_SLOT_BYTES = NTAP * V_TAP_BYTES;     // 16 KB: one step of V
constexpr int U_HALF_BYTES = 8 * KB * 32;            // 32 KB: 8 taps x 128 k x 32 B
constexpr int NUH = 4;                 // U slots
constexpr int NVSLOT = 3, NSD = 3, NSLAB = 2;
constexpr int EPI_WARP_BYTES = 2048;   // epilogue store staging per warp
constexpr int U_BASE = 0, V_BASE = NUH * U_HALF_BYTES;
constexpr int SLAB_BASE = V_BASE + NVSLOT * V_SLOT_BYTES;
constexpr int EPI_BASE = SLAB_BASE + NSLAB * SLAB_BYTES;
constexpr int NWARP = 15;
constexpr int NTHREAD = NWARP * 32;
// Warp w issues from scheduler (SMSP) w % 4.  The single MMA-issuing thread
// must not share its scheduler with a busy warp (it was measured starved to
// ~95 cycles per MMA next to a V producer), so scheduler 0 holds only the MMA
// warp, the mostly waiting U loader and the two epilogue warps that TMEM lane
// access pins there (warp w reads TMEM lanes 32*(w%4) ..): producers run on
// schedulers 1-3.
constexpr int WARP_MMA = 0, WARP_U = 4, WARP_S = 6, NWARP_V = 4, WARP_E0 = 7, NWARP_E = 8;
// producer index of a warp (warps 1, 2, 3, 5), or -1
__device__ __forceinline__ int producer_index(int warp) {
  return warp >= 1 && warp <= 3 ? warp - 1 : (warp == 5 ? 3 : -1);
}
constexpr int SMEM_BYTES = EPI_BASE + 8 * EPI_WARP_BYTES + 1024;

struct Shared {
  uint64_t ufull[NUH];
  uint64_t vfull[NVSLOT];
  uint64_t sdone[NSD];                 // MMAs of step it complete: sdone[it % NSD]
  uint64_t slabfull[NSLAB], slabfree[NSLAB];
  uint64_t accf[2];                    // last MMAs of a block done, per tap half
  uint64_t tapfree[2];                 // epilogue drained a tap half of TMEM
  uint32_t tmem_base;
  int abort_flag;
};

// Output-transform coefficient of tap t = 4a+b for output (i, j):
// At[i][a] * At[j][b] with At = [[1,1,1,0],[0,1,-1,-1]].
__host__ __device__ constexpr int at_coef(int i, int a) {
  return i == 0 ? (a == 3 ? 0 : 1) : (a == 0 ? 0 : (a == 1 ? 1 : -1));
}

// Per-variant constants: channels per step, U pieces (8 taps each) per
// step, operand format code of the instruction descriptor.
template <int VAR>
struct Traits {
  static constexpr int CH = VAR == VAR_F8 ? 32 : 16;
  static constexpr int UP = VAR == VAR_F16_HILO ? 4 : 2;
  static constexpr uint32_t FMT = VAR == VAR_BF16 ? 1u : 0u;  // bf16 / (f16 or e4m3)
  static constexpr int NCB = CH / 16;                          // XB channel blocks per step
};

// fp16x2 -> bf16x2 (round to nearest even through fp32).
__device__ __forceinline__ uint32_t h2_to_bf2(uint32_t w) {
  const float2 f = __half22float2(*reinterpret_cast<const __half2*>(&w));
  const __nv_bfloat162 b = __floats2bfloat162_rn(f.x, f.y);
  return *reinterpret_cast<const uint32_t*>(&b);
}

// (scale * fp16x2) -> two e4m3 bytes in the low 16 bits (saturating).
__device__ __forceinline__ uint32_t h2_to_e4m3x2(uint32_t w, uint32_t scale2) {
  uint32_t x = hmul2_u32(w, scale2);
  uint16_t r;
  asm("cvt.rn.satfinite.e4m3x2.f16x2 %0, %1;" : "=h"(r) : "r"(x));
  return r;
}

}  // namespace fused

using namespace fused;

// ---- work blocks --------------------------------------------------------
// A persistent CTA walks work blocks b = blockIdx.x, + gridDim.x, ...; every
// role walks the same sequence and asks its block source for the block's
// layer arguments and coordinates, so one kernel serves one layer or a
// table of layers (schedule configuration bits CFG_* in wino_batch.h).
struct BlockInfo {
  Geometry g;
  const __half* x;          // NCHW input
  __half* y;                // NKPQ output
  float* y32;               // split blocks: fp32 partial-sum output, else null
  const uint8_t* xb;        // XB records, or null (direct reads)
  const uint8_t* u;         // U cache
  int tb, kb;               // tile block, k block
  int split, per;           // split index, 16-channel steps per split (per = 0: all)
};

// Steps [s0, s1) of a block for a kernel stepping `ch` channels at a time.
__device__ __forceinline__ void block_steps(const BlockInfo& B, int ch, int& s0, int& s1) {
  const int cs = B.g.C / ch;
  if (B.per == 0) {
    s0 = 0;
    s1 = cs;
  } else {
    s0 = B.split * B.per;
    s1 = min(cs, s0 + B.per);
  }
}

__device__ __forceinline__ void block_coords(long long lb, const Geometry& g, int cfg, int& tb, int& kb) {
  if (cfg & CFG_KMAJOR) {
    kb = (int)(lb / g.nTB);
    tb = (int)(lb - (long long)kb * g.nTB);
  } else {
    tb = (int)(lb / g.nKB);
    kb = (int)(lb - (long long)tb * g.nKB);
  }
}

// Work blocks of a layer: (tile block, k block, split), splits innermost.
__device__ __forceinline__ BlockInfo make_block(const KernelParam& p, const Geometry& g, int cfg, long long lb) {
  BlockInfo B;
  B.g = g;
  B.x = static_cast<const __half*>(p.pin);
  B.y = static_cast<__half*>(p.pout);
  B.xb = (cfg & CFG_DIRECT) ? nullptr : static_cast<const uint8_t*>(p.transform_pin);
  B.u = static_cast<const uint8_t*>(p.transform_filter);
  int nsplit, per;
  split_plan(cfg, g.CS, nsplit, per);
  if (nsplit > 1) {
    B.split = (int)(lb % nsplit);
    lb /= nsplit;
    B.per = per;
    B.y32 = static_cast<float*>(p.mid_result);
  } else {
    B.split = 0;
    B.per = 0;
    B.y32 = nullptr;
  }
  block_coords(lb, g, cfg, B.tb, B.kb);
  return B;
}

__device__ __forceinline__ long long layer_blocks(const Geometry& g, int cfg) {
  int nsplit, per;
  split_plan(cfg, g.CS, nsplit, per);
  return g.nblocks * nsplit;
}

// One layer (the drop-in and single-conv entry points).
struct OneLayer {
  KernelParam p;
  Geometry g;
  int cfg;
  __device__ long long total() const { return layer_blocks(g, cfg); }
  __device__ BlockInfo get(long long b) const { return make_block(p, g, cfg, b); }
};

// A table of layers in global memory, blocks concatenated in table order
// (the batched persistent launch); entries are read through the read-only
// cache.
struct LayerTable {
  const BatchTable* t;
  long long tot;
  __device__ long long total() const { return tot; }
  __device__ BlockInfo get(long long b) const {
    int l = 0;
    const int nl = __ldg(&t->nlayers);
    while (l + 1 < nl && __ldg(&t->layer[l + 1].block_begin) <= b) ++l;
    const LayerDesc& d = t->layer[l];
    KernelParam p;
    p.pin = (void*)__ldg((const unsigned long long*)&d.p.pin);
    p.pout = (void*)__ldg((const unsigned long long*)&d.p.pout);
    p.transform_pin = (void*)__ldg((const unsigned long long*)&d.p.transform_pin);
    p.transform_filter = (void*)__ldg((const unsigned long long*)&d.p.transform_filter);
    p.n = __ldg(&d.p.n); p.c = __ldg(&d.p.c); p.h = __ldg(&d.p.h); p.w = __ldg(&d.p.w);
    p.k = __ldg(&d.p.k); p.Oh = __ldg(&d.p.Oh); p.Ow = __ldg(&d.p.Ow);
    const Geometry g = make_geometry(p, TILES);
    return make_block(p, g, __ldg(&d.cfg), b - __ldg(&d.block_begin));
  }
};

template <int VAR, typename Sched>
__device__ __forceinline__ void fused_body(const Sched& sched, const VariantArgs& va) {
  using T = Traits<VAR>;
  extern __shared__ __align__(1024) uint8_t smem_raw[];
  __shared__ Shared sh;
  uint8_t* smem = reinterpret_cast<uint8_t*>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
  const long long nblocks = sched.total();
  const int warp = warp_id();
  const int lane = lane_id();
  uint32_t* err = &g_fused_err;

  if (threadIdx.x == 0) {
    for (int s = 0; s < NUH; ++s) mbar_init(&sh.ufull[s], 1);
    for (int s = 0; s < NVSLOT; ++s) mbar_init(&sh.vfull[s], NWARP_V);  // every producer warp
    for (int s = 0; s < NSD; ++s) mbar_init(&sh.sdone[s], 1);
    for (int s = 0; s < NSLAB; ++s) {
      mbar_init(&sh.slabfull[s], 1);          // the staging lane (plus the copies' bytes)
      mbar_init(&sh.slabfree[s], NWARP_V);
    }
    for (int h = 0; h < 2; ++h) {
      mbar_init(&sh.accf[h], 1);
      mbar_init(&sh.tapfree[h], NWARP_E);
    }
    sh.abort_flag = 0;
    fence_barrier_init();
  }
  if (warp == WARP_MMA) {
    tmem_alloc(&sh.tmem_base, 512);
    tmem_relinquish();
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = sh.tmem_base;
  volatile int* abort_flag = &sh.abort_flag;
  const uint32_t smem_base = smem_u32(smem);
  auto u_slot = [&](uint32_t s) { return smem_base + U_BASE + s * U_HALF_BYTES; };
  auto v_slot = [&](uint32_t s) { return smem_base + V_BASE + s * V_SLOT_BYTES; };
  // Slot bookkeeping for step `it` (counted over this CTA's blocks):
  //   V slot it % NVSLOT, reused at it + NVSLOT (after sdone of step it);
  //   U piece pi = UP * it + j (j < UP) in slot pi % NUH, reused by piece
  //     pi + NUH (after sdone of step it);
  //   slab it % NSLAB, reused at it + NSLAB (after the producers' slabfree).
  // A waiter on sdone[j] for step it cannot miss its phase: the barrier's
  // next phase needs operands the waiter has not supplied yet.

  if (warp == WARP_MMA) {
    if (lane == 0) {
      const uint32_t idesc = instr_desc(128, TILES, T::FMT, T::FMT, /*a_mn=*/0, /*b_mn=*/0);
      // Descriptors are formed once; the start-address field (bits 0-13,
      // address >> 4) then advances by plain adds (shared addresses < 256 KB,
      // so the field never carries into the next one).  Keeping the issue
      // loop to a few instructions per MMA matters: a single thread feeds the
      // tensor pipe.
      const uint64_t adesc0 = smem_desc(u_slot(0), 128, 256);
      const uint64_t bdesc0 = smem_desc(v_slot(0), 128, 256);
      constexpr uint32_t BSTEP = V_TAP_BYTES >> 4;
      uint32_t it = 0, bi = 0;
      bool ok = true;
      for (long long b = blockIdx.x; b < nblocks && ok; b += gridDim.x, ++bi) {
        const BlockInfo B = sched.get(b);
        int s0, s1;                            // steps of the block
        block_steps(B, T::CH, s0, s1);
        const uint32_t astep = (uint32_t)(kblock_rows(B.kb, B.g.K) * 32) >> 4;
        for (int s = s0; s < s1 && ok; ++s, ++it) {
          const uint32_t vs = it % NVSLOT;
          ok = mbar_wait(&sh.vfull[vs], (it / NVSLOT) & 1, abort_flag, err, ERR_WAIT_FULL);
          const bool first_step = s == s0 && bi > 0;
#pragma unroll
          for (int j = 0; j < T::UP; ++j) {
            if (!ok) break;
            const int h = j & 1;               // tap half
            const uint32_t pi = T::UP * it + j, us = pi % NUH;
            ok = mbar_wait(&sh.ufull[us], (pi / NUH) & 1, abort_flag, err, ERR_WAIT_FULL);
            if (!ok) break;
            const uint64_t ad = adesc0 + ((us * U_HALF_BYTES) >> 4);
            const uint64_t bd = bdesc0 + ((vs * V_SLOT_BYTES + 8 * h * V_TAP_BYTES) >> 4);
            const uint32_t d = tmem + 8 * h * TILES;
            const uint32_t acc = (s > s0 || j >= 2) ? 1u : 0u;
            if (first_step && j < 2) {
              // the previous block's epilogue hands back each tap half of TMEM
              if (!mbar_wait(&sh.tapfree[h], (bi - 1) & 1, abort_flag, err, ERR_WAIT_DRAIN)) {
                ok = false;
                break;
              }
              tc_fence_after();
            }
#pragma unroll
            for (int tt = 0; tt < 8; ++tt) {
              if constexpr (VAR == VAR_F8)
                mma_f8(d + tt * TILES, ad + tt * astep, bd + tt * BSTEP, idesc, acc);
              else
                mma_f16(d + tt * TILES, ad + tt * astep, bd + tt * BSTEP, idesc, acc);
            }
            // after the block's last MMAs of a tap half the epilogue may drain it
            if (s == s1 - 1 && j >= T::UP - 2) mma_commit(&sh.accf[h]);
          }
          if (ok) mma_commit(&sh.sdone[it % NSD]);
        }
      }
    }
    __syncwarp();
  } else if (warp == WARP_U) {
    if (lane < T::UP) {
      // lane j copies piece j of every step (one copy in flight per thread)
      const int j = lane;
      uint32_t it = 0;
      bool ok = true;
      for (long long b = blockIdx.x; b < nblocks && ok; b += gridDim.x) {
        const BlockInfo B = sched.get(b);
        const Geometry& g = B.g;
        int s0, s1;
        block_steps(B, T::CH, s0, s1);
        const uint8_t* ubase = (VAR == VAR_F16_HILO && j >= 2) ? static_cast<const uint8_t*>(va.u_lo) : B.u;
        const int kb = B.kb;
        const int kbs = kblock_rows(kb, g.K);
        const uint32_t bytes = 8 * kbs * 32;  // 8 taps x kbs rows x 32 B
        for (int s = s0; s < s1; ++s, ++it) {
          const uint32_t pi = T::UP * it + j, us = pi % NUH;
          if (pi >= NUH) {
            const uint32_t st = (pi - NUH) / T::UP;  // step that last used the slot
            if (!mbar_wait(&sh.sdone[st % NSD], (st / NSD) & 1, abort_flag, err, ERR_WAIT_EMPTY)) {
              ok = false;
              break;
            }
          }
          // byte offset of the (k-block, step) piece: a k-block holds 16 x KB x C
          // elements, a step 16 taps x kbs rows x 32 B
          const size_t piece = (size_t)kb * KB * 16 * g.C * (VAR == VAR_F8 ? 1 : 2) +
                               (size_t)s * 16 * kbs * 32;
          mbar_arrive_expect_tx(&sh.ufull[us], bytes);
          bulk_g2s(smem + U_BASE + us * U_HALF_BYTES, ubase + piece + (size_t)(j & 1) * bytes, bytes,
                   &sh.ufull[us]);
        }
      }
      if (*abort_flag) __nanosleep(20000);  // let copies already issued land
    }
    __syncwarp();
  } else if (warp == WARP_S) {
    uint32_t it = 0;
    bool ok = true;
    // lane = segment + 4 * channel block of the step
    const int seg = lane & 3, cbi = lane >> 2;
    for (long long b = blockIdx.x; b < nblocks && ok; b += gridDim.x) {
      const BlockInfo B = sched.get(b);
      const Geometry& g = B.g;
      int s0, s1;
      block_steps(B, T::CH, s0, s1);
      const uint8_t* XB = B.xb;
      const uint32_t RB = (uint32_t)xb_row_bytes(g.W);
      const size_t img_stride = (size_t)(g.C >> 4) * xb_rows(g.H) * RB;   // one image of XB
      const size_t cb_stride = (size_t)xb_rows(g.H) * RB;                  // one channel block
      const int tile0 = B.tb * TILES;
      const SlabPlan pl = slab_plan(g, tile0, TILES);
      const bool use = XB != nullptr && slab_fits(g, pl, T::NCB);
      int ta = 0, rows = 0, rbase = 0;  // this lane's segment
#pragma unroll
      for (int k = 0; k < SLAB_MAXSEG; ++k)
        if (seg == k) { ta = pl.ta[k]; rows = pl.rows[k]; rbase = pl.row_base[k]; }
      const uint8_t* src0 = XB + (size_t)(pl.n0 + seg) * img_stride + (size_t)cbi * cb_stride +
                            (size_t)(2 * ta) * RB;
      const uint32_t dst0 = (uint32_t)(cbi * pl.total_rows + rbase) * RB;
      for (int s = s0; s < s1; ++s, ++it) {
        const uint32_t j = it % NSLAB;
        if (it >= NSLAB &&
            !mbar_wait_warp(&sh.slabfree[j], ((it - NSLAB) / NSLAB) & 1, abort_flag, err, ERR_WAIT_EMPTY, WINO_SLEEP_STAGE)) {
          ok = false;
          break;
        }
        if (use) {
          if (lane == 0) mbar_arrive_expect_tx(&sh.slabfull[j], (uint32_t)(T::NCB * pl.total_rows) * RB);
          __syncwarp();
          if (seg < pl.nseg && cbi < T::NCB)
            bulk_g2s(smem + SLAB_BASE + j * SLAB_BYTES + dst0, src0 + (size_t)s * T::NCB * cb_stride,
                     (uint32_t)rows * RB, &sh.slabfull[j]);
        } else if (lane == 0) {
          mbar_arrive(&sh.slabfull[j]);
        }
      }
    }
    if (*abort_flag) __nanosleep(20000);  // let copies already issued land
    __syncwarp();
  } else if (producer_index(warp) >= 0) {
    const int q = producer_index(warp);
    const int hh = q & 1;                     // K half of the step's operand row
    const int ar = q >> 1;                    // tap rows 2ar, 2ar+1 (taps 8ar .. 8ar+7)
    const uint32_t slab0 = smem_base + SLAB_BASE;
    bool ok = true;
    // K-major core matrices: tile group (lane/8) at 256 B, K half at 128 B,
    // tile row (lane%8) at 16 B: each lane writes whole 16-byte rows, eight
    // lanes 128 contiguous bytes (conflict-free).
    const uint32_t row_off = (lane >> 3) * 256 + hh * 128 + (lane & 7) * 16 + ar * 8 * V_TAP_BYTES;
    uint32_t it = 0;
    for (long long b = blockIdx.x; b < nblocks && ok; b += gridDim.x) {
      // per-block quantities once per block, 32-bit
      const BlockInfo B = sched.get(b);
      const Geometry& g = B.g;
      int s0, s1;
      block_steps(B, T::CH, s0, s1);
      const __half* X = B.x;
      const int tile0 = B.tb * TILES;
      const SlabPlan pl = slab_plan(g, tile0, TILES);
      const bool use_slab = B.xb != nullptr && slab_fits(g, pl, T::NCB);
      const TileCoord tc = tile_coord(g, tile0 + lane, tile0);
      // fp8: this warp's K half is a whole XB channel block (two 8-channel
      // halves), the second block of the step's slab for hh = 1
      const uint32_t cb_off = VAR == VAR_F8 ? (uint32_t)(hh * pl.total_rows) * (uint32_t)xb_row_bytes(g.W) : 0u;
      const SlabWindow sw0 = slab_window(g, pl, tc, VAR == VAR_F8 ? 0 : hh);
      const SlabWindow sw1 = slab_window(g, pl, tc, 1);
      for (int s = s0; s < s1 && ok; ++s, ++it) {
        const uint32_t j = it % NSLAB;
        const uint32_t vs = it % NVSLOT;
        if (!mbar_wait_warp(&sh.slabfull[j], (it / NSLAB) & 1, abort_flag, err, ERR_WAIT_FULL, WINO_SLEEP_PROD)) {
          ok = false;
          break;
        }
        if (it >= NVSLOT &&
            !mbar_wait_warp(&sh.sdone[(it - NVSLOT) % NSD], ((it - NVSLOT) / NSD) & 1, abort_flag, err,
                            ERR_WAIT_EMPTY, WINO_SLEEP_PROD)) {
          ok = false;
          break;
        }
        const uint32_t dst = v_slot(vs) + row_off;
        const uint32_t slab = slab0 + j * SLAB_BYTES + cb_off;
        if constexpr (VAR == VAR_F8) {
          // 16 channels c0 .. c0+15, two 8-channel halves, 8 bytes each
          const int c0 = s * 32 + 16 * hh;
#pragma unroll
          for (int half = 0; half < 2; ++half) {
            uint32_t sc[4];
#pragma unroll
            for (int pp = 0; pp < 4; ++pp) sc[pp] = va.inv_sv2[(c0 + 8 * half) / 2 + pp];
            auto sink = [&](int u, const uint32_t (&w)[4]) {
              const uint32_t lo = h2_to_e4m3x2(w[0], sc[0]) | (h2_to_e4m3x2(w[1], sc[1]) << 16);
              const uint32_t hi = h2_to_e4m3x2(w[2], sc[2]) | (h2_to_e4m3x2(w[3], sc[3]) << 16);
              asm volatile("st.shared.v2.b32 [%0], {%1, %2};" ::"r"(dst + u * V_TAP_BYTES + half * 8),
                           "r"(lo), "r"(hi)
                           : "memory");
            };
            if (use_slab) {
              const SlabWindow& sw = half ? sw1 : sw0;
              if (ar == 0) produce_v_half_xb<0>(slab, sw, sink);
              else produce_v_half_xb<1>(slab, sw, sink);
            } else {
#pragma unroll 1
              for (int qq = 0; qq < 2; ++qq) {
                auto qsink = [&](int t, uint32_t w0, uint32_t w1) {
                  if ((t >> 3) == ar) {
                    const uint32_t v = h2_to_e4m3x2(w0, sc[2 * qq]) | (h2_to_e4m3x2(w1, sc[2 * qq + 1]) << 16);
                    asm volatile("st.shared.b32 [%0], %1;" ::"r"(dst + (t & 7) * V_TAP_BYTES + half * 8 + qq * 4),
                                 "r"(v)
                                 : "memory");
                  }
                };
                produce_v_quarter_global(X, g, tc, c0 + 8 * half + 4 * qq, qsink);
              }
            }
          }
        } else {
          if (use_slab) {
            auto sink = [&](int u, const uint32_t (&w)[4]) {
              if constexpr (VAR == VAR_BF16)
                st_shared_v4(dst + u * V_TAP_BYTES, h2_to_bf2(w[0]), h2_to_bf2(w[1]), h2_to_bf2(w[2]),
                             h2_to_bf2(w[3]));
              else
                st_shared_v4(dst + u * V_TAP_BYTES, w[0], w[1], w[2], w[3]);
            };
            if (ar == 0)
              produce_v_half_xb<0>(slab, sw0, sink);
            else
              produce_v_half_xb<1>(slab, sw0, sink);
          } else {
            // direct NCHW reads: two channel quarters, keeping this warp's taps
#pragma unroll 1
            for (int qq = 0; qq < 2; ++qq) {
              auto sink = [&](int t, uint32_t w0, uint32_t w1) {
                if ((t >> 3) == ar) {
                  if constexpr (VAR == VAR_BF16) {
                    w0 = h2_to_bf2(w0);
                    w1 = h2_to_bf2(w1);
                  }
                  asm volatile("st.shared.v2.b32 [%0], {%1, %2};" ::"r"(dst + (t & 7) * V_TAP_BYTES + qq * 8),
                               "r"(w0), "r"(w1)
                               : "memory");
                }
              };
              produce_v_quarter_global(X, g, tc, s * 16 + 8 * hh + 4 * qq, sink);
            }
          }
        }
        fence_proxy_async_shared();
        __syncwarp();
        if (lane == 0) {
          mbar_arrive(&sh.slabfree[j]);
          mbar_arrive(&sh.vfull[vs]);
        }
      }
    }
  } else if (warp >= WARP_E0 && warp < WARP_E0 + NWARP_E) {
    const int quarter = warp & 3;            // TMEM lanes 32*quarter .. +31 = channels
    const int half = (warp - WARP_E0) >> 2;  // tiles 16*half .. +15 of the block
    uint32_t bi = 0;
    bool ok = true;
    for (long long b = blockIdx.x; b < nblocks && ok; b += gridDim.x, ++bi) {
      const BlockInfo B = sched.get(b);
      const Geometry& g = B.g;
      __half* Y = B.y;
      const bool q_even = (g.Q & 1) == 0;
      const long long tb = B.tb;
      const int kb = B.kb;
      const int kbs = kblock_rows(kb, g.K);
      float y[16][4];
#pragma unroll
      for (int j = 0; j < 16; ++j)
#pragma unroll
        for (int o = 0; o < 4; ++o) y[j][o] = 0.f;
      const uint32_t tbase = tmem + ((uint32_t)(quarter * 32) << 16) + half * 16;
      // fp8: per-(tap, output channel) scale of U
      float su[NTAP];
      if constexpr (VAR == VAR_F8) {
        const int kc = min(kb * KB + quarter * 32 + lane, g.K - 1);
#pragma unroll
        for (int t = 0; t < NTAP; ++t) su[t] = va.su[t * g.K + kc];
      }
#pragma unroll
      for (int t = 0; t < NTAP; ++t) {
        if ((t & 7) == 0) {
          if (!mbar_wait_warp(&sh.accf[t >> 3], bi & 1, abort_flag, err, ERR_WAIT_ACCUM, WINO_SLEEP_EPI)) {
            ok = false;
            break;
          }
          tc_fence_after();
        }
        float m[16];
        tmem_ld16(tbase + t * TILES, m);
        tmem_ld_wait();
        if ((t & 7) == 7) {
          tc_fence_before();
          __syncwarp();
          if (lane == 0) mbar_arrive(&sh.tapfree[t >> 3]);
        }
        if constexpr (VAR == VAR_F8) {
#pragma unroll
          for (int j = 0; j < 16; ++j) m[j] *= su[t];
        }
        const int a = t >> 2, bc = t & 3;
        const float c00 = (float)(at_coef(0, a) * at_coef(0, bc));
        const float c01 = (float)(at_coef(0, a) * at_coef(1, bc));
        const float c10 = (float)(at_coef(1, a) * at_coef(0, bc));
        const float c11 = (float)(at_coef(1, a) * at_coef(1, bc));
#pragma unroll
        for (int j = 0; j < 16; ++j) {
          y[j][0] += c00 * m[j];
          y[j][1] += c01 * m[j];
          y[j][2] += c10 * m[j];
          y[j][3] += c11 * m[j];
        }
      }
      if (!ok) break;
      if (B.y32 != nullptr) {
        // split block: add this block's fp32 partial outputs
        const int kk = quarter * 32 + lane;
        if (kk < kbs) {
          const int per_img = g.TP * g.TQ;
#pragma unroll
          for (int jt = 0; jt < 16; ++jt) {
            const int tile = (int)tb * TILES + half * 16 + jt;
            if (tile < (int)g.NT) {
              const int n = tile / per_img;
              const int rr = tile - n * per_img;
              const int ty = rr / g.TQ;
              const int oy = 2 * ty, ox = 2 * (rr - ty * g.TQ);
              float* o = B.y32 + (((size_t)n * g.K + (size_t)(kb * KB + kk)) * g.P + oy) * (size_t)g.Q + ox;
              atomicAdd(o, y[jt][0]);
              if (ox + 1 < g.Q) atomicAdd(o + 1, y[jt][1]);
              if (oy + 1 < g.P) {
                atomicAdd(o + g.Q, y[jt][2]);
                if (ox + 1 < g.Q) atomicAdd(o + g.Q + 1, y[jt][3]);
              }
            }
          }
        }
        continue;
      }
      // Stores go through a 2 KB per-warp staging buffer, 8 tiles at a time:
      // thread k writes its outputs as [k][row][8 tiles] half2 (16-byte
      // chunks XOR-swizzled by k so the writes are conflict-free), then each
      // store instruction writes 4 runs of 8 consecutive tiles (32 B of one
      // output row of one channel) instead of 32 scattered words.
      const uint32_t ebuf = smem_base + EPI_BASE + (uint32_t)(warp - WARP_E0) * EPI_WARP_BYTES;
      const int kq = quarter * 32;             // first channel of this warp in the k-block
      const size_t PQ = (size_t)g.P * g.Q;
      // Fused epilogue (optional): + bias[k] in fp32 here; + residual and
      // ReLU at the coalesced store below (ReLU here when there is no
      // residual).
      constexpr bool kEpi = VAR == VAR_F16;   // the fused epilogue is an fp16-path option
      if (kEpi && va.bias != nullptr) {
        const float bk = va.bias[min(kb * KB + kq + lane, g.K - 1)];
#pragma unroll
        for (int j = 0; j < 16; ++j)
#pragma unroll
          for (int o = 0; o < 4; ++o) y[j][o] += bk;
      }
      if (kEpi && va.relu && va.residual == nullptr) {
#pragma unroll
        for (int j = 0; j < 16; ++j)
#pragma unroll
          for (int o = 0; o < 4; ++o) y[j][o] = fmaxf(y[j][o], 0.f);
      }
      const __half* R = kEpi ? static_cast<const __half*>(va.residual) : nullptr;
#pragma unroll
      for (int r = 0; r < 2; ++r) {
        __syncwarp();  // the previous round's reads are done
#pragma unroll
        for (int c = 0; c < 4; ++c) {          // c = row * 2 + tile quad
          const int row = c >> 1, j0 = 8 * r + 4 * (c & 1);
          uint32_t w[4];
#pragma unroll
          for (int u = 0; u < 4; ++u) {
            const __half2 h2 = __floats2half2_rn(y[j0 + u][2 * row], y[j0 + u][2 * row + 1]);
            w[u] = *reinterpret_cast<const uint32_t*>(&h2);
          }
          st_shared_v4(ebuf + lane * 64 + ((c ^ ((lane >> 1) & 3)) << 4), w[0], w[1], w[2], w[3]);
        }
        __syncwarp();
        const int jj = lane & 7;                // tile within the round
        const int tile = (int)tb * TILES + half * 16 + 8 * r + jj;
        const bool tvalid = tile < (int)g.NT;
        const int per_img = g.TP * g.TQ;
        const int tt = tvalid ? tile : 0;
        const int n = tt / per_img;
        const int rr = tt - n * per_img;
        const int ty = rr / g.TQ;
        const int oy = 2 * ty, ox = 2 * (rr - ty * g.TQ);
        const bool two_cols = ox + 1 < g.Q, two_rows = oy + 1 < g.P;
        __half* o0 = Y + (((size_t)n * g.K + (size_t)(kb * KB + kq)) * g.P + oy) * (size_t)g.Q + ox;
#pragma unroll 4
        for (int i = 0; i < 16; ++i) {
          const int run = 4 * i + (lane >> 3);
          const int kk = run >> 1, row = run & 1;
          uint32_t v;
          asm volatile("ld.shared.b32 %0, [%1];"
                       : "=r"(v)
                       : "r"(ebuf + kk * 64 + (((row * 2 + (jj >> 2)) ^ ((kk >> 1) & 3)) << 4) + (jj & 3) * 4));
          if (tvalid && kq + kk < kbs && (row == 0 || two_rows)) {
            __half* o = o0 + (size_t)kk * PQ + (size_t)row * g.Q;
            if (kEpi && R != nullptr) {
              // + residual (same layout as y, read where y is written), then ReLU
              const __half* ro = R + (o - Y);
              const unsigned short* r16 = reinterpret_cast<const unsigned short*>(ro);
              const uint32_t rw = (two_cols && q_even) ? *reinterpret_cast<const uint32_t*>(ro)
                                                       : (uint32_t)r16[0] | (two_cols ? (uint32_t)r16[1] << 16 : 0u);
              float2 f = __half22float2(*reinterpret_cast<const __half2*>(&v));
              const float2 rf = __half22float2(*reinterpret_cast<const __half2*>(&rw));
              f.x += rf.x;
              f.y += rf.y;
              if (va.relu) {
                f.x = fmaxf(f.x, 0.f);
                f.y = fmaxf(f.y, 0.f);
              }
              const __half2 h2 = __floats2half2_rn(f.x, f.y);
              v = *reinterpret_cast<const uint32_t*>(&h2);
            }
            if (two_cols && q_even) {
              *reinterpret_cast<uint32_t*>(o) = v;
            } else {
              reinterpret_cast<unsigned short*>(o)[0] = (unsigned short)(v & 0xffffu);
              if (two_cols) reinterpret_cast<unsigned short*>(o)[1] = (unsigned short)(v >> 16);
            }
          }
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

// Rounds the fp32 sums of split blocks to the fp16 output.
__global__ void y32_to_f16_kernel(const float* __restrict__ y32, __half* __restrict__ y, long long count) {
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < count;
       i += (long long)gridDim.x * blockDim.x)
    y[i] = __float2half_rn(y32[i]);
}

// The drop-in kernel: its only argument is the plugin's parameter struct.
__global__ void __launch_bounds__(NTHREAD, 1) fused_wino_f16_kernel(KernelParam p) {
  const OneLayer one{p, make_geometry(p, TILES), 0};
  fused_body<VAR_F16>(one, VariantArgs{nullptr, nullptr, nullptr});
}

// Precision variants and schedule configurations of one layer.
template <int VAR>
__global__ void __launch_bounds__(NTHREAD, 1) fused_wino_var_kernel(KernelParam p, VariantArgs va, int cfg) {
  const OneLayer one{p, make_geometry(p, TILES), cfg};
  fused_body<VAR>(one, va);
}

template __global__ void fused_wino_var_kernel<VAR_F16>(KernelParam, VariantArgs, int);
template __global__ void fused_wino_var_kernel<VAR_BF16>(KernelParam, VariantArgs, int);
template __global__ void fused_wino_var_kernel<VAR_F8>(KernelParam, VariantArgs, int);
template __global__ void fused_wino_var_kernel<VAR_F16_HILO>(KernelParam, VariantArgs, int);

// A table of fp16 layers in one persistent launch.
__global__ void __launch_bounds__(NTHREAD, 1) fused_wino_batch_kernel(const BatchTable* t, long long total) {
  const LayerTable lt{t, total};
  fused_body<VAR_F16>(lt, VariantArgs{nullptr, nullptr, nullptr});
}

}  // namespace wino

using namespace wino;

extern "C" {

void* wino_fused_kernel_ptr() { return (void*)fused_wino_f16_kernel; }
int wino_fused_smem_bytes() { return fused::SMEM_BYTES; }
int wino_fused_threads() { return fused::NTHREAD; }

int wino_fused_prepare() {
  cudaError_t e = cudaFuncSetAttribute(fused_wino_f16_kernel,
                                       cudaFuncAttributeMaxDynamicSharedMemorySize, fused::SMEM_BYTES);
  return (int)e;
}

static void* var_kernel(int variant);

// Dynamic shared memory limit of a variant's kernel, set once per variant.
int wino_fused_prepare_variant(int variant) {
  static int done[4] = {-1, -1, -1, -1};
  if (variant < 0 || variant > 3) return (int)cudaErrorInvalidValue;
  if (done[variant] < 0)
    done[variant] = (int)cudaFuncSetAttribute(var_kernel(variant), cudaFuncAttributeMaxDynamicSharedMemorySize,
                                              fused::SMEM_BYTES);
  return done[variant];
}

static void* var_kernel(int variant) {
  switch (variant) {
    case VAR_F16: return (void*)fused_wino_var_kernel<VAR_F16>;
    case VAR_BF16: return (void*)fused_wino_var_kernel<VAR_BF16>;
    case VAR_F8: return (void*)fused_wino_var_kernel<VAR_F8>;
    case VAR_F16_HILO: return (void*)fused_wino_var_kernel<VAR_F16_HILO>;
    default: return nullptr;
  }
}

// Launch the fused kernel of a precision variant and schedule configuration
// (CFG_* bits) on `grid` CTAs.
int wino_fused_launch_variant(int variant, const KernelParam* p, const VariantArgs* va, int cfg,
                              unsigned grid, cudaStream_t stream) {
  void* fn = var_kernel(variant);
  if (!fn) return (int)cudaErrorInvalidValue;
  cudaError_t e = (cudaError_t)wino_fused_prepare_variant(variant);
  if (e != cudaSuccess) return (int)e;
  KernelParam pc = *p;
  VariantArgs vc = va ? *va : VariantArgs{nullptr, nullptr, nullptr};
  int cf = cfg;
  void* args[] = {&pc, &vc, &cf};
  e = cudaLaunchKernel(fn, dim3(grid), dim3(fused::NTHREAD), args, (size_t)fused::SMEM_BYTES, stream);
  return (int)e;
}

// The batched persistent launch over a device-resident layer table.
size_t wino_batch_table_bytes() { return sizeof(BatchTable); }
int wino_batch_max_layers() { return BATCH_MAX; }
size_t wino_batch_layer_desc_bytes() { return sizeof(LayerDesc); }

// Dynamic shared memory limits, set outside any stream capture.
int wino_fused_prepare_batch() {
  return (int)cudaFuncSetAttribute(fused_wino_batch_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                   fused::SMEM_BYTES);
}

int wino_fused_launch_batch(const void* table_dev, long long total_blocks, unsigned grid,
                            cudaStream_t stream) {
  static const int prepared = wino_fused_prepare_batch();
  if (prepared != 0) return prepared;
  cudaError_t e;
  const BatchTable* t = static_cast<const BatchTable*>(table_dev);
  long long tot = total_blocks;
  void* args[] = {&t, &tot};
  e = cudaLaunchKernel((void*)fused_wino_batch_kernel, dim3(grid), dim3(fused::NTHREAD), args,
                       (size_t)fused::SMEM_BYTES, stream);
  return (int)e;
}

// Work blocks of a problem (tile blocks x output-channel blocks).
long long wino_fused_nblocks(int n, int h, int w, int k) {
  const long long nt = (long long)n * ((h + 1) / 2) * ((w + 1) / 2);
  return ((nt + fused::TILES - 1) / fused::TILES) * ((k + KB - 1) / KB);
}

// ... and with a schedule configuration (splits multiply the blocks).
long long wino_fused_nblocks_cfg(int n, int c, int h, int w, int k, int cfg) {
  int nsplit, per;
  split_plan(cfg, c / 16, nsplit, per);
  return wino_fused_nblocks(n, h, w, k) * nsplit;
}

int wino_fused_cfg_splits(int c, int cfg) {
  int nsplit, per;
  split_plan(cfg, c / 16, nsplit, per);
  return nsplit;
}

int wino_launch_y32_to_f16(const float* y32, void* y, long long count, cudaStream_t stream) {
  const long long blocks = (count + 255) / 256;
  y32_to_f16_kernel<<<(unsigned)(blocks < (1LL << 20) ? blocks : (1LL << 20)), 256, 0, stream>>>(
      y32, static_cast<__half*>(y), count);
  return (int)cudaGetLastError();
}

uint32_t wino_fused_error_read_clear() {
  uint32_t v = 0, z = 0;
  cudaMemcpyFromSymbol(&v, g_fused_err, sizeof(v));
  cudaMemcpyToSymbol(g_fused_err, &z, sizeof(z));
  return v;
}

}  // extern "C"
