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
// Pipelines (shared memory, 216 KB): U in three 32 KB slots, each half of a
// step's piece (8 taps x 128 k x 16 c); V in three 16 KB slots, one per
// step; three 24 KB input slabs.  Barrier hand-offs cost a few hundred
// cycles on this part, so each side keeps several slots in flight.
//
// Warp roles (14 warps):
//   warp 0       TMEM allocation; one thread issues the MMAs
//   warp 1       one thread bulk-copies the U half-pieces
//   warps 2-5    V producers, all four on every step: copy the input band
//                of the step's block into a shared-memory slab two steps
//                ahead (cp.async), then B^T d B in packed fp16 from the slab
//                straight into the K-major operand (8 tiles x 8 channels per
//                core matrix); warp q forms channels 4q..4q+3, lane = tile
//   warps 6-13   epilogue: drain TMEM tap by tap (each drained tap is handed
//                back to the MMA thread at once, so the next block's MMAs
//                overlap the drain), A^T m A in fp32, fp16 NKPQ stores.
#include <cuda_runtime.h>
#include "tc_sm100.cuh"
#include "wino_common.cuh"
#include "vgen.cuh"

namespace wino {

static __device__ uint32_t g_fused_err;

namespace fused {

constexpr int TILES = 32;              // MMA N: tiles per block
constexpr int NTAP = 16;
constexpr int V_TAP_BYTES = TILES * 16 * 2;          // 1 KB per tap per step
constexpr int V_SLOT_BYTES = NTAP * V_TAP_BYTES;     // 16 KB: one step of V
constexpr int U_SLOT_BYTES = 8 * KB * 16 * 2;        // 32 KB: 8 taps of a step of U
constexpr int NVSLOT = 3, NUSLOT = 3, NSLAB = 3;
constexpr int U_BASE = 0, V_BASE = NUSLOT * U_SLOT_BYTES;
constexpr int SLAB_BASE = V_BASE + NVSLOT * V_SLOT_BYTES;
constexpr int NWARP = 14;
constexpr int NTHREAD = NWARP * 32;
constexpr int WARP_MMA = 0, WARP_U = 1, WARP_V0 = 2, NWARP_V = 4, WARP_E0 = 6, NWARP_E = 8;
constexpr int NPROD = NWARP_V * 32;   // producer threads
constexpr int SMEM_BYTES = NUSLOT * U_SLOT_BYTES + NVSLOT * V_SLOT_BYTES + NSLAB * SLAB_BYTES + 1024;

struct Shared {
  uint64_t ufull[NUSLOT], uempty[NUSLOT];
  uint64_t vfull[NVSLOT], vempty[NVSLOT];
  uint64_t slabfull[NSLAB], slabfree[NSLAB];
  uint64_t accf;
  uint64_t tapfree[NTAP];
  uint32_t tmem_base;
  int abort_flag;
};

// Output-transform coefficient of tap t = 4a+b for output (i, j):
// At[i][a] * At[j][b] with At = [[1,1,1,0],[0,1,-1,-1]].
__host__ __device__ constexpr int at_coef(int i, int a) {
  return i == 0 ? (a == 3 ? 0 : 1) : (a == 0 ? 0 : (a == 1 ? 1 : -1));
}

}  // namespace fused

using namespace fused;

__global__ void __launch_bounds__(NTHREAD, 1) fused_wino_f16_kernel(KernelParam p) {
  extern __shared__ __align__(1024) uint8_t smem_raw[];
  __shared__ Shared sh;
  uint8_t* smem = reinterpret_cast<uint8_t*>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
  const Geometry g = make_geometry(p, TILES);
  const int nKB = (g.K + KB - 1) / KB;
  const long long nblocks = (long long)g.nTB * nKB;
  const int warp = warp_id();
  const int lane = lane_id();
  uint32_t* err = &g_fused_err;

  if (threadIdx.x == 0) {
    for (int s = 0; s < NUSLOT; ++s) {
      mbar_init(&sh.ufull[s], 1);
      mbar_init(&sh.uempty[s], 1);
    }
    for (int s = 0; s < NVSLOT; ++s) {
      mbar_init(&sh.vfull[s], NWARP_V);  // every producer warp
      mbar_init(&sh.vempty[s], 1);
    }
    for (int s = 0; s < NSLAB; ++s) {
      mbar_init(&sh.slabfull[s], NPROD);   // each producer thread's copies
      mbar_init(&sh.slabfree[s], NWARP_V);
    }
    mbar_init(&sh.accf, 1);
    for (int t = 0; t < NTAP; ++t) mbar_init(&sh.tapfree[t], NWARP_E);
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
  auto u_slot = [&](uint32_t s) { return smem_base + U_BASE + s * U_SLOT_BYTES; };
  auto v_slot = [&](uint32_t s) { return smem_base + V_BASE + s * V_SLOT_BYTES; };

  if (warp == WARP_MMA) {
    if (lane == 0) {
      const uint32_t idesc = instr_desc(128, TILES, 0, 0, /*a_mn=*/0, /*b_mn=*/0);
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
        const int kb = (int)(b % nKB);
        const uint32_t astep = (uint32_t)(kblock_rows(kb, g.K) * 32) >> 4;
        for (int s = 0; s < g.CS && ok; ++s, ++it) {
          const uint32_t vs = it % NVSLOT;
          ok = mbar_wait(&sh.vfull[vs], (it / NVSLOT) & 1, abort_flag, err, ERR_WAIT_FULL);
          const uint32_t acc = s > 0 ? 1u : 0u;
          const bool first_step = s == 0 && bi > 0;
#pragma unroll
          for (int h = 0; h < 2; ++h) {
            if (!ok) break;
            const uint32_t ui = 2 * it + h, us = ui % NUSLOT;
            ok = mbar_wait(&sh.ufull[us], (ui / NUSLOT) & 1, abort_flag, err, ERR_WAIT_FULL);
            if (!ok) break;
            const uint64_t ad = adesc0 + ((us * U_SLOT_BYTES) >> 4);
            const uint64_t bd = bdesc0 + ((vs * V_SLOT_BYTES + 8 * h * V_TAP_BYTES) >> 4);
            const uint32_t d = tmem + 8 * h * TILES;
            if (first_step) {
              // the previous block's epilogue hands each tap's columns back in turn
#pragma unroll
              for (int tt = 0; tt < 8; ++tt) {
                if (!mbar_wait(&sh.tapfree[8 * h + tt], (bi - 1) & 1, abort_flag, err, ERR_WAIT_DRAIN)) {
                  ok = false;
                  break;
                }
                tc_fence_after();
                mma_f16(d + tt * TILES, ad + tt * astep, bd + tt * BSTEP, idesc, acc);
              }
            } else {
#pragma unroll
              for (int tt = 0; tt < 8; ++tt)
                mma_f16(d + tt * TILES, ad + tt * astep, bd + tt * BSTEP, idesc, acc);
            }
            mma_commit(&sh.uempty[us]);
          }
          mma_commit(&sh.vempty[vs]);
        }
        if (ok) mma_commit(&sh.accf);
      }
    }
    __syncwarp();
  } else if (warp == WARP_U) {
    if (lane == 0) {
      const uint8_t* ucache = static_cast<const uint8_t*>(p.transform_filter);
      uint32_t ui = 0;
      bool ok = true;
      for (long long b = blockIdx.x; b < nblocks && ok; b += gridDim.x) {
        const int kb = (int)(b % nKB);
        const int kbs = kblock_rows(kb, g.K);
        const uint32_t bytes = 8 * kbs * 16 * 2;
        for (int s = 0; s < g.CS && ok; ++s) {
          for (int h = 0; h < 2; ++h, ++ui) {
            const uint32_t us = ui % NUSLOT;
            if (ui >= NUSLOT &&
                !mbar_wait(&sh.uempty[us], (ui / NUSLOT - 1) & 1, abort_flag, err, ERR_WAIT_EMPTY)) {
              ok = false;
              break;
            }
            mbar_arrive_expect_tx(&sh.ufull[us], bytes);
            bulk_g2s(smem + U_BASE + us * U_SLOT_BYTES,
                     ucache + u_piece(kb, s, g.K, g.C) * 2 + (size_t)h * bytes, bytes, &sh.ufull[us]);
          }
        }
      }
      if (*abort_flag) __nanosleep(20000);  // let copies already issued land
    }
    __syncwarp();
  } else if (warp >= WARP_V0 && warp < WARP_V0 + NWARP_V) {
    // The four producer warps work on every step together.  Two steps ahead
    // they copy the input band of the step's block into a slab (cp.async,
    // completion counted on slabfull); then warp q forms channels 4q..4q+3
    // of the step's V for all 32 tiles (lane = tile) from the slab.
    const int q = warp - WARP_V0;
    const int ptid = threadIdx.x - WARP_V0 * 32;
    const __half* X = static_cast<const __half*>(p.pin);
    const int my_blocks =
        blockIdx.x < nblocks ? (int)((nblocks - blockIdx.x + gridDim.x - 1) / gridDim.x) : 0;
    const int CS = g.CS;
    const uint32_t slab0 = smem_base + SLAB_BASE;
    // Per-block quantities are formed once per block (32-bit math); the
    // staging side runs two steps ahead, possibly into the next block.
    auto block_tile0 = [&](int bi) { return (int)((blockIdx.x + (long long)bi * gridDim.x) / nKB) * TILES; };
    bool ok = true;
    int st_bi = 0, st_s = 0;                      // next step to stage
    SlabPlan st_pl = slab_plan(g, block_tile0(0), TILES);
    uint32_t st_it = 0;
    auto stage_next = [&]() {
      const uint32_t j = st_it % NSLAB;
      if (st_it >= NSLAB &&
          !mbar_wait_warp(&sh.slabfree[j], ((st_it - NSLAB) / NSLAB) & 1, abort_flag, err, ERR_WAIT_EMPTY, 32)) {
        ok = false;
        return;
      }
      if (slab_fits(g, st_pl)) slab_stage(X, g, st_pl, st_s * 16, slab0 + j * SLAB_BYTES, ptid, NPROD);
      cp_async_arrive(&sh.slabfull[j]);
      ++st_it;
      if (++st_s == CS) {
        st_s = 0;
        if (++st_bi < my_blocks) st_pl = slab_plan(g, block_tile0(st_bi), TILES);
      }
    };
    const uint32_t total = (uint32_t)my_blocks * CS;
    if (total > 0) stage_next();
    if (total > 1) stage_next();
    // K-major core matrices: tile group (lane/8) at 256 B, channel half at
    // 128 B, tile row (lane%8) at 16 B, channel quarter inside the row at 8 B.
    const uint32_t row_off = (lane >> 3) * 256 + (q >> 1) * 128 + (lane & 7) * 16 + (q & 1) * 8;
    uint32_t it = 0;
    for (int bi = 0; bi < my_blocks && ok; ++bi) {
      const int tile0 = block_tile0(bi);
      const SlabPlan pl = slab_plan(g, tile0, TILES);
      const bool use_slab = slab_fits(g, pl);
      const TileCoord tc = tile_coord(g, tile0 + lane);
      for (int s = 0; s < CS && ok; ++s, ++it) {
        if (it + 2 < total) stage_next();
        if (!ok) break;
        const uint32_t j = it % NSLAB;
        const uint32_t vs = it % NVSLOT;
        if (!mbar_wait_warp(&sh.slabfull[j], (it / NSLAB) & 1, abort_flag, err, ERR_WAIT_FULL, 32)) {
          ok = false;
          break;
        }
        if (it >= NVSLOT &&
            !mbar_wait_warp(&sh.vempty[vs], (it / NVSLOT - 1) & 1, abort_flag, err, ERR_WAIT_EMPTY, 32)) {
          ok = false;
          break;
        }
        const uint32_t dst = v_slot(vs) + row_off;
        auto sink = [&](int t, uint32_t w0, uint32_t w1) {
          asm volatile("st.shared.v2.b32 [%0], {%1, %2};" ::"r"(dst + t * V_TAP_BYTES), "r"(w0), "r"(w1)
                       : "memory");
        };
        if (use_slab)
          produce_v_quarter_slab(g, pl, slab0 + j * SLAB_BYTES, tc, 4 * q, sink);
        else
          produce_v_quarter_global(X, g, tc, s * 16 + 4 * q, sink);
        fence_proxy_async_shared();
        __syncwarp();
        if (lane == 0) {
          mbar_arrive(&sh.slabfree[j]);
          mbar_arrive(&sh.vfull[vs]);
        }
      }
    }
  } else if (warp >= WARP_E0) {
    const int quarter = warp & 3;            // TMEM lanes 32*quarter .. +31 = channels
    const int half = (warp - WARP_E0) >> 2;  // tiles 16*half .. +15 of the block
    __half* Y = static_cast<__half*>(p.pout);
    const long long per_img = (long long)g.TP * g.TQ;
    const bool q_even = (g.Q & 1) == 0;
    uint32_t bi = 0;
    for (long long b = blockIdx.x; b < nblocks; b += gridDim.x, ++bi) {
      if (!mbar_wait_warp(&sh.accf, bi & 1, abort_flag, err, ERR_WAIT_ACCUM, 128)) break;
      tc_fence_after();
      const long long tb = b / nKB;
      const int kb = (int)(b % nKB);
      const int kbs = kblock_rows(kb, g.K);
      float y[16][4];
#pragma unroll
      for (int j = 0; j < 16; ++j)
#pragma unroll
        for (int o = 0; o < 4; ++o) y[j][o] = 0.f;
      const uint32_t tbase = tmem + ((uint32_t)(quarter * 32) << 16) + half * 16;
#pragma unroll
      for (int t = 0; t < NTAP; ++t) {
        float m[16];
        tmem_ld16(tbase + t * TILES, m);
        tmem_ld_wait();
        tc_fence_before();
        __syncwarp();
        if (lane == 0) mbar_arrive(&sh.tapfree[t]);
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
      const int k = kb * KB + quarter * 32 + lane;
      if (quarter * 32 + lane < kbs) {
        long long tile = tb * TILES + half * 16;
        int n = (int)(tile / per_img);
        int r = (int)(tile - (long long)n * per_img);
        int ty = r / g.TQ, tx = r - ty * g.TQ;
#pragma unroll
        for (int j = 0; j < 16; ++j, ++tile) {
          if (tile < g.NT) {
            const int oy = 2 * ty, ox = 2 * tx;
            const bool two_cols = ox + 1 < g.Q, two_rows = oy + 1 < g.P;
            __half* o = Y + (((size_t)n * g.K + k) * g.P + oy) * (size_t)g.Q + ox;
            if (two_cols && q_even) {
              *reinterpret_cast<__half2*>(o) = __floats2half2_rn(y[j][0], y[j][1]);
              if (two_rows) *reinterpret_cast<__half2*>(o + g.Q) = __floats2half2_rn(y[j][2], y[j][3]);
            } else {
              o[0] = __float2half_rn(y[j][0]);
              if (two_cols) o[1] = __float2half_rn(y[j][1]);
              if (two_rows) {
                o[g.Q] = __float2half_rn(y[j][2]);
                if (two_cols) o[g.Q + 1] = __float2half_rn(y[j][3]);
              }
            }
          }
          if (++tx == g.TQ) {  // advance to the next tile
            tx = 0;
            if (++ty == g.TP) { ty = 0; ++n; }
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

// Work blocks of a problem (tile blocks x output-channel blocks).
long long wino_fused_nblocks(int n, int h, int w, int k) {
  const long long nt = (long long)n * ((h + 1) / 2) * ((w + 1) / 2);
  return ((nt + fused::TILES - 1) / fused::TILES) * ((k + KB - 1) / KB);
}

uint32_t wino_fused_error_read_clear() {
  uint32_t v = 0, z = 0;
  cudaMemcpyFromSymbol(&v, g_fused_err, sizeof(v));
  cudaMemcpyToSymbol(g_fused_err, &z, sizeof(z));
  return v;
}

}  // extern "C"
