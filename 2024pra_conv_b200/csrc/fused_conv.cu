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
// Pipelines (shared memory, 225 KB): U in four 32 KB half-step slots (two
// steps in flight); V in three 16 KB slots, one per step; two 16 KB input
// slabs; 16 KB of epilogue store staging.  The MMA thread commits once per step (each tcgen05.commit stalls
// the MMA pipe for ~90 cycles on this part) to a "step done" barrier that
// releases that step's U half-slots and V slot together.
//
// Warp roles (15 warps):
//   warp 0       TMEM allocation; one thread issues the MMAs
//   warp 1       lanes 0 and 1 bulk-copy the two U halves of a step (one
//                copy in flight per issuing thread, so two threads)
//   warps 2-5    V producers, all four on every step: warp q forms channel
//                half q&1 (8 channels) of tap rows 2(q>>1), 2(q>>1)+1 (8
//                taps) of the step's V for all 32 tiles (lane = tile):
//                B^T d B in packed fp16 straight into the K-major operand
//                (8 tiles x 8 channels per core matrix, one 16-byte row per
//                lane and tap).  They read the step's slab, or, without an
//                XB workspace or when a block's rows exceed a slab, the NCHW
//                input directly.
//   warps 6-13   epilogue: drain TMEM one tap half at a time (the block's
//                last MMAs commit each half separately, and each drained half
//                goes back to the MMA thread at once, so the drain overlaps
//                the MMAs on both sides), A^T m A in fp32, fp16 NKPQ stores.
//   warp 14      stager: with an XB workspace (p.transform_pin, written by
//                the pre-pass of input_layout.cu) bulk-copies each step's
//                input rows into a slab, up to two steps ahead (one copy
//                per image the block touches, issued from separate lanes).
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
constexpr int U_HALF_BYTES = 8 * KB * 16 * 2;        // 32 KB: 8 taps of a step of U
constexpr int NUH = 4;                 // U half-slots: two steps
constexpr int NVSLOT = 3, NSD = 3, NSLAB = 2;
constexpr int EPI_WARP_BYTES = 2048;   // epilogue store staging per warp
constexpr int U_BASE = 0, V_BASE = NUH * U_HALF_BYTES;
constexpr int SLAB_BASE = V_BASE + NVSLOT * V_SLOT_BYTES;
constexpr int EPI_BASE = SLAB_BASE + NSLAB * SLAB_BYTES;
constexpr int NWARP = 15;
constexpr int NTHREAD = NWARP * 32;
constexpr int WARP_MMA = 0, WARP_U = 1, WARP_V0 = 2, NWARP_V = 4, WARP_E0 = 6, NWARP_E = 8;
constexpr int WARP_S = 14;
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
  //   U half-slots 2 * (it % 2) + h, reused at it + 2 (after sdone of it);
  //   slab it % NSLAB, reused at it + NSLAB (after the producers' slabfree).
  // A waiter on sdone[j] for step it cannot miss its phase: the barrier's
  // next phase needs operands the waiter has not supplied yet.

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
            const uint32_t us = 2 * (it & 1) + h;
            ok = mbar_wait(&sh.ufull[us], (it >> 1) & 1, abort_flag, err, ERR_WAIT_FULL);
            if (!ok) break;
            const uint64_t ad = adesc0 + ((us * U_HALF_BYTES) >> 4);
            const uint64_t bd = bdesc0 + ((vs * V_SLOT_BYTES + 8 * h * V_TAP_BYTES) >> 4);
            const uint32_t d = tmem + 8 * h * TILES;
            if (first_step) {
              // the previous block's epilogue hands back each tap half of TMEM
              if (!mbar_wait(&sh.tapfree[h], (bi - 1) & 1, abort_flag, err, ERR_WAIT_DRAIN)) {
                ok = false;
                break;
              }
              tc_fence_after();
            }
#pragma unroll
            for (int tt = 0; tt < 8; ++tt)
              mma_f16(d + tt * TILES, ad + tt * astep, bd + tt * BSTEP, idesc, acc);
            // after the block's last MMAs of a tap half the epilogue may drain it
            if (s == g.CS - 1) mma_commit(&sh.accf[h]);
          }
          if (ok) mma_commit(&sh.sdone[it % NSD]);
        }
      }
    }
    __syncwarp();
  } else if (warp == WARP_U) {
    if (lane < 2) {
      const int h = lane;
      const uint8_t* ucache = static_cast<const uint8_t*>(p.transform_filter);
      uint32_t it = 0;
      bool ok = true;
      for (long long b = blockIdx.x; b < nblocks && ok; b += gridDim.x) {
        const int kb = (int)(b % nKB);
        const int kbs = kblock_rows(kb, g.K);
        const uint32_t bytes = 8 * kbs * 16 * 2;
        for (int s = 0; s < g.CS; ++s, ++it) {
          if (it >= 2 &&
              !mbar_wait(&sh.sdone[(it - 2) % NSD], ((it - 2) / NSD) & 1, abort_flag, err, ERR_WAIT_EMPTY)) {
            ok = false;
            break;
          }
          const uint32_t us = 2 * (it & 1) + h;
          mbar_arrive_expect_tx(&sh.ufull[us], bytes);
          bulk_g2s(smem + U_BASE + us * U_HALF_BYTES,
                   ucache + u_piece(kb, s, g.K, g.C) * 2 + (size_t)h * bytes, bytes, &sh.ufull[us]);
        }
      }
      if (*abort_flag) __nanosleep(20000);  // let copies already issued land
    }
    __syncwarp();
  } else if (warp == WARP_S) {
    const uint8_t* XB = static_cast<const uint8_t*>(p.transform_pin);
    const int my_blocks =
        blockIdx.x < nblocks ? (int)((nblocks - blockIdx.x + gridDim.x - 1) / gridDim.x) : 0;
    const uint32_t RB = (uint32_t)xb_row_bytes(g.W);
    const size_t img_stride = (size_t)(g.C >> 4) * xb_rows(g.H) * RB;   // one image of XB
    const size_t cb_stride = (size_t)xb_rows(g.H) * RB;                  // one channel block
    uint32_t it = 0;
    bool ok = true;
    for (int bi = 0; bi < my_blocks && ok; ++bi) {
      const int tile0 = (int)((blockIdx.x + (long long)bi * gridDim.x) / nKB) * TILES;
      const SlabPlan pl = slab_plan(g, tile0, TILES);
      const bool use = XB != nullptr && slab_fits(g, pl);
      int ta = 0, rows = 0, rbase = 0;  // this lane's segment
#pragma unroll
      for (int k = 0; k < SLAB_MAXSEG; ++k)
        if (lane == k) { ta = pl.ta[k]; rows = pl.rows[k]; rbase = pl.row_base[k]; }
      const uint8_t* src0 = XB + (size_t)(pl.n0 + lane) * img_stride + (size_t)(2 * ta) * RB;
      for (int s = 0; s < g.CS; ++s, ++it) {
        const uint32_t j = it % NSLAB;
        if (it >= NSLAB &&
            !mbar_wait_warp(&sh.slabfree[j], ((it - NSLAB) / NSLAB) & 1, abort_flag, err, ERR_WAIT_EMPTY, 64)) {
          ok = false;
          break;
        }
        if (use) {
          if (lane == 0) mbar_arrive_expect_tx(&sh.slabfull[j], (uint32_t)pl.total_rows * RB);
          __syncwarp();
          if (lane < pl.nseg)
            bulk_g2s(smem + SLAB_BASE + j * SLAB_BYTES + (uint32_t)rbase * RB, src0 + (size_t)s * cb_stride,
                     (uint32_t)rows * RB, &sh.slabfull[j]);
        } else if (lane == 0) {
          mbar_arrive(&sh.slabfull[j]);
        }
      }
    }
    if (*abort_flag) __nanosleep(20000);  // let copies already issued land
    __syncwarp();
  } else if (warp >= WARP_V0 && warp < WARP_V0 + NWARP_V) {
    const int q = warp - WARP_V0;
    const int hh = q & 1;                     // channel half: channels 8hh .. 8hh+7
    const int ar = q >> 1;                    // tap rows 2ar, 2ar+1 (taps 8ar .. 8ar+7)
    const __half* X = static_cast<const __half*>(p.pin);
    const bool have_xb = p.transform_pin != nullptr;
    const int my_blocks =
        blockIdx.x < nblocks ? (int)((nblocks - blockIdx.x + gridDim.x - 1) / gridDim.x) : 0;
    const int CS = g.CS;
    const uint32_t slab0 = smem_base + SLAB_BASE;
    bool ok = true;
    // K-major core matrices: tile group (lane/8) at 256 B, channel half at
    // 128 B, tile row (lane%8) at 16 B: each lane writes whole 16-byte rows,
    // eight lanes 128 contiguous bytes (conflict-free).
    const uint32_t row_off = (lane >> 3) * 256 + hh * 128 + (lane & 7) * 16 + ar * 8 * V_TAP_BYTES;
    uint32_t it = 0;
    for (int bi = 0; bi < my_blocks && ok; ++bi) {
      // per-block quantities once per block, 32-bit
      const int tile0 = (int)((blockIdx.x + (long long)bi * gridDim.x) / nKB) * TILES;
      const SlabPlan pl = slab_plan(g, tile0, TILES);
      const bool use_slab = have_xb && slab_fits(g, pl);
      const TileCoord tc = tile_coord(g, tile0 + lane, tile0);
      const SlabWindow sw = slab_window(g, pl, tc, hh);
      for (int s = 0; s < CS && ok; ++s, ++it) {
        const uint32_t j = it % NSLAB;
        const uint32_t vs = it % NVSLOT;
        if (!mbar_wait_warp(&sh.slabfull[j], (it / NSLAB) & 1, abort_flag, err, ERR_WAIT_FULL, 32)) {
          ok = false;
          break;
        }
        if (it >= NVSLOT &&
            !mbar_wait_warp(&sh.sdone[(it - NVSLOT) % NSD], ((it - NVSLOT) / NSD) & 1, abort_flag, err,
                            ERR_WAIT_EMPTY, 32)) {
          ok = false;
          break;
        }
        const uint32_t dst = v_slot(vs) + row_off;
        if (use_slab) {
          auto sink = [&](int u, const uint32_t (&w)[4]) {
            st_shared_v4(dst + u * V_TAP_BYTES, w[0], w[1], w[2], w[3]);
          };
          if (ar == 0)
            produce_v_half_xb<0>(slab0 + j * SLAB_BYTES, sw, sink);
          else
            produce_v_half_xb<1>(slab0 + j * SLAB_BYTES, sw, sink);
        } else {
          // direct NCHW reads: two channel quarters, keeping this warp's taps
#pragma unroll 1
          for (int qq = 0; qq < 2; ++qq) {
            auto sink = [&](int t, uint32_t w0, uint32_t w1) {
              if ((t >> 3) == ar)
                asm volatile("st.shared.v2.b32 [%0], {%1, %2};" ::"r"(dst + (t & 7) * V_TAP_BYTES + qq * 8),
                             "r"(w0), "r"(w1)
                             : "memory");
            };
            produce_v_quarter_global(X, g, tc, s * 16 + 8 * hh + 4 * qq, sink);
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
    __half* Y = static_cast<__half*>(p.pout);
    const bool q_even = (g.Q & 1) == 0;
    uint32_t bi = 0;
    bool ok = true;
    for (long long b = blockIdx.x; b < nblocks && ok; b += gridDim.x, ++bi) {
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
        if ((t & 7) == 0) {
          if (!mbar_wait_warp(&sh.accf[t >> 3], bi & 1, abort_flag, err, ERR_WAIT_ACCUM, 64)) {
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
      // Stores go through a 2 KB per-warp staging buffer, 8 tiles at a time:
      // thread k writes its outputs as [k][row][8 tiles] half2 (16-byte
      // chunks XOR-swizzled by k so the writes are conflict-free), then each
      // store instruction writes 4 runs of 8 consecutive tiles (32 B of one
      // output row of one channel) instead of 32 scattered words.
      const uint32_t ebuf = smem_base + EPI_BASE + (uint32_t)(warp - WARP_E0) * EPI_WARP_BYTES;
      const int kq = quarter * 32;             // first channel of this warp in the k-block
      const size_t PQ = (size_t)g.P * g.Q;
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
