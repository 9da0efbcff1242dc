// The plain unfused Winograd path: the comparator the fused kernel is
// measured against.  Same structure as the reference's pipeline (filter
// transform, input transform, 16 tap GEMMs, output transform, with V and M
// stored to global memory in fp16 between stages; reference
// src/preprocessing.cuh:273-424, src/matrixmul.cuh:139-556,
// src/conv2d.cpp:17-250), but every stage is an sm_100a kernel of its own:
//
//   unfused_input_transform   X (NCHW) -> V2 (tile-major, fp16)
//   unfused_gemm              16 x [tiles x C] * [C x K]^T on tcgen05 with
//                             128 x 256 output tiles (two 128 x 128 MMAs per
//                             K-step sharing the tile operand), double-
//                             buffered TMEM, fp32 accumulate
//                             -> M16[t][k][tile] fp16
//   unfused_output_transform  M16 -> Y (N K P Q), A^T m A in fp32
//
// The GEMM uses the same tcgen05 layer (tc_sm100.cuh) and the same operand
// layouts as the fused kernel, so the two differ by the fusion, not by a
// weaker GEMM.
#include <cuda_runtime.h>
#include "tc_sm100.cuh"
#include "wino_common.cuh"
#include "vgen.cuh"

namespace wino {

static __device__ uint32_t g_unfused_err;

namespace unfused {

constexpr int NSTAGE = 4;
constexpr int SK = 4;                         // K-steps (16 channels each) per stage
constexpr int KPU = 2;                        // 128-row k-blocks per work unit (share A)
constexpr int A_STEP = TB2 * 16 * 2;          // 4 KB: one K-step of a 128-tile block
constexpr int B_STEP_MAX = KB2 * 16 * 2;      // 4 KB: one K-step of a 128-row k-block
constexpr int STAGE_A = SK * A_STEP;
constexpr int STAGE_B = SK * B_STEP_MAX;      // one k-block's operand of a stage
constexpr int STAGE_BYTES = STAGE_A + KPU * STAGE_B;
constexpr int SMEM_BYTES = NSTAGE * STAGE_BYTES + 1024;
constexpr int NTHREAD = 6 * 32;               // producer, MMA, 4 epilogue warps

struct Shared {
  uint64_t full[NSTAGE], empty[NSTAGE];
  uint64_t accfull[2], accempty[2];
  uint32_t tmem_base;
  int abort_flag;
};

}  // namespace unfused

// ------------------------------------------------------- input transform ---
// grid (tile blocks, K-steps), 256 threads: thread = (8-tile group, channel).
__global__ void __launch_bounds__(256) unfused_input_transform(KernelParam p) {
  const Geometry g = make_geometry(p, TB2);
  const int tb = blockIdx.x, cs = blockIdx.y;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int grp = 2 * warp + (lane >> 4), cl = lane & 15;
  uint8_t* v2 = static_cast<uint8_t*>(p.transform_pin);
  const long long tile0 = (long long)tb * TB2 + grp * 8;
  const size_t inner = grp * 256 + (cl >> 3) * 128 + (cl & 7) * 16;
  produce_v8(static_cast<const __half*>(p.pin), g, tile0, cs * 16 + cl, -1,
             [&](int t, uint32_t a, uint32_t b, uint32_t c, uint32_t d) {
               uint8_t* dst = v2 + v2_piece(t, tb, cs, g.nTB, g.CS) * 2 + inner;
               *reinterpret_cast<uint4*>(dst) = make_uint4(a, b, c, d);
             });
}

// ------------------------------------------------------------- tap GEMMs ---
using namespace unfused;

// One batched tap GEMM: for every tap t, M[t][k][tile] = sum_c V2[t][tile][c]
// * U2[t][k][c] over `c_red` reduction channels, M stored as fp16 (M32 false)
// or fp32 (M32 true).  The F(2x2) comparator runs it with 16 taps and c_red =
// C; the F(4x4,3x3) path with 36 taps and c_red = C or 3C (hi+lo pieces).
// A work unit is (tap, 128-tile block, pair of 128-row k-blocks): each K-step
// issues two M=128 N<=128 MMAs that share the V operand, into two 128-column
// TMEM accumulators; units are double-buffered in TMEM (512 columns).
template <bool M32>
__device__ __forceinline__ void tap_gemm_body(const TapGemm& tg) {
  extern __shared__ __align__(1024) uint8_t smem_raw[];
  __shared__ unfused::Shared sh;
  uint8_t* smem = reinterpret_cast<uint8_t*>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
  struct { int nTB, CS, K, C; } g;
  g.nTB = tg.ntb; g.CS = tg.c_red >> 4; g.K = tg.k; g.C = tg.c_red;
  const int nKB2 = (g.K + KB2 - 1) / KB2;
  const int nKP = (nKB2 + KPU - 1) / KPU;
  const long long nunits = (long long)tg.taps * g.nTB * nKP;
  const int nst = (g.CS + SK - 1) / SK;  // stages per unit
  const int warp = warp_id(), lane = lane_id();
  uint32_t* err = &g_unfused_err;

  if (threadIdx.x == 0) {
    for (int s = 0; s < NSTAGE; ++s) { mbar_init(&sh.full[s], 1); mbar_init(&sh.empty[s], 1); }
    for (int a = 0; a < 2; ++a) { mbar_init(&sh.accfull[a], 1); mbar_init(&sh.accempty[a], 4); }
    sh.abort_flag = 0;
    fence_barrier_init();
  }
  if (warp == 1) { tmem_alloc(&sh.tmem_base, 512); tmem_relinquish(); }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = sh.tmem_base;
  volatile int* abort_flag = &sh.abort_flag;
  const uint32_t sbase = smem_u32(smem);

  // kb = first k-block of the unit; kbs[i] = rows of its i-th k-block (0: absent)
  auto unit_coords = [&](long long u, int& t, int& tb, int& kb, int (&kbs)[KPU]) {
    const int kp = (int)(u % nKP);
    tb = (int)((u / nKP) % g.nTB);
    t = (int)(u / ((long long)nKP * g.nTB));
    kb = kp * KPU;
#pragma unroll
    for (int i = 0; i < KPU; ++i) kbs[i] = kb + i < nKB2 ? kblock2_rows(kb + i, g.K) : 0;
  };

  if (warp == 0) {
    if (lane == 0) {
      const uint8_t* v2 = static_cast<const uint8_t*>(tg.v2);
      const uint8_t* u2 = static_cast<const uint8_t*>(tg.u2);
      uint32_t it = 0;
      for (long long u = blockIdx.x; u < nunits && !*abort_flag; u += gridDim.x) {
        int t, tb, kb, kbs[KPU];
        unit_coords(u, t, tb, kb, kbs);
        for (int j = 0; j < nst; ++j, ++it) {
          const int st = it % NSTAGE;
          if (it >= NSTAGE &&
              !mbar_wait(&sh.empty[st], (it / NSTAGE - 1) & 1, abort_flag, err, ERR_WAIT_EMPTY))
            break;
          const int nk = min(SK, g.CS - j * SK);
          const uint32_t abytes = nk * A_STEP;
          uint32_t tx = abytes;
#pragma unroll
          for (int i = 0; i < KPU; ++i) tx += nk * kbs[i] * 32;
          mbar_arrive_expect_tx(&sh.full[st], tx);
          bulk_g2s(smem + st * STAGE_BYTES, v2 + v2_piece(t, tb, j * SK, g.nTB, g.CS) * 2, abytes,
                   &sh.full[st]);
#pragma unroll
          for (int i = 0; i < KPU; ++i)
            if (kbs[i])
              bulk_g2s(smem + st * STAGE_BYTES + STAGE_A + i * STAGE_B,
                       u2 + u2_piece(t, kb + i, j * SK, g.K, g.C) * 2, nk * kbs[i] * 32, &sh.full[st]);
        }
      }
      if (*abort_flag) __nanosleep(20000);
    }
    __syncwarp();
  } else if (warp == 1) {
    if (lane == 0) {
      uint32_t it = 0, ui = 0;
      for (long long u = blockIdx.x; u < nunits && !*abort_flag; u += gridDim.x, ++ui) {
        int t, tb, kb, kbs[KPU];
        unit_coords(u, t, tb, kb, kbs);
        uint32_t idesc[KPU];
#pragma unroll
        for (int i = 0; i < KPU; ++i) idesc[i] = instr_desc(128, kbs[i] ? kbs[i] : 16, 0, 0, 1, 0);
        const int ab = ui & 1;
        if (ui >= 2 && !mbar_wait(&sh.accempty[ab], ((ui >> 1) - 1) & 1, abort_flag, err, ERR_WAIT_DRAIN))
          break;
        tc_fence_after();
        const uint32_t d = tmem + ab * (KPU * 128);
        for (int j = 0; j < nst; ++j, ++it) {
          const int st = it % NSTAGE;
          if (!mbar_wait(&sh.full[st], (it / NSTAGE) & 1, abort_flag, err, ERR_WAIT_FULL)) break;
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
        mma_commit(&sh.accfull[ab]);
      }
    }
    __syncwarp();
  } else {
    const int quarter = warp & 3;
    const size_t ntp = (size_t)g.nTB * TB2;
    uint32_t ui = 0;
    for (long long u = blockIdx.x; u < nunits; u += gridDim.x, ++ui) {
      int t, tb, kb, kbs[KPU];
      unit_coords(u, t, tb, kb, kbs);
      const int ab = ui & 1;
      if (!mbar_wait(&sh.accfull[ab], (ui >> 1) & 1, abort_flag, err, ERR_WAIT_ACCUM)) break;
      tc_fence_after();
      const size_t tile = (size_t)tb * TB2 + quarter * 32 + lane;
      const uint32_t taddr = tmem + ((uint32_t)(quarter * 32) << 16) + ab * (KPU * 128);
      // columns i * 128 + c of the unit's accumulators = output channel (kb + i) * 128 + c
      for (int cc = 0; cc < KPU * 128; cc += 16) {
        const int i = cc >> 7, c0 = cc & 127;
        if (c0 >= kbs[i]) continue;
        float v[16];
        tmem_ld16(taddr + cc, v);
        tmem_ld_wait();
        const size_t row = ((size_t)t * g.K + (size_t)(kb + i) * KB2 + c0) * ntp + tile;
        if constexpr (M32) {
          float* dst = static_cast<float*>(tg.m) + row;
#pragma unroll
          for (int j = 0; j < 16; ++j) dst[(size_t)j * ntp] = v[j];
        } else {
          __half* dst = static_cast<__half*>(tg.m) + row;
#pragma unroll
          for (int j = 0; j < 16; ++j) dst[(size_t)j * ntp] = __float2half_rn(v[j]);
        }
      }
      tc_fence_before();
      __syncwarp();
      if (lane == 0) mbar_arrive(&sh.accempty[ab]);
    }
  }
  tc_fence_before();
  __syncthreads();
  if (warp == 1) {
    tc_fence_after();
    tmem_dealloc(tmem, 512);
  }
}

__global__ void __launch_bounds__(NTHREAD, 1) unfused_gemm(KernelParam p) {
  const Geometry g = make_geometry(p, TB2);
  TapGemm s;
  s.v2 = p.transform_pin; s.u2 = p.transform_filter; s.m = p.mid_result;
  s.taps = 16; s.ntb = g.nTB; s.c_red = g.C; s.k = g.K;
  tap_gemm_body<false>(s);
}

__global__ void __launch_bounds__(NTHREAD, 1) tap_gemm_f32(TapGemm s) { tap_gemm_body<true>(s); }

// ------------------------------------------------------ output transform ---
// grid (ceil(tiles/256), K): thread = (tile, k); reads the 16 taps of M16.
__global__ void __launch_bounds__(256) unfused_output_transform(KernelParam p) {
  const Geometry g = make_geometry(p, TB2);
  const long long tile = (long long)blockIdx.x * 256 + threadIdx.x;
  const int k = blockIdx.y;
  if (tile >= g.NT) return;
  const size_t ntp = (size_t)g.nTB * TB2;
  const __half* m16 = static_cast<const __half*>(p.mid_result);
  float m[16];
#pragma unroll
  for (int t = 0; t < 16; ++t) m[t] = __half2float(m16[((size_t)t * g.K + k) * ntp + tile]);
  // A^T m A: rows first (z = At m), then columns.
  float z[2][4];
#pragma unroll
  for (int b = 0; b < 4; ++b) {
    z[0][b] = m[b] + m[4 + b] + m[8 + b];
    z[1][b] = m[4 + b] - m[8 + b] - m[12 + b];
  }
  float y[4];
#pragma unroll
  for (int i = 0; i < 2; ++i) {
    y[2 * i + 0] = z[i][0] + z[i][1] + z[i][2];
    y[2 * i + 1] = z[i][1] - z[i][2] - z[i][3];
  }
  const long long per_img = (long long)g.TP * g.TQ;
  const int n = (int)(tile / per_img);
  const int r = (int)(tile - (long long)n * per_img);
  const int ty = r / g.TQ, tx = r - (r / g.TQ) * g.TQ;
  const int oy = 2 * ty, ox = 2 * tx;
  __half* o = static_cast<__half*>(p.pout) + (((size_t)n * g.K + k) * g.P + oy) * (size_t)g.Q + ox;
  const bool two_cols = ox + 1 < g.Q, two_rows = oy + 1 < g.P;
  if (two_cols && (g.Q & 1) == 0) {
    *reinterpret_cast<__half2*>(o) = __floats2half2_rn(y[0], y[1]);
    if (two_rows) *reinterpret_cast<__half2*>(o + g.Q) = __floats2half2_rn(y[2], y[3]);
  } else {
    o[0] = __float2half_rn(y[0]);
    if (two_cols) o[1] = __float2half_rn(y[1]);
    if (two_rows) {
      o[g.Q] = __float2half_rn(y[2]);
      if (two_cols) o[g.Q + 1] = __float2half_rn(y[3]);
    }
  }
}

}  // namespace wino

using namespace wino;

extern "C" {

// Workspace bytes of the unfused path: V2 and M16.
size_t wino_unfused_v_bytes(int n, int c, int h, int w) {
  const long long nt = (long long)n * ((h + 1) / 2) * ((w + 1) / 2);
  const long long ntp = (nt + TB2 - 1) / TB2 * TB2;
  return (size_t)16 * ntp * c * 2;
}
size_t wino_unfused_m_bytes(int n, int k, int h, int w) {
  const long long nt = (long long)n * ((h + 1) / 2) * ((w + 1) / 2);
  const long long ntp = (nt + TB2 - 1) / TB2 * TB2;
  return (size_t)16 * ntp * k * 2;
}

int wino_unfused_prepare() {
  return (int)cudaFuncSetAttribute(unfused_gemm, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                   unfused::SMEM_BYTES);
}

// p: pin, pout, transform_pin = V2, transform_filter = U2, mid_result = M16.
int wino_unfused_launch(const KernelParam* p, int sms, cudaStream_t stream) {
  const int tp = (p->Oh + 1) / 2, tq = (p->Ow + 1) / 2;
  const long long nt = (long long)p->n * tp * tq;
  const int ntb = (int)((nt + TB2 - 1) / TB2);
  const int cs = p->c / 16;
  unfused_input_transform<<<dim3(ntb, cs), 256, 0, stream>>>(*p);
  const long long units = 16LL * ntb * (((p->k + KB2 - 1) / KB2 + KPU - 1) / KPU);
  const int grid = (int)(units < sms ? units : sms);
  unfused_gemm<<<grid, NTHREAD, unfused::SMEM_BYTES, stream>>>(*p);
  unfused_output_transform<<<dim3((unsigned)((nt + 255) / 256), p->k), 256, 0, stream>>>(*p);
  return (int)cudaGetLastError();
}

int wino_tap_gemm_f32_launch(const TapGemm* s, int sms, void* stream) {
  static const cudaError_t attr = cudaFuncSetAttribute(
      tap_gemm_f32, cudaFuncAttributeMaxDynamicSharedMemorySize, unfused::SMEM_BYTES);
  if (attr != cudaSuccess) return (int)attr;
  const long long units = (long long)s->taps * s->ntb * (((s->k + KB2 - 1) / KB2 + KPU - 1) / KPU);
  const int grid = (int)(units < sms ? units : sms);
  tap_gemm_f32<<<grid, NTHREAD, unfused::SMEM_BYTES, (cudaStream_t)stream>>>(*s);
  return (int)cudaGetLastError();
}

uint32_t wino_unfused_error_read_clear() {
  uint32_t v = 0, z = 0;
  cudaMemcpyFromSymbol(&v, g_unfused_err, sizeof(v));
  cudaMemcpyToSymbol(g_unfused_err, &z, sizeof(z));
  return v;
}

}  // extern "C"
