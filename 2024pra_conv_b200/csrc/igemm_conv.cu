// Implicit-GEMM convolution on the tcgen05 tensor cores, for the shapes the
// Winograd path does not take: any filter R x S, stride (u, v), padding
// (p, q), channel counts that are not multiples of 16 (stride-2 3x3
// downsampling layers, 1x1 projections).  The reference's getkernelInfo
// ignores r, s, u, v, p, q (src/conv2d.cpp:254-271); here those shapes run
// behind the same plugin ABI, on the tensor cores when the re-laid-out
// weights fit the caller's transform_filter, else on the CUDA-core direct
// kernel (direct_conv.cu).
//
//   D[pixel][k] = sum over K-steps (tap (r, s), 16-channel block cb) of
//                 X16[pixel][16 channels at tap] . W16[k][16 channels at tap]
//
// pixel = (n, oy, ox) flattened, K-steps tap-major (ks = (r * S + s) * CB +
// cb, CB = ceil(C / 16)), channels past C zero on both sides.  fp16
// operands, fp32 accumulation in TMEM, one fp16 rounding of y.
//
// Kernels:
//  - igemm_weight_kernel (slot 1 of the drop-in route): KCRS weights into
//    the MMA's K-major B layout, k-block major (256 output channels), K-step
//    next, each K-step a piece of rows x 32 bytes with output channel k,
//    channel c at (k >> 3) * 256 + (c >> 3) * 128 + (k & 7) * 16 + (c & 7) * 2.
//  - igemm_conv_kernel<PM> (slot 3): persistent; a unit is 128 * PM output
//    pixels x one k-block (PM = 2 when K <= 128, so the pixel operand of a
//    K-step feeds two MMAs of 128 pixels each and the accumulator is 256
//    columns either way).  Warps 8-15 build the pixel operand straight from
//    the NCHW input: for 1x1 / stride 1 / pad 0 layers whose H * W is a
//    multiple of 8 (FLAT), one 16-byte load of eight neighbouring pixels per
//    channel into an MN-major operand; otherwise eight 2-byte loads per
//    K-step (thread = pixel, 8-channel half, lanes on consecutive pixels,
//    zero outside the image) into a K-major one.  Warp 5 lane 0 bulk-copies
//    the weight pieces; warp 4 lane 0 issues one M128 x N(rows) x K16 MMA per
//    K-step and pixel half; warps 0-3 read the accumulator (TMEM lane =
//    pixel) and store y, each column a contiguous run of pixels of one output
//    channel, neighbouring lanes pairing up for 4-byte stores.  TMEM holds
//    two 256-column accumulators, so a unit's epilogue overlaps the next
//    unit's MMAs.
#include <cstring>
#include <cuda.h>
#include <cudaTypedefs.h>
#include <cuda_runtime.h>
#include <cuda_fp16.h>
#include "tc_sm100.cuh"
#include "wino_param.h"

namespace wino {

static __device__ uint32_t g_igemm_err;
// zero words the pixel producers read in place of padding and missing channels
static __device__ __align__(16) unsigned short g_igemm_zero[8];

namespace ig {
constexpr int NSTAGE = 4;
constexpr int PIECE = 128 * 16 * 2;       // 4 KB: 128 pixels x 16 channels
constexpr int NPIECE = 4;                 // pixel pieces per stage
constexpr int STAGE_A = NPIECE * PIECE;   // 16 KB
constexpr int KB = 256;                   // output channels per k-block
constexpr int STAGE_B = 4 * KB * 32;      // 32 KB: up to four K-steps of 256 rows
constexpr int STAGE = STAGE_A + STAGE_B;
constexpr int SMEM_BYTES = NSTAGE * STAGE + 1024;
// warps 0-3 epilogue, 4 MMA issue (lane 0), 5 weight loads (lane 0), 6-7
// idle, 8-15 pixel producers.  Launched with 128 registers a thread (the
// whole register file); the epilogue and MMA warpgroups hand registers to
// the producers, whose ring of in-flight loads they hold.
constexpr int WARP_E0 = 0, NWARP_E = 4, WARP_MMA = 4, WARP_LOAD = 5, WARP_P0 = 8, NWARP_P = 8;
constexpr int NTHREAD = (WARP_P0 + NWARP_P) * 32;
constexpr int REGS_LAUNCH = 128, REGS_EPI = 104, REGS_MMA = 56, REGS_PROD = 176;
static_assert(128 * REGS_EPI + 128 * REGS_MMA + 256 * REGS_PROD == NTHREAD * REGS_LAUNCH,
              "the warpgroups' register limits add up to the launch allocation");
constexpr uint32_t SLEEP_NS = 32;
// stages of 16-byte loads each octet producer keeps in registers (five
// measured 4-7 % faster than three on the 1x1 256->64 and 512->128 ResNet
// layers; seven slower)
#ifndef WINO_IG_RING
#define WINO_IG_RING 5
#endif
constexpr int RING_F = WINO_IG_RING;
static_assert(RING_F >= 2 && RING_F <= 8, "ring of two to eight stages");
// stages of 2-byte loads each gathering producer keeps in registers (32 a
// stage, one value a register; four measured 5-11 % slower than three)
#ifndef WINO_IG_RING_GATHER
#define WINO_IG_RING_GATHER 3
#endif
constexpr int RING_G = WINO_IG_RING_GATHER;
static_assert(RING_G >= 2 && RING_G <= 4, "ring of two to four stages");

struct Shared {
  uint64_t full[NSTAGE], empty[NSTAGE];
  uint64_t accfull[2], accempty[2];
  uint64_t mmadone;
  uint32_t tmem_base;
  int abort_flag;
};

// Pixel-operand producers: 2-byte gathers into a K-major operand; 16-byte
// octet loads into an MN-major one (1x1 / stride 1 / pad 0); TMA boxes of
// 64 pixels x 16 channels into a 128-byte-swizzled MN-major one (the same
// layers when H * W is a multiple of 64 and a tensor map is available).
enum : int { MODE_GATHER = 0, MODE_FLAT = 1, MODE_TMA = 2 };

struct Geo {
  int C, H, W, K, S, U, V, P, Q, OW;
  int HW, OHOW, CB, NKS, Kp, nKB, units;
  long long NPIX;
};

__host__ __device__ __forceinline__ int kstep_count(int c, int r, int s) { return r * s * ((c + 15) >> 4); }
__host__ __device__ __forceinline__ int kpad(int k) { return (k + 15) & ~15; }
__host__ __device__ __forceinline__ int block_rows(int kb, int Kp) { return min(KB, Kp - kb * KB); }

template <int PM>
__device__ __forceinline__ Geo geo(const KernelParam& p) {
  Geo g;
  g.C = p.c; g.H = p.h; g.W = p.w; g.K = p.k; g.S = p.s;
  g.U = p.u; g.V = p.v; g.P = p.p; g.Q = p.q; g.OW = p.Ow;
  g.HW = p.h * p.w;
  g.OHOW = p.Oh * p.Ow;
  g.CB = (p.c + 15) >> 4;
  g.NKS = kstep_count(p.c, p.r, p.s);
  g.Kp = kpad(p.k);
  g.nKB = (g.Kp + KB - 1) / KB;
  g.NPIX = (long long)p.n * g.OHOW;
  const long long npt = (g.NPIX + 128 * PM - 1) / (128 * PM);
  g.units = (int)(npt * g.nKB);
  return g;
}

// Unit u of the grid-stride order: pixel tile pt, k-block kb (k-blocks of
// one pixel tile on neighbouring CTAs, so the tile's input is gathered from
// L2 the second time).
__device__ __forceinline__ void unit_of(const Geo& g, int u, int& pt, int& kb) {
  pt = u / g.nKB;
  kb = u - pt * g.nKB;
}
}  // namespace ig

// KCRS weights -> the K-major B pieces (one 16-byte word per thread).
__global__ void __launch_bounds__(256) igemm_weight_kernel(KernelParam p) {
  using namespace ig;
  const int C = p.c, K = p.k, R = p.r, S = p.s;
  const int CB = (C + 15) >> 4, NKS = kstep_count(C, R, S), Kp = kpad(K);
  const long long nword = (long long)Kp * NKS * 2;
  const long long wi = (long long)blockIdx.x * 256 + threadIdx.x;
  if (wi >= nword) return;
  const int hh = (int)(wi & 1);
  const long long r2 = wi >> 1;
  const int k = (int)(r2 / NKS), ks = (int)(r2 - (long long)k * NKS);
  const int kb = k / KB, row = k - kb * KB, rows = block_rows(kb, Kp);
  const int tap = ks / CB, cb = ks - tap * CB;
  const int r = tap / S, s = tap - r * S;
  const unsigned short* w = static_cast<const unsigned short*>(p.pweight);
  uint32_t v[4];
#pragma unroll
  for (int e = 0; e < 8; e += 2) {
    const int c = cb * 16 + hh * 8 + e;
    uint32_t lo = 0, hi = 0;
    if (k < K && c < C) lo = w[(((size_t)k * C + c) * R + r) * S + s];
    if (k < K && c + 1 < C) hi = w[(((size_t)k * C + c + 1) * R + r) * S + s];
    v[e >> 1] = lo | (hi << 16);
  }
  uint8_t* dst = static_cast<uint8_t*>(p.transform_filter) + (size_t)kb * KB * NKS * 32 + (size_t)ks * rows * 32 +
                 (row >> 3) * 256 + hh * 128 + (row & 7) * 16;
  *reinterpret_cast<uint4*>(dst) = make_uint4(v[0], v[1], v[2], v[3]);
}

// FLAT: 1x1 filter, stride 1, no padding, H * W a multiple of 8 and a
// 16-byte aligned input.  The output pixels of an image are then its input
// pixels, eight consecutive ones of a channel are one aligned 16-byte word,
// and the pixel operand is staged MN-major (pixels contiguous): thread =
// (pixel octet, channel), one 16-byte load and one 16-byte shared store per
// octet, channel and K-step.  Otherwise thread = (pixel, channel half) and
// eight 2-byte loads build each K-major 16-byte row.
// MODE_TMA: the weight-loader thread also copies the pixel operand, two TMA
// boxes (64 pixels x 16 channels, 128-byte swizzle) per piece, through the
// tensor map at p.transform_pin (CUtensorMap over the input as [N][C][H*W]);
// the producer warps stay idle.
template <int PM, int MODE>
__global__ void __launch_bounds__(ig::NTHREAD, 1) igemm_conv_kernel(KernelParam p) {
  using namespace ig;
  constexpr bool FLAT = MODE == MODE_FLAT;
  constexpr bool TMA = MODE == MODE_TMA;
  constexpr bool MN = MODE != MODE_GATHER;  // MN-major pixel operand
  constexpr int SKS = NPIECE / PM;          // K-steps per stage
  extern __shared__ __align__(1024) uint8_t smem_raw[];
  __shared__ Shared sh;
  uint8_t* smem = reinterpret_cast<uint8_t*>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
  const Geo g = geo<PM>(p);
  const int warp = warp_id(), lane = lane_id();
  uint32_t* err = &g_igemm_err;
  const int G = (int)gridDim.x, g0 = (int)blockIdx.x;
  const int cnt = g0 < g.units ? (g.units - 1 - g0) / G + 1 : 0;
  const int nst = (g.NKS + SKS - 1) / SKS;
  // two pixel halves need both 128-column halves of an accumulator
  if (PM == 2 && g.Kp > 128) {
    if (threadIdx.x == 0) record_error(&g_igemm_err, ERR_BAD_SHAPE);
    return;
  }

  if (threadIdx.x == 0) {
    for (int s = 0; s < NSTAGE; ++s) {
      mbar_init(&sh.full[s], TMA ? 1 : NWARP_P + 1);
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

  if (warp >= WARP_MMA && warp < WARP_P0) {
    regs_dec<REGS_MMA>();
    if (warp == WARP_LOAD && lane == 0) {
      // weight pieces: stage j of a unit = K-steps j * SKS .., contiguous
      const uint8_t* wp = static_cast<const uint8_t*>(p.transform_filter);
      const void* tmap = p.transform_pin;
      if constexpr (TMA) tensormap_acquire(tmap);
      uint32_t it = 0;
      for (int i = 0; i < cnt && !*abort_flag; ++i) {
        int pt, kb;
        unit_of(g, g0 + i * G, pt, kb);
        const int rows = block_rows(kb, g.Kp);
        const uint8_t* src = wp + (size_t)kb * KB * g.NKS * 32;
        bool ok = true;
        for (int j = 0; j < nst; ++j, ++it) {
          const int st = it % NSTAGE;
          if (it >= NSTAGE &&
              !mbar_wait(&sh.empty[st], (it / NSTAGE - 1) & 1, abort_flag, err, ERR_WAIT_EMPTY)) {
            ok = false;
            break;
          }
          const int nk = min(SKS, g.NKS - j * SKS);
          const uint32_t bytes = (uint32_t)(nk * rows * 32);
          mbar_arrive_expect_tx(&sh.full[st], bytes + (TMA ? (uint32_t)(nk * PM * PIECE) : 0u));
          bulk_g2s(smem + st * STAGE + STAGE_A, src + (size_t)j * SKS * rows * 32, bytes, &sh.full[st]);
          if constexpr (TMA) {
            // piece q * PM + h = channels 16 (j SKS + q) .. of pixel half h:
            // boxes of 64 pixels at 2 KB steps (H * W % 64 == 0, so a box
            // lies in one image; past the last image the copy reads zeros)
            for (int q = 0; q < nk; ++q)
#pragma unroll
              for (int hb = 0; hb < 2 * PM; ++hb) {
                const long long P = (long long)pt * (128 * PM) + hb * 64;
                const int n = (int)(P / g.HW), x = (int)(P - (long long)n * g.HW);
                tma_load_3d(smem + st * STAGE + q * PM * PIECE + hb * 2048, tmap, x, (j * SKS + q) * 16, n,
                            &sh.full[st]);
              }
          }
        }
        if (!ok) break;
      }
      // copies still in flight land before the CTA leaves
      for (uint32_t s2 = it > (uint32_t)NSTAGE ? it - NSTAGE : 0; s2 < it; ++s2)
        mbar_wait(&sh.full[s2 % NSTAGE], (s2 / NSTAGE) & 1, nullptr, err, ERR_WAIT_FULL);
    }
    if (warp == WARP_MMA && lane == 0) {
      // pixel operand of a piece: K-major (8-channel halves 128 bytes apart,
      // pixel octets 256), FLAT MN-major (pixel octets 128 bytes apart,
      // channel halves 2048) or TMA MN-major swizzled (64-pixel atoms 2048
      // bytes apart, 8-channel groups 1024)
      auto a_desc = [](uint32_t a) {
        return TMA ? smem_desc_sw128(a, 2048, 1024) : FLAT ? smem_desc(a, 2048, 128) : smem_desc(a, 128, 256);
      };
      uint32_t it = 0;
      bool ok = true;
      for (int i = 0; ok && i < cnt && !*abort_flag; ++i) {
        int pt, kb;
        unit_of(g, g0 + i * G, pt, kb);
        const int rows = block_rows(kb, g.Kp);
        const uint32_t idesc = instr_desc(128, (uint32_t)rows, 0, 0, MN ? 1 : 0, 0);
        const int ab = i & 1;
        if (i >= 2 && !mbar_wait(&sh.accempty[ab], ((i >> 1) - 1) & 1, abort_flag, err, ERR_WAIT_DRAIN)) break;
        tc_fence_after();
        const uint32_t d = tmem + ab * 256;
        for (int j = 0; j < nst; ++j, ++it) {
          const int st = it % NSTAGE;
          if (!mbar_wait(&sh.full[st], (it / NSTAGE) & 1, abort_flag, err, ERR_WAIT_FULL)) {
            ok = false;
            break;
          }
          tc_fence_after();
          const int nk = min(SKS, g.NKS - j * SKS);
          const uint32_t a0 = sbase + st * STAGE, b0 = a0 + STAGE_A;
          for (int q = 0; q < nk; ++q) {
            const uint64_t bd = smem_desc(b0 + (uint32_t)(q * rows * 32), 128, 256);
#pragma unroll
            for (int h = 0; h < PM; ++h)
              mma_f16(d + h * 128, a_desc(a0 + (uint32_t)((q * PM + h) * PIECE)), bd, idesc,
                      (j > 0 || q > 0) ? 1u : 0u);
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
    regs_dec<REGS_EPI>();
    // epilogue: TMEM lane 32 * quarter + lane = pixel of the half
    const int quarter = warp & 3;
    __half* Y = static_cast<__half*>(p.pout);
    // pixel pairs share 4-byte stores when every image holds an even pixel
    // count (then NPIX is even too, and a pair is live or dead as a whole)
    const bool pair = (g.OHOW & 1) == 0;
    for (int ui = 0; ui < cnt; ++ui) {
      int pt, kb;
      unit_of(g, g0 + ui * G, pt, kb);
      const int rows = block_rows(kb, g.Kp);
      const int kval = min(rows, g.K - kb * KB);   // output channels of the block that exist
      const int ab = ui & 1;
      if (!mbar_wait_warp(&sh.accfull[ab], (ui >> 1) & 1, abort_flag, err, ERR_WAIT_ACCUM, SLEEP_NS)) break;
      tc_fence_after();
#pragma unroll 1
      for (int h = 0; h < PM; ++h) {
        const long long P = (long long)pt * (128 * PM) + h * 128 + quarter * 32 + lane;
        const bool live = P < g.NPIX;
        long long n = 0, rem = 0;
        if (live) {
          n = P / g.OHOW;
          rem = P - n * g.OHOW;
        }
        __half* yb = Y + ((size_t)n * g.K + (size_t)kb * KB) * g.OHOW + rem;
        const uint32_t taddr = tmem + ((uint32_t)(quarter * 32) << 16) + ab * 256 + h * 128;
        auto ld = [&](int cc, float* v) {
          tmem_ld16(taddr + cc, v);
          if (cc + 16 < rows) tmem_ld16(taddr + cc + 16, v + 16);
        };
        // pixel pairs of one image share 4-byte stores (see `pair`)
        auto st = [&](int cc, const float* v) {
          store_cols_f16<32>(yb + (size_t)cc * g.OHOW, (size_t)g.OHOW, v, kval - cc, live, pair);
        };
        float va[32], vb[32];
        ld(0, va);
        tmem_ld_wait();
        for (int cc = 0; cc < rows; cc += 64) {
          if (cc + 32 < rows) ld(cc + 32, vb);
          st(cc, va);
          tmem_ld_wait();
          if (cc + 32 >= rows) break;
          if (cc + 64 < rows) ld(cc + 64, va);
          st(cc + 32, vb);
          tmem_ld_wait();
        }
      }
      tc_fence_before();
      __syncwarp();
      if (lane == 0) mbar_arrive(&sh.accempty[ab]);
    }
  } else if constexpr (FLAT) {
    regs_inc<REGS_PROD>();
    // octet producers: warp pw covers octets 4 (pw & 3) .. + 3 of each
    // 128-pixel half and channels 8 (pw >> 2) .. + 7 of the K-step; lane l
    // takes octet l >> 3 of those and channel l & 7, so the eight lanes of a
    // shared-store phase fill one 128-byte octet row without bank conflicts
    // and lanes 8 apart load neighbouring octets of a channel.
    const int pw = warp - WARP_P0;
    const int o = (lane >> 3) + 4 * (pw & 3), c16 = (lane & 7) + 8 * (pw >> 2);
    const __half* X = static_cast<const __half*>(p.pin);
    const uint4* zero4 = reinterpret_cast<const uint4*>(g_igemm_zero);
    int lu = 0, lj = 0;
    long long off[PM];
    bool live[PM];
#pragma unroll
    for (int h = 0; h < PM; ++h) {
      off[h] = 0;
      live[h] = false;
    }
    uint4 ring[RING_F][NPIECE];
    auto issue = [&](uint4 (&w)[NPIECE]) {
      if (lu >= cnt) return;
      if (lj == 0) {
        int pt, kb;
        unit_of(g, g0 + lu * G, pt, kb);
#pragma unroll
        for (int h = 0; h < PM; ++h) {
          const long long P = (long long)pt * (128 * PM) + h * 128 + 8 * o;   // octets lie in one image
          live[h] = P < g.NPIX;
          const long long n = live[h] ? P / g.HW : 0;
          off[h] = n * g.C * g.HW + (P - n * g.HW);
        }
      }
#pragma unroll
      for (int q = 0; q < SKS; ++q) {
        const int ch = (lj * SKS + q) * 16 + c16;      // one K-step per 16 channels
        const bool kv = lj * SKS + q < g.NKS && ch < g.C;
#pragma unroll
        for (int h = 0; h < PM; ++h)
          w[q * PM + h] = __ldg(kv && live[h] ? reinterpret_cast<const uint4*>(X + off[h] + (long long)ch * g.HW)
                                              : zero4);
      }
      if (++lj == nst) { lj = 0; ++lu; }
    };
    uint32_t it = 0;
    int cu = 0, cj = 0;
    auto consume = [&](const uint4 (&w)[NPIECE]) -> bool {
      const int st = it % NSTAGE;
      if (it >= NSTAGE &&
          !mbar_wait_warp(&sh.empty[st], (it / NSTAGE - 1) & 1, abort_flag, err, ERR_WAIT_EMPTY, SLEEP_NS))
        return false;
      const int npc = min(NPIECE, (g.NKS - cj * SKS) * PM);
      uint8_t* adst = smem + st * STAGE + (c16 >> 3) * 2048 + o * 128 + (c16 & 7) * 16;
#pragma unroll
      for (int pc = 0; pc < NPIECE; ++pc)
        if (pc < npc) *reinterpret_cast<uint4*>(adst + pc * PIECE) = w[pc];
      fence_proxy_async_shared();
      __syncwarp();
      if (lane == 0) mbar_arrive(&sh.full[st]);
      ++it;
      if (++cj == nst) { cj = 0; ++cu; }
      return cu < cnt && !*abort_flag;
    };
    if (cnt > 0) {
      // RING_F - 1 stages of loads in flight while one is stored
#pragma unroll
      for (int r = 0; r + 1 < RING_F; ++r) issue(ring[r]);
      bool more = true;
      while (more) {
#pragma unroll
        for (int r = 0; r < RING_F; ++r) {
          issue(ring[(r + RING_F - 1) % RING_F]);
          if (!consume(ring[r])) {
            more = false;
            break;
          }
        }
      }
    }
  } else if constexpr (MODE == MODE_GATHER) {
    regs_inc<REGS_PROD>();
    // pixel producers: thread = (pixel tl of each 128-pixel half, channel
    // half hh).  The load cursor (lu, lj) runs up to two stages ahead of
    // the store cursor; a ring slot holds one stage's loads (NPIECE pieces x
    // 8 channels, one 2-byte value a register).
    const int pw = warp - WARP_P0;
    const int tl = (pw & 3) * 32 + lane, hh = pw >> 2;
    const unsigned short* X = static_cast<const unsigned short*>(p.pin);
    int lu = 0, lj = 0;
    int kr = 0, kx = 0, kc = 0;           // tap row, tap column, channel block of the next K-step
    const unsigned short* img[PM];
    int iy0[PM], ix0[PM];
    bool live[PM];
#pragma unroll
    for (int h = 0; h < PM; ++h) {
      img[h] = X;
      iy0[h] = ix0[h] = 0;
      live[h] = false;
    }
    uint32_t wr[RING_G][NPIECE][8];
    auto issue = [&](uint32_t (&w)[NPIECE][8]) {
      if (lu >= cnt) return;
      if (lj == 0) {
        int pt, kb;
        unit_of(g, g0 + lu * G, pt, kb);
#pragma unroll
        for (int h = 0; h < PM; ++h) {
          const long long P = (long long)pt * (128 * PM) + h * 128 + tl;
          live[h] = P < g.NPIX;
          long long n = 0;
          int rem = 0;
          if (live[h]) {
            n = P / g.OHOW;
            rem = (int)(P - n * g.OHOW);
          }
          const int oy = rem / g.OW, ox = rem - oy * g.OW;
          img[h] = X + (size_t)n * g.C * g.HW;
          iy0[h] = oy * g.U - g.P;
          ix0[h] = ox * g.V - g.Q;
        }
        kr = kx = kc = 0;
      }
#pragma unroll
      for (int q = 0; q < SKS; ++q) {
        const int c0 = kc * 16 + hh * 8;
        const int nc = lj * SKS + q < g.NKS ? g.C - c0 : 0;   // channels of this thread's half that exist
#pragma unroll
        for (int h = 0; h < PM; ++h) {
          const int iy = iy0[h] + kr, ix = ix0[h] + kx;
          const bool ok = live[h] && nc > 0 && (unsigned)iy < (unsigned)g.H && (unsigned)ix < (unsigned)g.W;
          // every load is unconditional (so none waits on another): what is
          // outside the image or past C reads the zero words instead
          const unsigned short* src = ok ? img[h] + (c0 * g.HW + iy * g.W + ix) : g_igemm_zero;
          const int step = ok ? g.HW : 0;
          if (nc >= 8) {
#pragma unroll
            for (int e = 0; e < 8; ++e) w[q * PM + h][e] = __ldg(src + e * step);
          } else {
#pragma unroll
            for (int e = 0; e < 8; ++e) w[q * PM + h][e] = __ldg(e < nc ? src + e * step : g_igemm_zero);
          }
        }
        if (++kc == g.CB) {
          kc = 0;
          if (++kx == g.S) { kx = 0; ++kr; }
        }
      }
      if (++lj == nst) { lj = 0; ++lu; }
    };
    uint32_t it = 0;
    int cu = 0, cj = 0;
    auto consume = [&](const uint32_t (&w)[NPIECE][8]) -> bool {
      const int st = it % NSTAGE;
      if (it >= NSTAGE &&
          !mbar_wait_warp(&sh.empty[st], (it / NSTAGE - 1) & 1, abort_flag, err, ERR_WAIT_EMPTY, SLEEP_NS))
        return false;
      const int npc = min(NPIECE, (g.NKS - cj * SKS) * PM);
      uint8_t* adst = smem + st * STAGE + (tl >> 3) * 256 + hh * 128 + (tl & 7) * 16;
#pragma unroll
      for (int pc = 0; pc < NPIECE; ++pc) {
        if (pc < npc) {
          const uint4 v = make_uint4(w[pc][0] | (w[pc][1] << 16), w[pc][2] | (w[pc][3] << 16),
                                     w[pc][4] | (w[pc][5] << 16), w[pc][6] | (w[pc][7] << 16));
          *reinterpret_cast<uint4*>(adst + pc * PIECE) = v;
        }
      }
      fence_proxy_async_shared();
      __syncwarp();
      if (lane == 0) mbar_arrive(&sh.full[st]);
      ++it;
      if (++cj == nst) { cj = 0; ++cu; }
      return cu < cnt && !*abort_flag;
    };
    if (cnt > 0) {
      // RING_G - 1 stages of loads in flight while one is stored
#pragma unroll
      for (int r = 0; r + 1 < RING_G; ++r) issue(wr[r]);
      bool more = true;
      while (more) {
#pragma unroll
        for (int r = 0; r < RING_G; ++r) {
          issue(wr[(r + RING_G - 1) % RING_G]);
          if (!consume(wr[r])) {
            more = false;
            break;
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

// Bytes of the re-laid-out weights: K rounded up to 16 rows, R * S *
// ceil(C / 16) K-steps of 32 bytes a row.
size_t wino_igemm_operand_bytes(int c, int k, int r, int s) {
  return (size_t)ig::kpad(k) * (size_t)ig::kstep_count(c, r, s) * 32;
}

// The extension API's weight buffer: the operand, then (at a 128-byte
// boundary) a 128-byte slot for the input's tensor map.
size_t wino_igemm_map_offset(int c, int k, int r, int s) {
  return (wino_igemm_operand_bytes(c, k, r, s) + 127) / 128 * 128;
}
size_t wino_igemm_weight_bytes(int c, int k, int r, int s) { return wino_igemm_map_offset(c, k, r, s) + 128; }

unsigned wino_igemm_weight_grid(int c, int k, int r, int s) {
  const long long nword = (long long)ig::kpad(k) * ig::kstep_count(c, r, s) * 2;
  return (unsigned)((nword + 255) / 256);
}

void* wino_igemm_weight_kernel_ptr() { return (void*)igemm_weight_kernel; }

// Two pixel halves a unit when the output channels fit one 128-row block.
static int igemm_pm(int k) { return ig::kpad(k) <= 128 ? 2 : 1; }

// The octet-loading (FLAT) instance serves 1x1 / stride 1 / pad 0 problems
// with H * W a multiple of 8 and a 16-byte aligned input.
int wino_igemm_flat(const void* x, int h, int w, int r, int s, int u, int v, int p, int q) {
  return r == 1 && s == 1 && u == 1 && v == 1 && p == 0 && q == 0 && ((long long)h * w) % 8 == 0 &&
         (reinterpret_cast<uintptr_t>(x) & 15) == 0;
}

// TMA boxes for the pixel operand (MODE_TMA) where they measured faster
// than the octet loads: 1x1 64->256 at 56x56, N128, 110 -> 100 us (one pixel
// half a unit); with two pixel halves (K <= 128: 1x1 256->64) they were
// slower, 97 -> 117 us, so those keep the octet loads.
#ifndef WINO_IG_TMA
#define WINO_IG_TMA 1
#endif

// The driver's tensor-map encoder (looked up once; null when unavailable).
static PFN_cuTensorMapEncodeTiled_v12000 map_encoder() {
  static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
  static bool looked = false;
  if (!looked) {
    looked = true;
    void* f = nullptr;
    cudaDriverEntryPointQueryResult q{};
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &f, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(f);
  }
  return fn;
}

// Pixel-operand producer for a problem (ig::MODE_*): TMA for FLAT problems
// with H * W a multiple of 64 and one pixel half a unit (K > 128) when the
// build enables it and the driver encodes tensor maps.
int wino_igemm_mode(const void* x, int k, int h, int w, int r, int s, int u, int v, int p, int q) {
  if (!wino_igemm_flat(x, h, w, r, s, u, v, p, q)) return ig::MODE_GATHER;
  if (WINO_IG_TMA && igemm_pm(k) == 1 && ((long long)h * w) % 64 == 0 && map_encoder() != nullptr)
    return ig::MODE_TMA;
  return ig::MODE_FLAT;
}

// Tensor map of the input x (N C H*W fp16) with boxes of 64 pixels x 16
// channels and the 128-byte swizzle, written to the 128 bytes at map_host.
int wino_igemm_encode_map(void* map_host, const void* x, int n, int c, int hw) {
  PFN_cuTensorMapEncodeTiled_v12000 fn = map_encoder();
  if (!fn || !map_host || !x) return 1;
  CUtensorMap m;
  const cuuint64_t dims[3] = {(cuuint64_t)hw, (cuuint64_t)c, (cuuint64_t)n};
  const cuuint64_t strides[2] = {(cuuint64_t)hw * 2, (cuuint64_t)c * hw * 2};
  const cuuint32_t box[3] = {64, 16, 1};
  const cuuint32_t es[3] = {1, 1, 1};
  if (fn(&m, CU_TENSOR_MAP_DATA_TYPE_FLOAT16, 3, const_cast<void*>(x), dims, strides, box, es,
         CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
         CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) != CUDA_SUCCESS)
    return 1;
  static_assert(sizeof(CUtensorMap) == 128, "a tensor map is 128 bytes");
  std::memcpy(map_host, &m, sizeof(m));
  return 0;
}

void* wino_igemm_kernel_ptr(int k, int mode) {
  const bool two = igemm_pm(k) == 2;
  switch (mode) {
    case ig::MODE_TMA: return two ? (void*)igemm_conv_kernel<2, ig::MODE_TMA> : (void*)igemm_conv_kernel<1, ig::MODE_TMA>;
    case ig::MODE_FLAT: return two ? (void*)igemm_conv_kernel<2, ig::MODE_FLAT> : (void*)igemm_conv_kernel<1, ig::MODE_FLAT>;
    default: return two ? (void*)igemm_conv_kernel<2, ig::MODE_GATHER> : (void*)igemm_conv_kernel<1, ig::MODE_GATHER>;
  }
}

int wino_igemm_threads() { return ig::NTHREAD; }
int wino_igemm_smem_bytes() { return ig::SMEM_BYTES; }

long long wino_igemm_units(int n, int k, int oh, int ow) {
  const int pm = igemm_pm(k);
  const long long npix = (long long)n * oh * ow;
  const long long kb = (ig::kpad(k) + ig::KB - 1) / ig::KB;
  return (npix + 128 * pm - 1) / (128 * pm) * kb;
}

unsigned wino_igemm_grid(int n, int k, int oh, int ow, int sms) {
  const long long u = wino_igemm_units(n, k, oh, ow);
  return (unsigned)(u < sms ? u : sms);
}

// Shapes the kernel indexes correctly: one image's input in 32-bit element
// offsets and the unit count in an int.
int wino_igemm_shape_ok(int n, int c, int h, int w, int k, int oh, int ow) {
  if ((long long)c * h * w >= (1LL << 31)) return 0;
  if (wino_igemm_units(n, k, oh, ow) >= (1LL << 31)) return 0;
  return 1;
}

int wino_igemm_prepare() {
  // attributes are per function and device: set them once per device (a
  // repeated set from another thread is harmless)
  static int done[64] = {};
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) return 1;
  if (dev >= 0 && dev < 64 && done[dev]) return 0;
  const void* fns[6] = {(void*)igemm_conv_kernel<1, ig::MODE_GATHER>, (void*)igemm_conv_kernel<2, ig::MODE_GATHER>,
                        (void*)igemm_conv_kernel<1, ig::MODE_FLAT>,   (void*)igemm_conv_kernel<2, ig::MODE_FLAT>,
                        (void*)igemm_conv_kernel<1, ig::MODE_TMA>,    (void*)igemm_conv_kernel<2, ig::MODE_TMA>};
  for (const void* f : fns) {
    if (cudaFuncSetAttribute(f, cudaFuncAttributeMaxDynamicSharedMemorySize, ig::SMEM_BYTES) != cudaSuccess)
      return 1;
    // the warpgroups split exactly the registers the block launches with
    cudaFuncAttributes fa{};
    if (cudaFuncGetAttributes(&fa, f) != cudaSuccess || fa.numRegs != ig::REGS_LAUNCH) return 1;
  }
  if (dev >= 0 && dev < 64) done[dev] = 1;
  return 0;
}

uint32_t wino_igemm_error_read_clear() {
  uint32_t v = 0, z = 0;
  cudaMemcpyFromSymbol(&v, g_igemm_err, sizeof(v));
  cudaMemcpyToSymbol(g_igemm_err, &z, sizeof(z));
  return v;
}

}  // extern "C"
