// Thin inline-PTX layer for the sm_100a features the Winograd kernels use:
// mbarriers with bounded waits, bulk copies global->shared, tcgen05 tensor
// memory (alloc / mma / commit / ld / st) and cluster shared-memory access.
//
// Every wait is bounded: after WINO_WAIT_NS nanoseconds the waiter records an
// error code in the kernel's device error word and returns false, so a
// protocol bug ends the kernel with a status the host reads instead of a hung
// GPU.
#pragma once
#include <cstdint>
#include <cuda_fp16.h>
#include <cuda_bf16.h>

namespace wino {

// ---------------------------------------------------------------- errors ---
// Error codes written to the device error word (first error wins).
enum : uint32_t {
  ERR_NONE = 0,
  ERR_WAIT_FULL = 1,      // consumer waited too long for a filled stage
  ERR_WAIT_EMPTY = 2,     // producer waited too long for a free stage
  ERR_WAIT_ACCUM = 3,     // epilogue waited too long for the accumulator
  ERR_WAIT_DRAIN = 4,     // MMA warp waited too long for the epilogue
  ERR_WAIT_CLUSTER = 5,   // cluster exchange waited too long
  ERR_WAIT_WORK = 6,      // persistent scheduler dependency never signalled
  ERR_BAD_SHAPE = 16,     // kernel launched with a shape it cannot run
};

// Longest any single wait may take before it is declared failed (ns).
#ifndef WINO_WAIT_NS
#define WINO_WAIT_NS 1000000000ull
#endif

__device__ __forceinline__ uint64_t globaltimer_ns() {
  uint64_t t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ void record_error(uint32_t* err, uint32_t code) {
  if (err) atomicCAS(err, 0u, code);
}

// --------------------------------------------------------------- mbarrier ---
__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count));
}

__device__ __forceinline__ void fence_barrier_init() {
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

__device__ __forceinline__ void mbar_arrive(uint64_t* bar) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(bar)) : "memory");
}

__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t* bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)),
               "r"(bytes)
               : "memory");
}

// Arrive on an mbarrier of another CTA of the cluster (address from mapa).
__device__ __forceinline__ void mbar_arrive_remote(uint32_t cluster_addr) {
  asm volatile("mbarrier.arrive.release.cluster.shared::cluster.b64 _, [%0];" ::"r"(cluster_addr)
               : "memory");
}

// Arrive on an mbarrier of the cluster (own CTA or peer, address from mapa)
// with CTA-scope release: it orders this thread's shared-memory and tensor
// memory accesses before the arrival without waiting for its outstanding
// global loads and stores, which a cluster-scope release would.  Used where
// the data handed over is in shared memory (operands for the pair MMA, made
// visible to it by fence.proxy.async) or in TMEM (drained accumulators).
__device__ __forceinline__ void mbar_arrive_peer(uint32_t cluster_addr) {
  asm volatile("mbarrier.arrive.shared::cluster.b64 _, [%0];" ::"r"(cluster_addr) : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
      "selp.u32 %0, 1, 0, p;\n\t}"
      : "=r"(ok)
      : "r"(smem_u32(bar)), "r"(parity)
      : "memory");
  return ok != 0;
}

// Cluster-scope acquire variant (for barriers that remote CTAs arrive on).
__device__ __forceinline__ bool mbar_try_wait_cluster(uint64_t* bar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "mbarrier.try_wait.parity.acquire.cluster.shared::cta.b64 p, [%1], %2;\n\t"
      "selp.u32 %0, 1, 0, p;\n\t}"
      : "=r"(ok)
      : "r"(smem_u32(bar)), "r"(parity)
      : "memory");
  return ok != 0;
}

// Bounded wait.  `abort` is a shared flag that any failing waiter raises so
// that the other roles of the CTA stop waiting as well.
template <bool kCluster>
__device__ __forceinline__ bool mbar_wait_impl(uint64_t* bar, uint32_t parity, volatile int* abort,
                                               uint32_t* err, uint32_t code) {
  auto poll = [&]() { return kCluster ? mbar_try_wait_cluster(bar, parity) : mbar_try_wait(bar, parity); };
  if (poll()) return true;
  const uint64_t t0 = globaltimer_ns();
  for (uint32_t i = 1;; ++i) {
    if (poll()) return true;
    if (abort && *abort) return false;
    if ((i & 63) == 0 && globaltimer_ns() - t0 > WINO_WAIT_NS) break;
  }
  record_error(err, code);
  if (abort) *abort = 1;
  return false;
}

__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t parity, volatile int* abort,
                                          uint32_t* err, uint32_t code) {
  return mbar_wait_impl<false>(bar, parity, abort, err, code);
}

// Warp-wide wait: lane 0 polls (bounded, optional sleep between polls once
// the wait is long) and the outcome is broadcast; all lanes of the warp call.
__device__ __forceinline__ bool mbar_wait_warp(uint64_t* bar, uint32_t parity, volatile int* abort,
                                               uint32_t* err, uint32_t code, uint32_t sleep_ns = 0) {
  uint32_t ok = 1;
  if ((threadIdx.x & 31) == 0) {
    ok = 0;
    if (mbar_try_wait(bar, parity)) {
      ok = 1;
    } else {
      const uint64_t t0 = globaltimer_ns();
      for (uint32_t i = 1;; ++i) {
        if (mbar_try_wait(bar, parity)) { ok = 1; break; }
        if (abort && *abort) break;
        if (sleep_ns && i > 8) __nanosleep(sleep_ns);
        if ((i & 63) == 0 && globaltimer_ns() - t0 > WINO_WAIT_NS) {
          record_error(err, code);
          if (abort) *abort = 1;
          break;
        }
      }
    }
  }
  return __shfl_sync(0xffffffffu, ok, 0) != 0;
}

__device__ __forceinline__ bool mbar_wait_cluster(uint64_t* bar, uint32_t parity,
                                                  volatile int* abort, uint32_t* err,
                                                  uint32_t code) {
  return mbar_wait_impl<true>(bar, parity, abort, err, code);
}

// ------------------------------------------------------------ bulk copies ---
// 1-D bulk copy global -> this CTA's shared memory, completing `bytes` of
// transaction count on `bar`.  Both addresses 16-byte aligned, bytes % 16 == 0.
__device__ __forceinline__ void bulk_g2s(void* dst_smem, const void* src_gmem, uint32_t bytes,
                                         uint64_t* bar) {
  asm volatile(
      "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
          smem_u32(dst_smem)),
      "l"(src_gmem), "r"(bytes), "r"(smem_u32(bar))
      : "memory");
}

// Same with an L2 eviction-priority hint (policy from createpolicy).
__device__ __forceinline__ void bulk_g2s_hint(void* dst_smem, const void* src_gmem, uint32_t bytes,
                                              uint64_t* bar, uint64_t policy) {
  asm volatile(
      "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes.L2::cache_hint [%0], [%1], "
      "%2, [%3], %4;" ::"r"(smem_u32(dst_smem)),
      "l"(src_gmem), "r"(bytes), "r"(smem_u32(bar)), "l"(policy)
      : "memory");
}

// 3-D tiled TMA load of one box of the tensor map at `tmap` (a CUtensorMap in
// global memory) at coordinates (x, y, z), completing its bytes on `bar`.
// x times the element size must be a multiple of 16 bytes; coordinates past
// the tensor's extent read zeros.
__device__ __forceinline__ void tma_load_3d(void* dst_smem, const void* tmap, int x, int y, int z, uint64_t* bar) {
  asm volatile(
      "cp.async.bulk.tensor.3d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4}], "
      "[%5];" ::"r"(smem_u32(dst_smem)),
      "l"(tmap), "r"(x), "r"(y), "r"(z), "r"(smem_u32(bar))
      : "memory");
}

// Makes a tensor map written to global memory before the launch visible to
// the copy engine's reads of it.
__device__ __forceinline__ void tensormap_acquire(const void* tmap) {
  asm volatile("fence.proxy.tensormap::generic.acquire.gpu [%0], 128;" ::"l"(tmap) : "memory");
}

// Bring [src, src + bytes) from device memory into L2 without a destination
// (16-byte aligned, bytes % 16 == 0); completes on its own.
__device__ __forceinline__ void bulk_prefetch_l2(const void* src, uint32_t bytes) {
  asm volatile("cp.async.bulk.prefetch.L2.global [%0], %1;" ::"l"(src), "r"(bytes) : "memory");
}

__device__ __forceinline__ uint64_t policy_evict_last() {
  uint64_t p;
  asm volatile("createpolicy.fractional.L2::evict_last.b64 %0, 1.0;" : "=l"(p));
  return p;
}

__device__ __forceinline__ uint64_t policy_evict_first() {
  uint64_t p;
  asm volatile("createpolicy.fractional.L2::evict_first.b64 %0, 1.0;" : "=l"(p));
  return p;
}

// ---------------------------------------------------------------- cluster ---
__device__ __forceinline__ uint32_t cluster_ctarank() {
  uint32_t r;
  asm volatile("mov.u32 %0, %%cluster_ctarank;" : "=r"(r));
  return r;
}

// Map a shared::cta address of this CTA to the same offset in CTA `rank`.
__device__ __forceinline__ uint32_t mapa_shared(uint32_t addr, uint32_t rank) {
  uint32_t out;
  asm volatile("mapa.shared::cluster.u32 %0, %1, %2;" : "=r"(out) : "r"(addr), "r"(rank));
  return out;
}

__device__ __forceinline__ void st_cluster_v4(uint32_t addr, float a, float b, float c, float d) {
  asm volatile("st.shared::cluster.v4.f32 [%0], {%1, %2, %3, %4};" ::"r"(addr), "f"(a), "f"(b),
               "f"(c), "f"(d)
               : "memory");
}

__device__ __forceinline__ void cluster_arrive() {
  asm volatile("barrier.cluster.arrive.release.aligned;" ::: "memory");
}
__device__ __forceinline__ void cluster_wait() {
  asm volatile("barrier.cluster.wait.acquire.aligned;" ::: "memory");
}
__device__ __forceinline__ void cluster_sync() {
  cluster_arrive();
  cluster_wait();
}

// ----------------------------------------------------------------- tcgen05 --
// Allocate `ncols` TMEM columns (power of two >= 32); whole warp calls.
__device__ __forceinline__ void tmem_alloc(uint32_t* dst_smem, uint32_t ncols) {
  asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                   smem_u32(dst_smem)),
               "r"(ncols)
               : "memory");
}
__device__ __forceinline__ void tmem_relinquish() {
  asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
}
__device__ __forceinline__ void tmem_dealloc(uint32_t taddr, uint32_t ncols) {
  asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(taddr), "r"(ncols)
               : "memory");
}

__device__ __forceinline__ void tc_fence_before() {
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
}
__device__ __forceinline__ void tc_fence_after() {
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
}

// Shared-memory matrix descriptor, no swizzle ("interleaved" canonical
// layout): core matrices of 8 rows x 16 bytes stored as 128 contiguous bytes.
// lbo = byte distance between core matrices adjacent along K,
// sbo = byte distance between core matrices adjacent along M (or N).
// Bits: [0,14) addr>>4, [16,30) lbo>>4, [32,46) sbo>>4, [46,48) version 1,
// [61,64) layout 0 (no swizzle).
__device__ __forceinline__ uint64_t smem_desc(uint32_t saddr, uint32_t lbo, uint32_t sbo) {
  uint64_t d = 0;
  d |= (uint64_t)((saddr >> 4) & 0x3FFFu);
  d |= (uint64_t)((lbo >> 4) & 0x3FFFu) << 16;
  d |= (uint64_t)((sbo >> 4) & 0x3FFFu) << 32;
  d |= (uint64_t)1 << 46;
  return d;
}

// Same with the 128-byte swizzle (layout type 2 in bits [61, 64)): the
// operand is stored in 1024-byte atoms of 8 rows x 128 bytes whose 16-byte
// chunks are XOR-permuted by the row index, as a TMA copy with
// CU_TENSOR_MAP_SWIZZLE_128B writes them.  For an MN-major operand lbo is the
// byte distance between atoms along M/N and sbo between 8-row groups along K.
__device__ __forceinline__ uint64_t smem_desc_sw128(uint32_t saddr, uint32_t lbo, uint32_t sbo) {
  return smem_desc(saddr, lbo, sbo) | ((uint64_t)2 << 61);
}

// Instruction descriptor for kind::f16 / kind::f8f6f4 with fp32 accumulate.
// a_fmt/b_fmt: kind::f16 -> 0 f16, 1 bf16; kind::f8f6f4 -> 0 e4m3, 1 e5m2.
// a_mn/b_mn: 0 = K-major, 1 = MN-major.
__host__ __device__ constexpr uint32_t instr_desc(uint32_t M, uint32_t N, uint32_t a_fmt,
                                                  uint32_t b_fmt, uint32_t a_mn, uint32_t b_mn,
                                                  uint32_t neg_a = 0, uint32_t neg_b = 0) {
  return (1u << 4)                 // D = f32
         | (a_fmt << 7) | (b_fmt << 10) | (neg_a << 13) | (neg_b << 14) | (a_mn << 15) |
         (b_mn << 16) | ((N >> 3) << 17) | ((M >> 4) << 24);
}

// D[tmem] (+)= A[smem] * B[smem]^T, issued by one thread.
__device__ __forceinline__ void mma_f16(uint32_t d_tmem, uint64_t a_desc, uint64_t b_desc,
                                        uint32_t idesc, uint32_t accumulate) {
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}" ::"r"(d_tmem),
      "l"(a_desc), "l"(b_desc), "r"(idesc), "r"(accumulate)
      : "memory");
}

__device__ __forceinline__ void mma_f8(uint32_t d_tmem, uint64_t a_desc, uint64_t b_desc,
                                       uint32_t idesc, uint32_t accumulate) {
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::f8f6f4 [%0], %1, %2, %3, p;\n\t}" ::"r"(d_tmem),
      "l"(a_desc), "l"(b_desc), "r"(idesc), "r"(accumulate)
      : "memory");
}

// Arrive once on `bar` when all previously issued MMAs of this thread finish.
__device__ __forceinline__ void mma_commit(uint64_t* bar) {
  asm volatile(
      "tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
          smem_u32(bar))
      : "memory");
}

// 32 lanes x 32 bit, 16 consecutive columns -> 16 registers per thread.
// Thread i of the warp reads TMEM lane (lane_base + i).
__device__ __forceinline__ void tmem_ld16(uint32_t taddr, float* v) {
  uint32_t r[16];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 "
      "{%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]),
        "=r"(r[7]), "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]),
        "=r"(r[14]), "=r"(r[15])
      : "r"(taddr));
#pragma unroll
  for (int i = 0; i < 16; ++i) v[i] = __uint_as_float(r[i]);
}

__device__ __forceinline__ void tmem_ld8(uint32_t taddr, float* v) {
  uint32_t r[8];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x8.b32 {%0,%1,%2,%3,%4,%5,%6,%7}, [%8];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]),
        "=r"(r[7])
      : "r"(taddr));
#pragma unroll
  for (int i = 0; i < 8; ++i) v[i] = __uint_as_float(r[i]);
}

__device__ __forceinline__ void tmem_ld_wait() {
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
}

// Epilogue store of NC accumulator columns held one row a lane (v[c] = row
// lane, column c, as tcgen05.ld 32x32b returns them) into fp16 memory where
// a row's consecutive elements are neighbours and columns are `stride`
// elements apart: element (lane, c) goes to row[c * stride], `row` being this
// lane's element of column 0.  Columns c < lim are stored (lim uniform across
// the warp; v may hold garbage past it).  With `pair` (stride even, the even
// lane's row element 4-byte aligned, lanes 2i and 2i + 1 live together) the
// two lanes of a pair swap one value per column pair, so each stores one
// 4-byte word of both rows: half the stores and one two-value conversion per
// word.  The loop has no early exit, so the shuffles of a chunk issue back
// to back.  All 32 lanes call.
template <int NC>
__device__ __forceinline__ void store_cols_f16(__half* row, size_t stride, const float* v, int lim, bool live,
                                               bool pair) {
  const bool odd = (threadIdx.x & 1) != 0;
  if (pair) {
    __half* first = row - (odd ? 1 : 0);   // the pair's even row
    // groups of eight column pairs: eight shuffles in flight, then their stores
#pragma unroll
    for (int j0 = 0; j0 < NC / 2; j0 += 8) {
      float other[8];
#pragma unroll
      for (int j = 0; j < 8; ++j)
        other[j] = __shfl_xor_sync(0xffffffffu, odd ? v[2 * (j0 + j)] : v[2 * (j0 + j) + 1], 1);
#pragma unroll
      for (int j = 0; j < 8; ++j) {
        const int c = 2 * (j0 + j);
        const __half2 hv = odd ? __floats2half2_rn(other[j], v[c + 1]) : __floats2half2_rn(v[c], other[j]);
        const int col = c + (odd ? 1 : 0);
        if (live && col < lim) *reinterpret_cast<__half2*>(first + (size_t)col * stride) = hv;
      }
    }
  } else if (live) {
#pragma unroll
    for (int jj = 0; jj < NC; ++jj)
      if (jj < lim) row[(size_t)jj * stride] = __float2half_rn(v[jj]);
  }
}

// ------------------------------------------------- CTA pairs (cta_group::2) --
// A cluster of two CTAs on two SMs runs one MMA over both: A (M = 256) is
// split by rows, each CTA holding 128 rows in its own shared memory; B is
// split by columns, each CTA holding N/2 rows of B; each CTA's TMEM receives
// its 128 rows of D for all N columns.  Rank 0 of the pair issues the MMAs
// and commits; shared-memory descriptors and TMEM addresses name the same
// offsets in both CTAs.

__device__ __forceinline__ uint32_t cluster_id_x() {
  uint32_t r;
  asm volatile("mov.u32 %0, %%clusterid.x;" : "=r"(r));
  return r;
}
__device__ __forceinline__ uint32_t cluster_count_x() {
  uint32_t r;
  asm volatile("mov.u32 %0, %%nclusterid.x;" : "=r"(r));
  return r;
}

// Both CTAs' same warp calls these (paired allocation of the same columns).
__device__ __forceinline__ void tmem_alloc_pair(uint32_t* dst_smem, uint32_t ncols) {
  asm volatile("tcgen05.alloc.cta_group::2.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                   smem_u32(dst_smem)),
               "r"(ncols)
               : "memory");
}
__device__ __forceinline__ void tmem_relinquish_pair() {
  asm volatile("tcgen05.relinquish_alloc_permit.cta_group::2.sync.aligned;" ::: "memory");
}
__device__ __forceinline__ void tmem_dealloc_pair(uint32_t taddr, uint32_t ncols) {
  asm volatile("tcgen05.dealloc.cta_group::2.sync.aligned.b32 %0, %1;" ::"r"(taddr), "r"(ncols)
               : "memory");
}

// D[tmem] (+)= A * B^T over the pair, issued by one thread of rank 0.
__device__ __forceinline__ void mma_f16_pair(uint32_t d_tmem, uint64_t a_desc, uint64_t b_desc,
                                             uint32_t idesc, uint32_t accumulate) {
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::2.kind::f16 [%0], %1, %2, %3, p;\n\t}" ::"r"(d_tmem),
      "l"(a_desc), "l"(b_desc), "r"(idesc), "r"(accumulate)
      : "memory");
}

// Arrive once on the mbarrier at offset `bar` in every CTA of `mask` when all
// previously issued pair MMAs of this thread finish.
__device__ __forceinline__ void mma_commit_pair(uint64_t* bar, uint16_t mask) {
  asm volatile(
      "tcgen05.commit.cta_group::2.mbarrier::arrive::one.shared::cluster.multicast::cluster.b64 "
      "[%0], %1;" ::"r"(smem_u32(bar)),
      "h"(mask)
      : "memory");
}

// ------------------------------------------------------------ misc helpers -
__device__ __forceinline__ uint32_t lane_id() { return threadIdx.x & 31; }
__device__ __forceinline__ uint32_t warp_id() { return threadIdx.x >> 5; }

__device__ __forceinline__ bool elect_one() {
  uint32_t pred = 0;
  asm volatile(
      "{\n\t.reg .b32 rx;\n\t.reg .pred px;\n\t"
      "elect.sync rx|px, 0xffffffff;\n\t"
      "selp.b32 %0, 1, 0, px;\n\t}"
      : "=r"(pred));
  return pred != 0;
}

__device__ __forceinline__ void st_shared_v4(uint32_t addr, uint32_t a, uint32_t b, uint32_t c,
                                             uint32_t d) {
  asm volatile("st.shared.v4.b32 [%0], {%1, %2, %3, %4};" ::"r"(addr), "r"(a), "r"(b), "r"(c),
               "r"(d)
               : "memory");
}

// 32-byte store of eight 32-bit words (dst 32-byte aligned).
__device__ __forceinline__ void st_global_v8(void* dst, const uint32_t* v) {
  asm volatile("st.global.v8.b32 [%0], {%1, %2, %3, %4, %5, %6, %7, %8};" ::"l"(dst), "r"(v[0]), "r"(v[1]),
               "r"(v[2]), "r"(v[3]), "r"(v[4]), "r"(v[5]), "r"(v[6]), "r"(v[7])
               : "memory");
}

// Bring the 128-byte line holding `p` into L1 ahead of its use.
__device__ __forceinline__ void prefetch_l1(const void* p) {
  asm volatile("prefetch.global.L1 [%0];" ::"l"(p));
}

// Make generic-proxy shared-memory writes visible to the async proxy
// (tensor core reads of operands written by ordinary stores).
__device__ __forceinline__ void fence_proxy_async_shared() {
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

// Per-warpgroup register limits (all 128 threads of the warpgroup execute
// it).  An increase waits until other warpgroups have released enough of
// the registers the block was launched with, so the limits of all
// warpgroups must add up to no more than that.
template <uint32_t N>
__device__ __forceinline__ void regs_inc() {
  static_assert(N % 8 == 0 && N >= 24 && N <= 256, "register limit");
  asm volatile("setmaxnreg.inc.sync.aligned.u32 %0;" ::"n"(N));
}
template <uint32_t N>
__device__ __forceinline__ void regs_dec() {
  static_assert(N % 8 == 0 && N >= 24 && N <= 256, "register limit");
  asm volatile("setmaxnreg.dec.sync.aligned.u32 %0;" ::"n"(N));
}

}  // namespace wino
