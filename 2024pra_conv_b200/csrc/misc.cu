// Small kernels shared by the drop-in ABI, and the self-test of the bounded
// waits.
#include <cuda_runtime.h>
#include "wino_param.h"
#include "tc_sm100.cuh"

namespace wino {

// Empty kernel for the unused launch slots: the reference harness launches
// all four slots unconditionally (reference src/main.cpp:105-108, 121-124).
__global__ void noop_kernel(KernelParam) {}

static __device__ uint32_t g_selftest_err[2];

// Failure-detection self-test: one warp waits (warp-wide, as the producers
// do) and one thread waits (as the MMA thread does) on mbarriers that nothing
// ever arrives on.  Both waits run out after WINO_WAIT_NS, record their code
// in this kernel's own error word and return; the kernel ends normally and
// the context stays usable.  No fault, trap or unbounded wait is involved.
__global__ void wait_timeout_selftest_kernel() {
  __shared__ uint64_t never[2];
  __shared__ int abort_flag;
  if (threadIdx.x == 0) {
    mbar_init(&never[0], 1);
    mbar_init(&never[1], 1);
    abort_flag = 0;
    fence_barrier_init();
  }
  __syncthreads();
  if (threadIdx.x < 32) {
    const bool ok = mbar_wait_warp(&never[0], 0, nullptr, &g_selftest_err[0], ERR_WAIT_FULL, 64);
    if (ok) record_error(&g_selftest_err[0], 0xbad);        // cannot happen: nothing arrives
  } else if (threadIdx.x == 32) {
    const bool ok = mbar_wait(&never[1], 0, &abort_flag, &g_selftest_err[1], ERR_WAIT_EMPTY);
    if (ok) record_error(&g_selftest_err[1], 0xbad);
  }
}

}  // namespace wino

extern "C" void* wino_noop_kernel_ptr() { return (void*)wino::noop_kernel; }

// Runs the self-test kernel and returns the codes its two waits recorded in
// code[0] (warp-wide wait: ERR_WAIT_FULL expected) and code[1] (single-thread
// wait: ERR_WAIT_EMPTY expected); returns a cudaError_t.
extern "C" int wino_selftest_wait_timeout(uint32_t* code) {
  if (!code) return (int)cudaErrorInvalidValue;
  const uint32_t z[2] = {0, 0};
  cudaError_t e = cudaMemcpyToSymbol(wino::g_selftest_err, z, sizeof(z));
  if (e != cudaSuccess) return (int)e;
  wino::wait_timeout_selftest_kernel<<<1, 64>>>();
  e = cudaGetLastError();
  if (e == cudaSuccess) e = cudaDeviceSynchronize();
  if (e == cudaSuccess) e = cudaMemcpyFromSymbol(code, wino::g_selftest_err, 2 * sizeof(uint32_t));
  return (int)e;
}
