// Conv entry point for callers that cannot allocate device memory.
//
// The regular paths need a caller-provided U cache (the transformed filter,
// 16*K*C fp16) in addition to the input and output.  Some callers have no way
// to provide one: plugin hosts that hand the operator only its input and
// output tensors and forbid allocations inside the call, runtimes whose
// device memory is carved up once at start-up, or code paths that must not
// touch the allocator while other work is being recorded.  For them this file
// keeps the U cache in a fixed, file-scope device array and runs the same two
// kernels as the regular path (filter transform, then the fused conv) on it.
//
// Limits and behaviour:
//   * capacity: K * C <= kNoAllocMaxKC (a 512 x 512 filter bank), i.e. 8 MiB
//     of fp16; every GPU that loads the library holds this array until the
//     process exits.  Larger filters are rejected with WINO_ESCRATCH before
//     anything is launched;
//   * every call looks up the array's device address on the current device
//     (cudaGetSymbolAddress, with that device current) and checks the result;
//     nothing is cached, so the address stays right after a cudaDeviceReset.
//     The first call on a device may also load the library's kernels onto it:
//     make that first call before any stream capture starts on that device;
//   * every call, on every stream, uses the same array and leaves the last
//     call's U in it.  Each call rewrites the whole part it reads, so nothing
//     needs to start at zero, but calls whose kernels overlap on the GPU race
//     on the array: serialise them (one stream, or events between streams);
//   * no cudaMalloc, cudaFree or allocating library routine is called.
#include <cuda_runtime.h>

#include "winoconv.h"
#include "wino_param.h"

namespace {

constexpr long long kNoAllocMaxKC = 512LL * 512LL;
constexpr size_t kNoAllocElems = 16 * (size_t)kNoAllocMaxKC;  // fp16 elements

// The scratch itself.  In host code this name is only a handle for the
// runtime; the device address comes from cudaGetSymbolAddress below.
static __device__ __align__(256) unsigned short g_noalloc_ucache[kNoAllocElems];

// Device address of the scratch on the current device.  Looked up on every
// call (the lookup is a host-side table read): a cached address would go stale
// when the caller resets the device.
int scratch_address(void** out) {
  void* p = nullptr;
  if (cudaGetSymbolAddress(&p, g_noalloc_ucache) != cudaSuccess || !p) return WINO_ECUDA;
  *out = p;
  return WINO_OK;
}

}  // namespace

extern "C" {
int wino_launch_filter_transform(const void* weight, void* ucache, void* ucache_lo, int K, int C,
                                 int bf16, int layout, cudaStream_t stream);
void* wino_fused_kernel_ptr();
int wino_fused_prepare();
int wino_fused_smem_bytes();
int wino_fused_threads();
long long wino_fused_nblocks(int n, int h, int w, int k);

long long wino_noalloc_max_kc() { return kNoAllocMaxKC; }

int wino_conv2d_noalloc(const void* x, const void* weight, void* y, int n, int c, int h, int w,
                        int k, void* stream) {
  if (!x || !weight || !y) return WINO_EINVAL;
  const int st = wino_check_shape(n, c, h, w, k);
  if (st != WINO_OK) return st;
  if ((long long)k * c > kNoAllocMaxKC) return WINO_ESCRATCH;
  void* ucache = nullptr;
  if (scratch_address(&ucache) != WINO_OK) return WINO_ECUDA;
  const cudaStream_t s = static_cast<cudaStream_t>(stream);
  if (wino_launch_filter_transform(weight, ucache, nullptr, k, c, 0, 0, s) != 0) return WINO_ECUDA;
  if (wino_fused_prepare() != 0) return WINO_ECUDA;

  wino::KernelParam p;
  p.pin = const_cast<void*>(x);
  p.pweight = const_cast<void*>(weight);
  p.pout = y;
  p.transform_pin = nullptr;
  p.transform_filter = ucache;
  p.mid_result = nullptr;
  p.n = (short)n; p.c = (short)c; p.h = (short)h; p.w = (short)w; p.k = (short)k;
  p.r = 3; p.s = 3; p.u = 1; p.v = 1; p.p = 1; p.q = 1;
  p.Oh = (short)h; p.Ow = (short)w;

  int dev = 0, sms = 148;
  if (cudaGetDevice(&dev) == cudaSuccess)
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  const long long nb = wino_fused_nblocks(n, h, w, k);
  const unsigned grid = (unsigned)(nb < sms ? nb : sms);
  void* args[] = {&p};
  const cudaError_t e = cudaLaunchKernel(wino_fused_kernel_ptr(), dim3(grid),
                                         dim3(wino_fused_threads()), args,
                                         (size_t)wino_fused_smem_bytes(), s);
  return e == cudaSuccess ? WINO_OK : WINO_ECUDA;
}

}  // extern "C"
