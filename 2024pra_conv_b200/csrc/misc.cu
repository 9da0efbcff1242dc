// Small kernels shared by the drop-in ABI.
#include <cuda_runtime.h>
#include "wino_param.h"

namespace wino {

// Empty kernel for the unused launch slots: the reference harness launches
// all four slots unconditionally (reference src/main.cpp:105-108, 121-124).
__global__ void noop_kernel(KernelParam) {}

}  // namespace wino

extern "C" void* wino_noop_kernel_ptr() { return (void*)wino::noop_kernel; }
