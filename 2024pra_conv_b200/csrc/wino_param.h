// Device-side view of the kernel argument.
//
// Layout-identical mirror of mykernelParamType (include/mykernelParamType.cuh,
// itself the reference's src/mykernelParamType.cuh:5-26) with untyped
// pointers: nvcc's device pass cannot compile `_Float16`, so kernels take this
// struct and cast the pointers to __half.  wino_abi.cpp checks sizeof and
// every offsetof against the host declaration.
#pragma once
#include <cstddef>
#include <cstdint>

namespace wino {

struct KernelParam {
  void* pin;               // input, NCHW fp16
  void* pweight;           // weights, KCRS fp16
  void* pout;              // output, N K Oh Ow fp16
  void* transform_pin;     // workspace: V (unfused path)
  void* transform_filter;  // workspace: U cache
  void* mid_result;        // workspace: M (unfused path)
  short n, c, h, w, k, r, s, u, v, p, q, Oh, Ow;
};

static_assert(sizeof(KernelParam) == 80, "KernelParam must stay 80 bytes");
static_assert(offsetof(KernelParam, n) == 48, "dims start after six pointers");
static_assert(offsetof(KernelParam, Ow) == 72, "thirteen shorts");

}  // namespace wino
