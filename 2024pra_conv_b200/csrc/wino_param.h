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

// Extra arguments of the non-drop-in fused kernels (zero = unused).
struct VariantArgs {
  const void* u_lo;          // VAR_F16_HILO: residual U cache (fp16, same layout)
  const float* su;           // VAR_F8: su[t * K + k]
  const uint32_t* inv_sv2;   // VAR_F8: (1/sv[2i], 1/sv[2i+1]) as fp16x2, i < C/2
  const float* bias;         // epilogue: + bias[k]
  const void* residual;      // epilogue: + residual (fp16, the output's layout; may alias it)
  int relu;                  // epilogue: max(., 0) last
  int pad;
};
static_assert(offsetof(KernelParam, n) == 48, "dims start after six pointers");
static_assert(offsetof(KernelParam, Ow) == 72, "thirteen shorts");

// Arguments of one batched tap GEMM of the unfused layouts (V2 / U2 of
// wino_common.cuh): `taps` taps, `ntb` 128-tile blocks, `c_red` reduction
// channels (a multiple of 16), `k` output channels (a multiple of 16).
struct TapGemm {
  const void* v2;
  const void* u2;
  void* m;                   // M[t][k][tile], tiles padded to ntb * 128
  int taps, ntb, c_red, k;
};

}  // namespace wino

// fp32-M instance of the tap GEMM (unfused_conv.cu), on `sms` persistent CTAs.
extern "C" int wino_tap_gemm_f32_launch(const wino::TapGemm* s, int sms, void* stream);
