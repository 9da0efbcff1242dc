// Input re-layout pre-pass for the fused kernel: NCHW fp16 -> XB records
// (layout described in vgen.cuh), zero outside the image.  For the fp8
// variant a second instantiation also records the per-channel max |x| into
// p.mid_result (the plain one never touches that field, which in the
// drop-in parameter struct is the caller's workspace).
//
// The reference's pipeline also writes an intermediate form of the input into
// the caller's `transform_pin` workspace before its GEMMs (the transformed
// tiles V, 4x the input, src/preprocessing.cuh:273-424 writing
// transform_pin); here that workspace receives the same-size channel-blocked
// copy of the input and the transform itself happens on chip.
//
// One thread per (record row, entry e): it reads columns 2e and 2e+1 of the
// row for all 16 channels (one 4-byte load per channel when W is even) and
// writes par-0 entry e (column 2e) and par-1 entry e+1 (column 2e+1) of the
// two channel halves; the thread of the last entry also writes the par-1
// entry 0 (column -1, zero).  Consecutive threads read consecutive words of
// each channel row and write consecutive 16-byte words of each (par, half)
// run.  HBM-bound; items are counted in 32 bits (the host
// checks N*(C/16)*rows*entries < 2^31).
#include <cuda_runtime.h>
#include <cuda_fp16.h>
#include "wino_param.h"
#include "vgen.cuh"

namespace wino {

template <bool AMAX>
__global__ void __launch_bounds__(256) xb_layout_kernel(KernelParam p) {
  const int C = p.c, H = p.h, W = p.w;
  const int CB = C >> 4, HP = xb_rows(H), E = xb_entries(W);
  const uint32_t items = (uint32_t)p.n * CB * HP * E;
  const unsigned short* X = static_cast<const unsigned short*>(p.pin);
  uint4* XB = static_cast<uint4*>(p.transform_pin);
  const size_t plane = (size_t)H * W;
  const bool w_even = (W & 1) == 0;
  // optional (fp8 variant): per-channel max |x| as fp16 magnitude bits
  unsigned* amax = AMAX ? static_cast<unsigned*>(p.mid_result) : nullptr;
  for (uint32_t it = blockIdx.x * blockDim.x + threadIdx.x; it < items; it += gridDim.x * blockDim.x) {
    const uint32_t rec = it / E;
    const int e = (int)(it - rec * E);
    const int r = (int)(rec % HP);
    const uint32_t ncb = rec / HP;
    const int cb = (int)(ncb % CB);
    const int n = (int)(ncb / CB);
    const int y = r - 1;
    const int x0 = 2 * e;                         // columns x0 (par 0) and x0 + 1 (par 1)
    const bool ok0 = y >= 0 && y < H && x0 < W;
    const bool ok1 = y >= 0 && y < H && x0 + 1 < W;
    uint32_t lo[16], hi[16];                      // column x0 / x0+1 of channel 16cb + i
    const unsigned short* src = X + ((size_t)n * C + 16 * cb) * plane + (size_t)(y < 0 ? 0 : y) * W + x0;
    if (w_even && ok1) {
#pragma unroll
      for (int i = 0; i < 16; ++i) {
        const uint32_t v = *reinterpret_cast<const uint32_t*>(src + i * plane);
        lo[i] = v & 0xffffu;
        hi[i] = v >> 16;
      }
    } else {
#pragma unroll
      for (int i = 0; i < 16; ++i) {
        lo[i] = ok0 ? src[i * plane] : 0u;
        hi[i] = ok1 ? src[i * plane + 1] : 0u;
      }
    }
    if (AMAX) {
      // per-channel max |x| (fp16 magnitude bits order like the values):
      // reduced over the warp when all its lanes hold the same channel block
      const unsigned act = __activemask();
      const int cb0 = __shfl_sync(act, cb, __ffs(act) - 1);
      const bool uni = __all_sync(act, cb == cb0);
#pragma unroll
      for (int i = 0; i < 16; ++i) {
        uint32_t m = max(lo[i] & 0x7fffu, hi[i] & 0x7fffu);
        if (uni) {
          m = __reduce_max_sync(act, m);
          if ((int)threadIdx.x % 32 == __ffs(act) - 1 && m) atomicMax(amax + 16 * cb + i, m);
        } else if (m) {
          atomicMax(amax + 16 * cb + i, m);
        }
      }
    }
    uint4* out = XB + (size_t)rec * (4 * E);
#pragma unroll
    for (int hh = 0; hh < 2; ++hh) {
      const uint32_t* l = lo + 8 * hh;
      const uint32_t* u = hi + 8 * hh;
      out[hh * E + e] = make_uint4(l[0] | (l[1] << 16), l[2] | (l[3] << 16), l[4] | (l[5] << 16),
                                   l[6] | (l[7] << 16));
      if (e + 1 < E)
        out[(2 + hh) * E + e + 1] = make_uint4(u[0] | (u[1] << 16), u[2] | (u[3] << 16),
                                               u[4] | (u[5] << 16), u[6] | (u[7] << 16));
      else
        out[(2 + hh) * E] = make_uint4(0u, 0u, 0u, 0u);
    }
  }
}

// fp8 scales from the per-channel input maxima: |V| <= 4 max|x_c| (each
// V element is a signed sum of four inputs), so V / sv[c] with
// sv[c] = 4 max|x_c| / 448 stays inside e4m3's range.  The producers multiply
// by inv = fp16(1 / sv[c]) (clamped to fp16's range), so sv[c] is recorded as
// exactly 1 / inv for folding into U.  One thread per channel pair.
__global__ void xb_f8_scales_kernel(const unsigned* __restrict__ amax, float* __restrict__ sv,
                                    uint32_t* __restrict__ inv_sv2, int C) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (2 * i >= C) return;
  uint32_t packed = 0;
#pragma unroll
  for (int k = 0; k < 2; ++k) {
    const int c = 2 * i + k;
    const unsigned short bits = (unsigned short)amax[c];
    const float a = __half2float(*reinterpret_cast<const __half*>(&bits));
    float inv = a > 0.f ? 448.f / (4.f * a) : 1.f;
    inv = fminf(inv, 65504.f);
    const __half hinv = __float2half_rn(inv);
    sv[c] = 1.f / __half2float(hinv);
    packed |= (uint32_t)(*reinterpret_cast<const unsigned short*>(&hinv)) << (16 * k);
  }
  inv_sv2[i] = packed;
}

}  // namespace wino

using namespace wino;

extern "C" {

void* wino_xb_layout_kernel_ptr() { return (void*)xb_layout_kernel<false>; }

size_t wino_xb_bytes(int n, int c, int h, int w) { return xb_bytes(n, c, h, w); }

// Items of the pre-pass (one per record row and entry); the kernel counts
// them in 32 bits.
long long wino_xb_items(int n, int c, int h, int w) {
  return (long long)n * (c >> 4) * xb_rows(h) * xb_entries(w);
}

// Grid of the pre-pass: 256-thread CTAs over the items, capped (the kernel strides).
unsigned wino_xb_layout_grid(int n, int c, int h, int w) {
  const long long blocks = (wino_xb_items(n, c, h, w) + 255) / 256;
  const long long cap = 148LL * 64;
  return (unsigned)(blocks < cap ? (blocks > 0 ? blocks : 1) : cap);
}

int wino_launch_xb_f8_scales(const unsigned* amax, float* sv, uint32_t* inv_sv2, int C,
                             cudaStream_t stream) {
  xb_f8_scales_kernel<<<(C / 2 + 127) / 128, 128, 0, stream>>>(amax, sv, inv_sv2, C);
  return (int)cudaGetLastError();
}

int wino_launch_xb_layout(const KernelParam* p, cudaStream_t stream) {
  void* args[] = {const_cast<KernelParam*>(p)};
  return (int)cudaLaunchKernel((void*)xb_layout_kernel<false>,
                               dim3(wino_xb_layout_grid(p->n, p->c, p->h, p->w)), dim3(256), args, 0, stream);
}

// The fp8 variant's pre-pass: also the per-channel max |x| into p->mid_result
// (C unsigned words, zeroed by the caller).
int wino_launch_xb_layout_amax(const KernelParam* p, cudaStream_t stream) {
  void* args[] = {const_cast<KernelParam*>(p)};
  return (int)cudaLaunchKernel((void*)xb_layout_kernel<true>,
                               dim3(wino_xb_layout_grid(p->n, p->c, p->h, p->w)), dim3(256), args, 0, stream);
}

}  // extern "C"
