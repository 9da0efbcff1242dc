// Drop-in demo: a C++ caller written only against include/conv2d.h, doing
// what the reference's harness does with its plugin (allocate the device
// buffers and workspaces at the harness's sizes, getParamsize, getkernelInfo,
// launch the four slots with args[0] = param, time 100 iterations; reference
// src/main.cpp:33-131) -- with cudaLaunchKernel in place of the HIP launch.
//
//   conv2ddemo [n c h w k]        (default: 8 64 32 32 64)
//
// It then checks sampled outputs against a double-precision direct
// convolution computed here (relative error <= 1e-2 each, the harness's own
// 1 % rule), prints one line and exits 0 on success.
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <vector>
#include <cuda_runtime.h>

#include "conv2d.h"

namespace {

#define CHECK(x)                                                                      \
  do {                                                                                \
    cudaError_t e_ = (x);                                                             \
    if (e_ != cudaSuccess) {                                                          \
      std::fprintf(stderr, "%s failed: %s\n", #x, cudaGetErrorString(e_));            \
      std::exit(2);                                                                   \
    }                                                                                 \
  } while (0)

// Deterministic values in [0, 1) (the harness draws (rand() % 255) / 255).
struct Lcg {
  uint64_t s;
  uint64_t raw() {
    s = s * 6364136223846793005ull + 1442695040888963407ull;
    return s >> 33;
  }
  double next() { return (double)(raw() % 255) / 255.0; }
};

}  // namespace

int main(int argc, char** argv) {
  int n = 8, c = 64, h = 32, w = 32, k = 64;
  if (argc == 6) {
    n = std::atoi(argv[1]); c = std::atoi(argv[2]); h = std::atoi(argv[3]);
    w = std::atoi(argv[4]); k = std::atoi(argv[5]);
  }
  const int r = 3, s = 3, u = 1, v = 1, p = 1, q = 1;
  const int oh = (h - r + 2 * p) / u + 1, ow = (w - s + 2 * q) / v + 1;
  const size_t nin = (size_t)n * c * h * w, nw = (size_t)k * c * r * s, nout = (size_t)n * k * oh * ow;

  std::vector<_Float16> xin(nin), wt(nw), out(nout);
  Lcg g{12345};
  for (auto& e : xin) e = (_Float16)g.next();
  for (auto& e : wt) e = (_Float16)(g.next() - 0.5);

  _Float16 *d_in, *d_w, *d_out, *d_mid, *d_tpin, *d_tfil;
  CHECK(cudaMalloc(&d_in, nin * 2));
  CHECK(cudaMalloc(&d_w, nw * 2));
  CHECK(cudaMalloc(&d_out, nout * 2));
  CHECK(cudaMalloc(&d_mid, (size_t)4 * k * h * w * n * 2));    // harness sizes
  CHECK(cudaMalloc(&d_tpin, (size_t)4 * h * h * n * c * 2));
  CHECK(cudaMalloc(&d_tfil, (size_t)k * c * 16 * 2));
  CHECK(cudaMemcpy(d_in, xin.data(), nin * 2, cudaMemcpyHostToDevice));
  CHECK(cudaMemcpy(d_w, wt.data(), nw * 2, cudaMemcpyHostToDevice));

  problem_t pr;
  pr.in = d_in; pr.weight = d_w; pr.out = d_out;
  pr.transform_pin = d_tpin; pr.transform_filter = d_tfil; pr.mid_result = d_mid;
  pr.n = n; pr.c = c; pr.h = h; pr.w = w; pr.k = k;
  pr.r = r; pr.s = s; pr.u = u; pr.v = v; pr.p = p; pr.q = q;

  int psize = 0;
  if (getParamsize(&pr, &psize) != 0) return 3;
  void* param = std::malloc(psize);
  kernelInfo_t ki;
  const int rc = getkernelInfo(&pr, &ki, param);
  if (rc != 0) {
    std::printf("getkernelInfo rejected the problem: %d\n", rc);
    return 4;
  }
  auto launch_all = [&]() {
    const unsigned* slot[4] = {&ki.blockx1, &ki.blockx2, &ki.blockx3, &ki.blockx4};
    void* fn[4] = {ki.kernelPtr1, ki.kernelPtr2, ki.kernelPtr3, ki.kernelPtr4};
    for (int i = 0; i < 4; ++i) {
      const unsigned* b = slot[i];
      CHECK(cudaLaunchKernel(fn[i], dim3(b[0], b[1], b[2]), dim3(b[3], b[4], b[5]), (void**)&param,
                             (size_t)b[6], 0));
    }
  };
  launch_all();
  CHECK(cudaDeviceSynchronize());
  CHECK(cudaMemcpy(out.data(), d_out, nout * 2, cudaMemcpyDeviceToHost));

  cudaEvent_t a, b;
  CHECK(cudaEventCreate(&a));
  CHECK(cudaEventCreate(&b));
  const int iters = 100;
  CHECK(cudaEventRecord(a, 0));
  for (int i = 0; i < iters; ++i) launch_all();
  CHECK(cudaEventRecord(b, 0));
  CHECK(cudaEventSynchronize(b));
  float ms = 0.f;
  CHECK(cudaEventElapsedTime(&ms, a, b));

  // sampled check against a double-precision direct convolution
  int bad = 0, checked = 0;
  Lcg pick{777};
  for (int t = 0; t < 512; ++t) {
    const size_t o = (size_t)(pick.raw() % nout);
    const int ox = (int)(o % ow), oy = (int)((o / ow) % oh), kk = (int)((o / ((size_t)ow * oh)) % k);
    const int nn = (int)(o / ((size_t)ow * oh * k));
    double acc = 0.0;
    for (int cc = 0; cc < c; ++cc)
      for (int i = 0; i < r; ++i)
        for (int j = 0; j < s; ++j) {
          const int y = oy * u - p + i, x = ox * v - q + j;
          if (y < 0 || y >= h || x < 0 || x >= w) continue;
          acc += (double)xin[(((size_t)nn * c + cc) * h + y) * w + x] *
                 (double)wt[(((size_t)kk * c + cc) * r + i) * s + j];
        }
    const double got = (double)out[o];
    if (std::fabs(got - acc) > 1e-2 * std::fabs(acc) + 1e-2) ++bad;
    ++checked;
  }
  std::printf("{\"n\": %d, \"c\": %d, \"h\": %d, \"w\": %d, \"k\": %d, \"paramsize\": %d, "
              "\"us_per_iter\": %.2f, \"checked\": %d, \"error\": %d}\n",
              n, c, h, w, k, psize, ms * 1000.f / iters, checked, bad);
  std::free(param);
  cudaFree(d_in); cudaFree(d_w); cudaFree(d_out); cudaFree(d_mid); cudaFree(d_tpin); cudaFree(d_tfil);
  return bad == 0 ? 0 : 1;
}
