// Thin C-ABI wrapper around the reference's own CPU convolution,
// conv2dcpu() from include/verfiy.h:5-43, compiled UNMODIFIED from the
// reference tree (the header is found through -I; it is never copied here).
//
// TEST INFRASTRUCTURE ONLY: used to pin the oracle and as the timed CPU
// baseline.  The product path never loads the library this file builds.
//
// ref_conv2dcpu      -- calls conv2dcpu exactly as the reference harness does
//                       (src/main.cpp:138): one call, one thread.
// ref_conv2dcpu_omp  -- the same unmodified function called once per image
//                       (n = 1 slices, pointer offsets of c*h*w and k*oh*ow)
//                       from an OpenMP loop, to use every host core.
#include <cstddef>
#include <cstdint>
#include <omp.h>
#include "verfiy.h"

extern "C" {

void ref_conv2dcpu(uint16_t *pin, uint16_t *pwei, uint16_t *pout,
                   int n, int c, int h, int w, int k, int r, int s,
                   int u, int v, int p, int q)
{
    conv2dcpu(reinterpret_cast<_Float16 *>(pin), reinterpret_cast<_Float16 *>(pwei),
              reinterpret_cast<_Float16 *>(pout), n, c, h, w, k, r, s, u, v, p, q);
}

void ref_conv2dcpu_omp(uint16_t *pin, uint16_t *pwei, uint16_t *pout,
                       int n, int c, int h, int w, int k, int r, int s,
                       int u, int v, int p, int q, int threads)
{
    const int oh = (h + 2 * p - r) / u + 1;
    const int ow = (w + 2 * q - s) / v + 1;
    if (threads > 0) omp_set_num_threads(threads);
#pragma omp parallel for schedule(dynamic, 1)
    for (int i = 0; i < n; i++) {
        conv2dcpu(reinterpret_cast<_Float16 *>(pin) + (size_t)i * c * h * w,
                  reinterpret_cast<_Float16 *>(pwei),
                  reinterpret_cast<_Float16 *>(pout) + (size_t)i * k * oh * ow,
                  1, c, h, w, k, r, s, u, v, p, q);
    }
}

int ref_max_threads(void) { return omp_get_max_threads(); }

}  // extern "C"
