/*
 * FP64 direct-convolution oracle.  TEST INFRASTRUCTURE ONLY: nothing on the
 * product path links, loads or calls this file.  Only tests/, the smoke check
 * in __graft_entry__.py and bench.py's CPU-baseline leg use it, as a checker.
 *
 * Restates conv2dcpu() of the reference (include/verfiy.h:5-43):
 *   - output size  oh = (h + 2p - r)/u + 1, ow = (w + 2q - s)/v + 1   (verfiy.h:7-8)
 *   - loop order n, k, oh, ow, then c, kh, kw with the in-bounds test
 *     (verfiy.h:10-36) so that the double sum is formed in the same order;
 *   - one difference on purpose: every product is formed as
 *     (double)in * (double)w.  The reference writes (double)(in*w) with
 *     _Float16 operands; with exact float evaluation (the default on x86-64
 *     without AVX512-FP16) that is the same number, because an fp16 x fp16
 *     product has at most 22 significant bits.  On hosts with native fp16
 *     arithmetic the reference rounds each product to fp16 first; this oracle
 *     never does.
 *   - the result is kept in double (no fp16 store, unlike verfiy.h:38) so
 *     that error metrics are taken against the exact-product FP64 value.
 *
 * Inputs are float arrays holding fp16 values exactly (the caller widens the
 * fp16 bits), outputs double.  Images are split over OpenMP threads; each
 * output element is still summed by one thread in the reference order.
 */
#include <stddef.h>

void oracle_conv2d_f64(const float *pin, const float *pwei, double *pout,
                       int n, int c, int h, int w, int k, int r, int s,
                       int u, int v, int p, int q)
{
    const int oh = (h + 2 * p - r) / u + 1;
    const int ow = (w + 2 * q - s) / v + 1;
    const long long nk = (long long)n * k;

#pragma omp parallel for schedule(dynamic, 1)
    for (long long nkIdx = 0; nkIdx < nk; nkIdx++) {
        const int nNum = (int)(nkIdx / k);
        const int kNum = (int)(nkIdx % k);
        const float *img = pin + (size_t)nNum * c * h * w;
        const float *flt = pwei + (size_t)kNum * c * r * s;
        double *dst = pout + ((size_t)nNum * k + kNum) * oh * ow;
        for (int i = 0; i < oh; i++) {
            for (int j = 0; j < ow; j++) {
                double sum = 0.0;
                const int posh = i * u - p;
                const int posw = j * v - q;
                for (int cNum = 0; cNum < c; cNum++) {
                    for (int kh = 0; kh < r; kh++) {
                        for (int kw = 0; kw < s; kw++) {
                            const int y = posh + kh;
                            const int x = posw + kw;
                            if (x >= 0 && y >= 0 && x < w && y < h) {
                                sum += (double)img[(size_t)cNum * h * w + (size_t)y * w + x] *
                                       (double)flt[(size_t)cNum * r * s + kh * s + kw];
                            }
                        }
                    }
                }
                dst[(size_t)i * ow + j] = sum;
            }
        }
    }
}
