/*
 * Drop-in launch interface of the 3x3 fp16 conv2d operator.
 *
 * Same declarations as the contest plugin ABI the reference implements
 * (reference include/conv2d.h:8-70): identical type names, field names,
 * field order and field types, and the two entry points with C++ linkage,
 * so a caller written against that header (for example the reference's
 * src/main.cpp) compiles and links against this library unchanged.
 * C-linkage aliases with the same signatures are provided for FFI callers.
 *
 * Data layouts (reference readme.txt:21-24): input NCHW, weights KCRS,
 * output N K Oh Ow, all fp16.  Oh = (h - r + 2p)/u + 1, Ow = (w - s + 2q)/v + 1.
 *
 * Contract of this implementation (sm_100a):
 *   - every dim >= 1 and <= 32767 (the `short` fields of mykernelParamType),
 *     a filter no larger than the padded input, non-null in / weight / out;
 *     anything else returns an error code instead of the reference's silent
 *     mis-dispatch outside its six hard-coded shapes;
 *   - the caller owns every buffer: in, weight, out and the three
 *     workspaces sized as the reference harness sizes them
 *     (src/main.cpp:36-38): transform_pin >= 4*h*h*n*c, mid_result >=
 *     4*k*h*w*n and transform_filter >= 16*k*c fp16 elements;
 *   - getkernelInfo fills four launch slots that the caller launches in
 *     order on one stream, each with args[0] pointing at `param`.  Which
 *     kernels go in the slots depends on the shape and on which workspaces
 *     are usable (wino_dropin_route in winoconv.h reports the choice):
 *
 *     two-stage route: r = s = 3, u = v = 1, p = q = 1, c % 16 == k % 16
 *       == 0, even h and w, all three workspaces present, transform_pin
 *       16-byte aligned and large enough for the pre-pass output:
 *         slot 1  filter transform   weight -> transform_filter (U)
 *         slot 2  input pre-pass     in -> transform_pin (c <= 256: the
 *                                    transformed tiles V, 16*c*tiles rounded
 *                                    up to 8 tiles; c > 256: the
 *                                    channel-blocked input)
 *         slot 3  tap GEMMs          transform_pin, transform_filter ->
 *                                    mid_result (M, 16*k*n*(h/2)*(w/2) fp16,
 *                                    all of the caller's 4*k*h*w*n)
 *         slot 4  output transform   mid_result -> out
 *       All three workspaces are written, as the reference's own pipeline
 *       writes them.
 *     fused route with re-layout: the Winograd shape contract holds and
 *       transform_pin is usable, but h or w is odd or mid_result is null:
 *         slot 1  weight -> transform_filter (U); slot 2 in -> transform_pin;
 *         slot 3  fused input transform + tensor-core GEMM + output
 *                 transform -> out;  slot 4  empty kernel.
 *       mid_result is left untouched.
 *     fused route: as above without a usable transform_pin (null, not
 *       16-byte aligned or too small): slot 2 is an empty kernel and the
 *       fused kernel reads `in` directly; transform_pin and mid_result are
 *       left untouched.
 *     implicit-GEMM route: any other shape (filter size, stride, padding,
 *       channel counts not multiples of 16) whose re-laid-out weights,
 *       r*s*ceil(c/16)*round16(k) rows of 32 bytes, fit transform_filter
 *       (non-null, 16-byte aligned): slot 1 weight -> transform_filter in the
 *       tensor-core operand layout; slot 3 tcgen05 implicit GEMM reading `in`
 *       directly -> out (fp32 accumulation); slots 2, 4 empty kernels;
 *       mid_result is left untouched, and so is transform_pin except for
 *       1x1 / stride 1 / pad 0 layers with h*w % 64 == 0 and k > 128, whose
 *       first 128 bytes receive the input's TMA tensor map (written by
 *       getkernelInfo itself with a synchronous copy, so no kernel still
 *       using transform_pin may be in flight on another stream then;
 *       transform_pin 128-byte aligned, else those layers read the input
 *       without TMA).
 *     direct route: the remaining shapes (e.g. c = 3 with a 7x7 filter) or a
 *       null transform_filter: slot 3 is a direct convolution on CUDA cores
 *       (fp32 accumulation), slots 1, 2, 4 empty kernels; no workspace is
 *       touched.
 *   - return value 0 on success, non-zero (a WINO_E* code from winoconv.h)
 *     for unsupported shapes, null pointers or a CUDA attribute failure.
 */
#ifndef WINO_CONV2D_FP16_FWD_HEADER
#define WINO_CONV2D_FP16_FWD_HEADER

#define __in__
#define __out__
#define __in_out__

typedef struct
{
    _Float16*       in;                 /* input,  NCHW, device memory            */
    _Float16*       weight;             /* weights, KCRS, device memory           */
    _Float16*       out;                /* output, N K Oh Ow, device memory       */
    _Float16*       transform_pin;      /* workspace: pre-pass output (V, input) */
    _Float16*       transform_filter;   /* workspace: U, or the igemm weights     */
    _Float16*       mid_result;         /* workspace: tap GEMM output M           */
    unsigned int    n;                  /* batch size                             */
    unsigned int    c;                  /* input channels                         */
    unsigned int    h;                  /* input height                           */
    unsigned int    w;                  /* input width                            */
    unsigned int    k;                  /* output channels (filters)              */
    unsigned int    r;                  /* filter height                          */
    unsigned int    s;                  /* filter width                           */
    unsigned int    u;                  /* vertical stride                        */
    unsigned int    v;                  /* horizontal stride                      */
    unsigned int    p;                  /* vertical padding                       */
    unsigned int    q;                  /* horizontal padding                     */
} problem_t;

typedef struct
{
    unsigned int    blockx1;            /* slot 1: grid x, y, z                   */
    unsigned int    blocky1;
    unsigned int    blockz1;
    unsigned int    threadx1;           /* slot 1: block x, y, z                  */
    unsigned int    thready1;
    unsigned int    threadz1;
    unsigned int    dynmicLdsSize1;     /* slot 1: dynamic shared memory (bytes)  */
    void*           kernelPtr1;         /* slot 1: kernel entry (cudaLaunchKernel) */

    unsigned int    blockx2;
    unsigned int    blocky2;
    unsigned int    blockz2;
    unsigned int    threadx2;
    unsigned int    thready2;
    unsigned int    threadz2;
    unsigned int    dynmicLdsSize2;
    void*           kernelPtr2;

    unsigned int    blockx3;
    unsigned int    blocky3;
    unsigned int    blockz3;
    unsigned int    threadx3;
    unsigned int    thready3;
    unsigned int    threadz3;
    unsigned int    dynmicLdsSize3;
    void*           kernelPtr3;

    unsigned int    blockx4;
    unsigned int    blocky4;
    unsigned int    blockz4;
    unsigned int    threadx4;
    unsigned int    thready4;
    unsigned int    threadz4;
    unsigned int    dynmicLdsSize4;
    void*           kernelPtr4;
} kernelInfo_t;

#ifdef __cplusplus
/* Reference: src/conv2d.cpp:9-14.  *paramSize = sizeof(mykernelParamType). */
int getParamsize(__in__ problem_t* problem, __out__ int* paramSize);
/* Reference: src/conv2d.cpp:254-517.  Fills the four slots and `param`. */
int getkernelInfo(__in__ problem_t* problem, __out__ kernelInfo_t* kernelInfo,
                  __in_out__ void* param);
extern "C" {
#endif

/* C-linkage aliases of the two entry points above (same behaviour). */
int wino_getParamsize(problem_t* problem, int* paramSize);
int wino_getkernelInfo(problem_t* problem, kernelInfo_t* kernelInfo, void* param);

#ifdef __cplusplus
}
#endif

#endif /* WINO_CONV2D_FP16_FWD_HEADER */
