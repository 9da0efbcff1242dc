/*
 * Kernel argument passed by value to every kernel getkernelInfo returns.
 *
 * Same layout as the reference's src/mykernelParamType.cuh:5-26 (six fp16
 * pointers followed by thirteen `short` dimensions, 80 bytes on x86-64), so
 * that getParamsize() reports the size a reference caller expects and the
 * caller's malloc(paramSize) buffer holds it.  The dims are `short` there and
 * here, which caps every dimension at 32767; getkernelInfo rejects larger
 * problems.
 *
 * Device code does not see this declaration: nvcc's device pass cannot
 * compile `_Float16`, so kernels take wino::KernelParam (csrc/wino_param.h),
 * a layout-identical mirror whose equality with this struct is checked by
 * static_assert in the host translation unit that fills it.
 */
#ifndef WINO_MYKERNELPARAMTYPE_H
#define WINO_MYKERNELPARAMTYPE_H

typedef struct mykernelParamType
{
    _Float16* __restrict__ pin;                /* input, NCHW               */
    _Float16* __restrict__ pweight;            /* weights, KCRS             */
    _Float16* __restrict__ pout;               /* output, N K Oh Ow         */
    _Float16* __restrict__ transform_pin;      /* workspace                 */
    _Float16* __restrict__ transform_filter;   /* workspace: U cache        */
    _Float16* __restrict__ mid_result;         /* workspace                 */
    short      n;                              /* batch size                */
    short      c;                              /* input channels            */
    short      h;                              /* input height              */
    short      w;                              /* input width               */
    short      k;                              /* output channels           */
    short      r;                              /* filter height             */
    short      s;                              /* filter width              */
    short      u;                              /* vertical stride           */
    short      v;                              /* horizontal stride         */
    short      p;                              /* vertical padding          */
    short      q;                              /* horizontal padding        */
    short      Oh;                             /* output height             */
    short      Ow;                             /* output width              */
} mykernelParamType;

#endif /* WINO_MYKERNELPARAMTYPE_H */
