"""Python host layer over libwinoconv.so (the B200 Winograd conv2d library).

Import with ``importlib.import_module("2024pra_conv_b200")`` (the directory
name starts with a digit).  Everything here is a thin ctypes veneer over the
C-ABI declared in include/conv2d.h and include/winoconv.h; device memory and
streams come from torch.  There is no CPU path: if the compiled library is
missing, import-time loading raises.

Mirrors of the reference interface (reference include/conv2d.h:8-70):
``Problem`` (problem_t), ``KernelInfo`` (kernelInfo_t), ``get_param_size``
(getParamsize) and ``get_kernel_info`` (getkernelInfo) take the same fields
and return the same codes as the C entry points.
"""
from __future__ import annotations

import ctypes
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "_build", "libwinoconv.so")

# Error codes of include/winoconv.h.
WINO_OK, WINO_EINVAL, WINO_EUNSUPPORTED, WINO_ECUDA, WINO_EDEVICE = 0, 1, 2, 3, 4
WINO_ESCRATCH, WINO_ESTALE, WINO_EIO = 5, 6, 7
VAR_F16, VAR_BF16, VAR_F8, VAR_F16_HILO = 0, 1, 2, 3


class WinoError(RuntimeError):
    def __init__(self, code, what):
        super().__init__(f"{what} failed with code {code}")
        self.code = code


class Problem(ctypes.Structure):
    """problem_t (reference include/conv2d.h:8-27)."""
    _fields_ = [("in_", ctypes.c_void_p), ("weight", ctypes.c_void_p), ("out", ctypes.c_void_p),
                ("transform_pin", ctypes.c_void_p), ("transform_filter", ctypes.c_void_p),
                ("mid_result", ctypes.c_void_p)] + [
        (f, ctypes.c_uint) for f in ("n", "c", "h", "w", "k", "r", "s", "u", "v", "p", "q")]


def _kernel_info_fields():
    out = []
    for i in range(1, 5):
        out += [(f"{f}{i}", ctypes.c_uint) for f in
                ("blockx", "blocky", "blockz", "threadx", "thready", "threadz", "dynmicLdsSize")]
        out.append((f"kernelPtr{i}", ctypes.c_void_p))
    return out


class KernelInfo(ctypes.Structure):
    """kernelInfo_t (reference include/conv2d.h:29-66)."""
    _fields_ = _kernel_info_fields()

    def slot(self, i):
        g = lambda f: getattr(self, f"{f}{i}")
        return dict(grid=(g("blockx"), g("blocky"), g("blockz")),
                    block=(g("threadx"), g("thready"), g("threadz")),
                    lds=g("dynmicLdsSize"), kernel=g("kernelPtr"))


_lib = None


def lib():
    """The loaded library; raises if it has not been built."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise FileNotFoundError(
                f"{LIB_PATH} not built: run `python 2024pra_conv_b200/build.py` "
                "(there is no fallback path)")
        L = ctypes.CDLL(LIB_PATH)
        vp, i, sz = ctypes.c_void_p, ctypes.c_int, ctypes.c_size_t
        sigs = {
            "wino_getParamsize": ([ctypes.POINTER(Problem), ctypes.POINTER(i)], i),
            "wino_getkernelInfo": ([ctypes.POINTER(Problem), ctypes.POINTER(KernelInfo), vp], i),
            "wino_check_shape": ([i, i, i, i, i], i),
            "wino_ucache_bytes": ([i, i, i], sz),
            "wino_filter_transform": ([vp, vp, i, i, vp], i),
            "wino_conv2d_fused": ([vp, vp, vp, i, i, i, i, i, vp], i),
            "wino_fused_workspace_bytes": ([i, i, i, i], sz),
            "wino_input_layout": ([vp, vp, i, i, i, i, vp], i),
            "wino_conv2d_fused_epilogue": ([vp, vp, vp, vp, vp, vp, i, i, i, i, i, i, vp], i),
            "wino_conv2d_direct": ([vp, vp, vp] + [i] * 11 + [vp], i),
            "wino_igemm_weight_bytes": ([i, i, i, i], sz),
            "wino_igemm_weight_transform": ([vp, vp, i, i, i, i, vp], i),
            "wino_conv2d_igemm": ([vp, vp, vp] + [i] * 11 + [vp], i),
            "wino_weight_tag": ([vp, i, i, ctypes.POINTER(ctypes.c_ulonglong), vp], i),
            "wino_ucache_save": ([ctypes.c_char_p, vp, i, i, ctypes.c_ulonglong], i),
            "wino_ucache_load": ([ctypes.c_char_p, vp, i, i, ctypes.c_ulonglong], i),
            "wino_variant_workspace_bytes": ([i, i, i, i, i, i], sz),
            "wino_conv2d_fused_cfg": ([vp, vp, vp, vp, i, i, i, i, i, i, vp], i),
            "wino_fused_cfg_workspace_bytes": ([i, i, i, i, i, i], sz),
            "wino_fused_tune_workspace_bytes": ([i, i, i, i, i], sz),
            "wino_tune_layer": ([vp, vp, vp, vp, i, i, i, i, i, i, ctypes.POINTER(ctypes.c_float),
                                 ctypes.POINTER(i), vp], i),
            "wino_batch_create": ([ctypes.POINTER(vp)], i),
            "wino_batch_destroy": ([vp], i),
            "wino_batch_add_layer": ([vp, vp, vp, vp, vp, i, i, i, i, i], i),
            "wino_batch_num_layers": ([vp], i),
            "wino_batch_set_config": ([vp, i, i], i),
            "wino_batch_get_config": ([vp, i, ctypes.POINTER(i)], i),
            "wino_batch_set_route": ([vp, i, i], i),
            "wino_batch_get_route": ([vp, i, ctypes.POINTER(i), ctypes.POINTER(ctypes.c_float),
                                      ctypes.POINTER(ctypes.c_float)], i),
            "wino_batch_set_order": ([vp, ctypes.POINTER(i), i], i),
            "wino_batch_get_order": ([vp, ctypes.POINTER(i), i], i),
            "wino_batch_commit": ([vp], i),
            "wino_batch_run": ([vp, vp], i),
            "wino_batch_tune": ([vp, i, ctypes.POINTER(ctypes.c_float), ctypes.POINTER(ctypes.c_float), vp], i),
            "wino_batch_graph_capture": ([vp, vp], i),
            "wino_batch_graph_launch": ([vp, vp], i),
            "wino_conv2d_variant": ([i, vp, vp, vp, vp, i, i, i, i, i, vp], i),
            "wino_conv2d_fused_ws": ([vp, vp, vp, vp, i, i, i, i, i, vp], i),
            "wino_launch_kernelinfo": ([vp, vp, vp], i),
            "wino_filter_transform_unfused": ([vp, vp, i, i, vp], i),
            "wino_unfused_workspace_bytes": ([i, i, i, i, i, ctypes.POINTER(sz), ctypes.POINTER(sz)], i),
            "wino_conv2d_unfused": ([vp, vp, vp, vp, vp, i, i, i, i, i, vp], i),
            "wino_error_read_clear": ([ctypes.POINTER(ctypes.c_uint32)], i),
            "wino_twostage_workspace_bytes": ([i, i, i, i, i], sz),
            "wino_dropin_route": ([vp], i),
            "wino_conv2d_twostage": ([vp, vp, vp, vp, i, i, i, i, i, vp], i),
            "wino_twostage_stage": ([i, vp, vp, vp, vp, i, i, i, i, i, vp], i),
            "wino_twostage_gemm_kernel_ptr_for": ([i], vp),
            "wino_twostage_pair_kernel_ptr": ([], vp),
            "wino_twostage_res_kernel_ptr": ([], vp),
            "wino_twostage_resv_kernel_ptr": ([], vp),
            "wino_twostage_prepass_bytes": ([i, i, i, i], sz),
            "wino_twostage_f8_workspace_bytes": ([i, i, i, i, i, i], sz),
            "wino_conv2d_twostage_f8": ([vp, vp, vp, vp, i, i, i, i, i, i, vp], i),
            "wino_twostage_f8_kernel_ptr": ([i], vp),
            "wino_twostage_stream_kernel_ptr": ([], vp),
            "wino_dropin_filter_u2_kernel_ptr": ([], vp),
            "wino_twostage_output_kernel_ptr": ([], vp),
            "wino_fused_kernel_ptr": ([], vp),
            "wino_f4_filter_bytes": ([i, i, i], sz),
            "wino_f4_workspace_bytes": ([i, i, i, i, i, i], sz),
            "wino_f4_filter_transform": ([vp, i, i, i, vp, sz, vp], i),
            "wino_conv2d_f4": ([vp, vp, i, i, i, i, i, i, vp, sz, vp], i),
        }
        for name, (args, res) in sigs.items():
            fn = getattr(L, name)
            fn.argtypes = args
            fn.restype = res
        _lib = L
    return _lib


def _check(code, what):
    if code != WINO_OK:
        raise WinoError(code, what)


def _stream(stream=None):
    import torch
    s = stream if stream is not None else torch.cuda.current_stream()
    return ctypes.c_void_p(s.cuda_stream)


# ------------------------------------------------------------ drop-in ABI ---
def get_param_size(problem: Problem) -> int:
    n = ctypes.c_int(0)
    _check(lib().wino_getParamsize(ctypes.byref(problem), ctypes.byref(n)), "getParamsize")
    return n.value


def get_kernel_info(problem: Problem, param: ctypes.Array):
    """Returns (code, KernelInfo); the code is returned, not raised, so tests
    can check the rejection paths exactly as a C caller sees them."""
    ki = KernelInfo()
    code = lib().wino_getkernelInfo(ctypes.byref(problem), ctypes.byref(ki),
                                    ctypes.cast(param, ctypes.c_void_p))
    return code, ki


def launch_kernel_info(ki: KernelInfo, param: ctypes.Array, stream=None):
    _check(lib().wino_launch_kernelinfo(ctypes.byref(ki), ctypes.cast(param, ctypes.c_void_p),
                                        _stream(stream)), "launch_kernelinfo")


def make_problem(x, w, y, transform_pin=None, transform_filter=None, mid_result=None,
                 r=3, s=3, u=1, v=1, p=1, q=1) -> Problem:
    n, c, h, wd = x.shape
    k = w.shape[0]
    ptr = lambda t: 0 if t is None else t.data_ptr()
    return Problem(ptr(x), ptr(w), ptr(y), ptr(transform_pin), ptr(transform_filter),
                   ptr(mid_result), n, c, h, wd, k, r, s, u, v, p, q)


class DropinWorkspaces:
    """The caller-owned buffers of the reference harness for one shape
    (src/main.cpp:33-38): transform_pin 4*h*h*n*c, mid_result 4*k*h*w*n and
    transform_filter 16*k*c fp16 elements."""

    def __init__(self, n, c, h, w, k, device, transform_pin=True):
        import torch
        self.transform_pin = (torch.empty(4 * h * h * n * c, dtype=torch.float16, device=device)
                              if transform_pin else None)
        self.mid_result = torch.empty(4 * k * h * w * n, dtype=torch.float16, device=device)
        self.transform_filter = torch.empty(16 * k * c, dtype=torch.float16, device=device)


def dropin_conv2d(x, w, stream=None, ws=None, transform_pin=True, stride=1, pad=None):
    """Run the drop-in path the way the reference harness does
    (src/main.cpp:33-108): caller-allocated output and workspaces sized as
    there, getParamsize, getkernelInfo, then the four launch slots.  With
    transform_pin=False the caller passes no transform_pin workspace and the
    fused kernel reads the NCHW input directly."""
    import torch
    n, c, h, wd = x.shape
    k, _, r, s = w.shape
    pad = (r // 2) if pad is None else pad
    oh, ow = (h - r + 2 * pad) // stride + 1, (wd - s + 2 * pad) // stride + 1
    ws = ws or DropinWorkspaces(n, c, h, wd, k, x.device, transform_pin)
    y = torch.empty((n, k, oh, ow), dtype=torch.float16, device=x.device)
    pr = make_problem(x, w, y, ws.transform_pin, ws.transform_filter, ws.mid_result,
                      r=r, s=s, u=stride, v=stride, p=pad, q=pad)
    size = get_param_size(pr)
    param = (ctypes.c_char * size)()
    code, ki = get_kernel_info(pr, param)
    _check(code, "getkernelInfo")
    launch_kernel_info(ki, param, stream)
    return y


# ------------------------------------------------------------ extension API -
def ucache_bytes(k, c, variant=VAR_F16) -> int:
    return int(lib().wino_ucache_bytes(k, c, variant))


def filter_transform(w, stream=None):
    """fp16 KCRS weights -> fp16 U cache (flat tensor, tile-major layout)."""
    import torch
    k, c = w.shape[:2]
    u = torch.empty(16 * k * c, dtype=torch.float16, device=w.device)
    _check(lib().wino_filter_transform(ctypes.c_void_p(w.data_ptr()), ctypes.c_void_p(u.data_ptr()),
                                       k, c, _stream(stream)), "filter_transform")
    return u


def fused_workspace_bytes(n, c, h, w) -> int:
    return int(lib().wino_fused_workspace_bytes(n, c, h, w))


def input_layout(x, workspace, stream=None):
    """The fused path's pre-pass alone: NCHW input -> channel-blocked workspace."""
    n, c, h, wd = x.shape
    _check(lib().wino_input_layout(ctypes.c_void_p(x.data_ptr()), ctypes.c_void_p(workspace.data_ptr()),
                                   n, c, h, wd, _stream(stream)), "input_layout")


def conv2d_fused(x, ucache, k, out=None, stream=None, workspace=True):
    """Fused conv on a prepared U cache.  workspace=True (default) allocates
    (or takes, if a uint8 tensor is given) the channel-blocked input
    workspace and runs the pre-pass + staged fused kernel; workspace=False
    runs the fused kernel on the NCHW input directly."""
    import torch
    n, c, h, wd = x.shape
    y = out if out is not None else torch.empty((n, k, h, wd), dtype=torch.float16, device=x.device)
    if workspace is False or workspace is None:
        _check(lib().wino_conv2d_fused(ctypes.c_void_p(x.data_ptr()), ctypes.c_void_p(ucache.data_ptr()),
                                       ctypes.c_void_p(y.data_ptr()), n, c, h, wd, k, _stream(stream)),
               "conv2d_fused")
        return y
    if workspace is True:
        workspace = torch.empty(fused_workspace_bytes(n, c, h, wd), dtype=torch.uint8, device=x.device)
    _check(lib().wino_conv2d_fused_ws(ctypes.c_void_p(x.data_ptr()), ctypes.c_void_p(ucache.data_ptr()),
                                      ctypes.c_void_p(workspace.data_ptr()),
                                      ctypes.c_void_p(y.data_ptr()), n, c, h, wd, k, _stream(stream)),
           "conv2d_fused_ws")
    return y


def conv2d_fused_epilogue(x, ucache, k, bias=None, residual=None, relu=False, out=None,
                          workspace=None, stream=None):
    """relu?(conv(x) + bias[k] + residual) in one fused kernel (plus the input
    pre-pass).  bias: float32 [K] tensor or None; residual: fp16 tensor of the
    output's shape or None (may be `out` itself)."""
    import torch
    n, c, h, wd = x.shape
    y = out if out is not None else torch.empty((n, k, h, wd), dtype=torch.float16, device=x.device)
    if workspace is None:
        workspace = torch.empty(fused_workspace_bytes(n, c, h, wd), dtype=torch.uint8, device=x.device)
    ptr = lambda t: ctypes.c_void_p(0 if t is None else t.data_ptr())
    _check(lib().wino_conv2d_fused_epilogue(ptr(x), ptr(ucache), ptr(workspace), ptr(y), ptr(bias),
                                            ptr(residual), 1 if relu else 0, n, c, h, wd, k, _stream(stream)),
           "conv2d_fused_epilogue")
    return y


def conv2d_direct(x, w, stride=1, pad=1, out=None, stream=None):
    """Direct convolution of any filter size / stride / padding (fp16 in and
    out, fp32 accumulation)."""
    import torch
    n, c, h, wd = x.shape
    k, _, r, s = w.shape
    oh, ow = (h - r + 2 * pad) // stride + 1, (wd - s + 2 * pad) // stride + 1
    y = out if out is not None else torch.empty((n, k, oh, ow), dtype=torch.float16, device=x.device)
    _check(lib().wino_conv2d_direct(ctypes.c_void_p(x.data_ptr()), ctypes.c_void_p(w.data_ptr()),
                                    ctypes.c_void_p(y.data_ptr()), n, c, h, wd, k, r, s, stride, stride,
                                    pad, pad, _stream(stream)), "conv2d_direct")
    return y


def igemm_weight_bytes(c, k, r, s) -> int:
    return int(lib().wino_igemm_weight_bytes(c, k, r, s))


def igemm_weight_transform(w, stream=None):
    """fp16 KCRS weights -> the implicit-GEMM weight operand (flat uint8
    tensor of igemm_weight_bytes bytes)."""
    import torch
    k, c, r, s = w.shape
    wp = torch.empty(igemm_weight_bytes(c, k, r, s), dtype=torch.uint8, device=w.device)
    _check(lib().wino_igemm_weight_transform(ctypes.c_void_p(w.data_ptr()), ctypes.c_void_p(wp.data_ptr()),
                                             k, c, r, s, _stream(stream)), "igemm_weight_transform")
    return wp


def conv2d_igemm(x, w, stride=1, pad=1, wprep=None, out=None, stream=None):
    """Tensor-core implicit-GEMM convolution of any filter size / stride /
    padding (fp16 in and out, fp32 accumulation).  wprep: the weights from
    igemm_weight_transform (made here when None)."""
    import torch
    n, c, h, wd = x.shape
    k, _, r, s = w.shape
    oh, ow = (h - r + 2 * pad) // stride + 1, (wd - s + 2 * pad) // stride + 1
    if wprep is None:
        wprep = igemm_weight_transform(w, stream)
    y = out if out is not None else torch.empty((n, k, oh, ow), dtype=torch.float16, device=x.device)
    _check(lib().wino_conv2d_igemm(ctypes.c_void_p(x.data_ptr()), ctypes.c_void_p(wprep.data_ptr()),
                                   ctypes.c_void_p(y.data_ptr()), n, c, h, wd, k, r, s, stride, stride,
                                   pad, pad, _stream(stream)), "conv2d_igemm")
    return y


def conv2d(x, w, stream=None):
    """Filter transform followed by the fused conv (fp16 variant)."""
    return conv2d_fused(x, filter_transform(w, stream), w.shape[0], stream=stream)


def variant_workspace_bytes(variant, n, c, h, w, k) -> int:
    return int(lib().wino_variant_workspace_bytes(variant, n, c, h, w, k))


def conv2d_variant(x, w, variant, out=None, workspace=None, stream=None):
    """Conv with a precision variant of the GEMM stage (VAR_F16, VAR_BF16,
    VAR_F8, VAR_F16_HILO); filter transform, pre-pass and fused kernel per call."""
    import torch
    n, c, h, wd = x.shape
    k = w.shape[0]
    y = out if out is not None else torch.empty((n, k, h, wd), dtype=torch.float16, device=x.device)
    nb = variant_workspace_bytes(variant, n, c, h, wd, k)
    if nb == 0:
        raise WinoError(WINO_EUNSUPPORTED, "variant_workspace_bytes")
    if workspace is None:
        workspace = torch.empty(nb + 256, dtype=torch.uint8, device=x.device)
    off = (-workspace.data_ptr()) % 256
    _check(lib().wino_conv2d_variant(variant, ctypes.c_void_p(x.data_ptr()), ctypes.c_void_p(w.data_ptr()),
                                     ctypes.c_void_p(y.data_ptr()),
                                     ctypes.c_void_p(workspace.data_ptr() + off), n, c, h, wd, k,
                                     _stream(stream)), "conv2d_variant")
    return y


def weight_tag(w, stream=None) -> int:
    """64-bit content tag of fp16 KCRS weights (computed on the GPU)."""
    k, c = w.shape[:2]
    t = ctypes.c_ulonglong(0)
    _check(lib().wino_weight_tag(ctypes.c_void_p(w.data_ptr()), k, c, ctypes.byref(t), _stream(stream)),
           "weight_tag")
    return t.value


def filter_transform_persistent(w, path, stream=None):
    """The U cache of `w`, loaded from `path` when the file holds the U of
    exactly these weights, else computed and written there.  Returns
    (ucache, loaded)."""
    import torch
    k, c = w.shape[:2]
    tag = weight_tag(w, stream)
    u = torch.empty(16 * k * c, dtype=torch.float16, device=w.device)
    rc = lib().wino_ucache_load(os.fsencode(path), ctypes.c_void_p(u.data_ptr()), k, c, tag)
    if rc == WINO_OK:
        return u, True
    if rc not in (WINO_ESTALE, WINO_EIO):
        raise WinoError(rc, "ucache_load")
    u = filter_transform(w, stream)
    # wino_ucache_save reads U with a copy on the legacy stream, which is not
    # ordered against `stream` when that is a non-blocking stream
    (stream if stream is not None else torch.cuda.current_stream()).synchronize()
    _check(lib().wino_ucache_save(os.fsencode(path), ctypes.c_void_p(u.data_ptr()), k, c, tag), "ucache_save")
    return u, False


def filter_transform_unfused(w, stream=None):
    """fp16 KCRS weights -> fp16 U in the unfused GEMM's layout."""
    import torch
    k, c = w.shape[:2]
    u = torch.empty(16 * k * c, dtype=torch.float16, device=w.device)
    _check(lib().wino_filter_transform_unfused(ctypes.c_void_p(w.data_ptr()),
                                               ctypes.c_void_p(u.data_ptr()), k, c, _stream(stream)),
           "filter_transform_unfused")
    return u


def twostage_workspace_bytes(n, c, h, w, k) -> int:
    return int(lib().wino_twostage_workspace_bytes(n, c, h, w, k))


def conv2d_twostage(x, ucache2, k, out=None, workspace=None, stream=None):
    """Two-stage conv on a U cache in the unfused layout (filter_transform_unfused):
    input pre-pass, input transform fused into full-rate tap GEMMs writing
    fp16 M, then the output transform.  workspace: uint8 tensor of
    twostage_workspace_bytes() bytes (allocated when None)."""
    import torch
    n, c, h, wd = x.shape
    y = out if out is not None else torch.empty((n, k, h, wd), dtype=torch.float16, device=x.device)
    nb = twostage_workspace_bytes(n, c, h, wd, k)
    if nb == 0:
        raise WinoError(WINO_EUNSUPPORTED, "twostage_workspace_bytes")
    if workspace is None:
        workspace = _aligned_ws(nb, x.device)
    _check(lib().wino_conv2d_twostage(ctypes.c_void_p(x.data_ptr()), ctypes.c_void_p(ucache2.data_ptr()),
                                      ctypes.c_void_p(workspace.data_ptr()), ctypes.c_void_p(y.data_ptr()),
                                      n, c, h, wd, k, _stream(stream)), "conv2d_twostage")
    return y


def conv2d_twostage_f8(x, ucache2, k, hilo=True, out=None, workspace=None, stream=None):
    """Two-stage conv with an fp8 e4m3 tensor-core GEMM on a U cache from
    filter_transform_unfused: hilo=True splits U and V into hi + lo terms
    (three kind::f8f6f4 MMAs per 32-channel step, fp16-level accuracy),
    hilo=False uses single terms (one MMA, faster, single-term fp8
    accuracy).  C a multiple of 32, at most 256."""
    import torch
    n, c, h, wd = x.shape
    y = out if out is not None else torch.empty((n, k, h, wd), dtype=torch.float16, device=x.device)
    nb = int(lib().wino_twostage_f8_workspace_bytes(n, c, h, wd, k, int(hilo)))
    if nb == 0:
        raise WinoError(WINO_EUNSUPPORTED, "wino_twostage_f8_workspace_bytes")
    if workspace is None:
        workspace = _aligned_ws(nb, x.device)
    _check(lib().wino_conv2d_twostage_f8(ctypes.c_void_p(x.data_ptr()), ctypes.c_void_p(ucache2.data_ptr()),
                                         ctypes.c_void_p(workspace.data_ptr()), ctypes.c_void_p(y.data_ptr()),
                                         n, c, h, wd, k, int(hilo), _stream(stream)), "conv2d_twostage_f8")
    return y


def twostage_stage(stage, x, ucache2, k, out, workspace, stream=None):
    """One stage of conv2d_twostage (0 pre-pass, 1 tap GEMM, 2 output
    transform) on a workspace of twostage_workspace_bytes()."""
    n, c, h, wd = x.shape
    _check(lib().wino_twostage_stage(stage, ctypes.c_void_p(x.data_ptr()), ctypes.c_void_p(ucache2.data_ptr()),
                                     ctypes.c_void_p(workspace.data_ptr()), ctypes.c_void_p(out.data_ptr()),
                                     n, c, h, wd, k, _stream(stream)), "twostage_stage")
    return out


class UnfusedWorkspace:
    """Caller-owned V and M buffers of the unfused path for one shape."""

    def __init__(self, n, c, h, w, k, device):
        import torch
        vb, mb = ctypes.c_size_t(0), ctypes.c_size_t(0)
        _check(lib().wino_unfused_workspace_bytes(n, c, h, w, k, ctypes.byref(vb), ctypes.byref(mb)),
               "unfused_workspace_bytes")
        self.v = torch.empty(vb.value, dtype=torch.uint8, device=device)
        self.m = torch.empty(mb.value, dtype=torch.uint8, device=device)


def conv2d_unfused(x, ucache2, k, ws=None, out=None, stream=None):
    import torch
    n, c, h, wd = x.shape
    ws = ws or UnfusedWorkspace(n, c, h, wd, k, x.device)
    y = out if out is not None else torch.empty((n, k, h, wd), dtype=torch.float16, device=x.device)
    _check(lib().wino_conv2d_unfused(ctypes.c_void_p(x.data_ptr()), ctypes.c_void_p(ucache2.data_ptr()),
                                     ctypes.c_void_p(y.data_ptr()), ctypes.c_void_p(ws.v.data_ptr()),
                                     ctypes.c_void_p(ws.m.data_ptr()), n, c, h, wd, k, _stream(stream)),
           "conv2d_unfused")
    return y


CFG_KMAJOR, CFG_DIRECT, CFG_SPLIT_SHIFT, NCFG = 1, 2, 2, 16


def cfg_split(level):
    return level << CFG_SPLIT_SHIFT

# The uneven ResNet-style 3x3 stride-1 pad-1 layer set of the batched launch,
# as (C, K, H=W): two each of the four square stages plus the four C != K
# transitions.
RESNET_LAYER_SET = [(64, 64, 56), (64, 64, 56), (128, 128, 28), (128, 128, 28),
                    (256, 256, 14), (256, 256, 14), (512, 512, 7), (512, 512, 7),
                    (64, 128, 56), (128, 256, 28), (256, 512, 14), (512, 256, 7)]


def _p(t):
    return ctypes.c_void_p(0 if t is None else t.data_ptr())


def _aligned_ws(nbytes, device):
    """A uint8 workspace view starting on a 256-byte boundary (None for 0 bytes)."""
    import torch
    if nbytes == 0:
        return None
    buf = torch.empty(nbytes + 256, dtype=torch.uint8, device=device)
    off = (-buf.data_ptr()) % 256
    return buf[off:off + nbytes]


# ------------------------------------------------------ F(4x4,3x3) path ---
def f4_workspace_bytes(n, c, h, w, k, hilo=True) -> int:
    return int(lib().wino_f4_workspace_bytes(n, c, h, w, k, int(bool(hilo))))


class ConvF4:
    """Winograd F(4x4,3x3) conv of one weight tensor over inputs of one shape.

    The filter transform runs once (constructor / set_weight) into the head of
    the workspace; every call runs input transform, 36-tap GEMM and output
    transform.  hilo=True stores U and V as fp16 hi + lo pairs (the accurate
    form); hilo=False as single fp16 values (about ten times larger error)."""

    def __init__(self, w, n, h, wd, hilo=True, stream=None):
        self.k, self.c = w.shape[:2]
        self.n, self.h, self.wd, self.hilo = n, h, wd, int(bool(hilo))
        self.nbytes = f4_workspace_bytes(n, self.c, h, wd, self.k, self.hilo)
        self.ws = _aligned_ws(self.nbytes, w.device)
        self.set_weight(w, stream)

    def set_weight(self, w, stream=None):
        if tuple(w.shape) != (self.k, self.c, 3, 3) or w.dtype.itemsize != 2:
            raise WinoError(WINO_EINVAL, "ConvF4.set_weight: weight shape")
        self._w = w
        _check(lib().wino_f4_filter_transform(ctypes.c_void_p(w.data_ptr()), self.k, self.c, self.hilo,
                                              ctypes.c_void_p(self.ws.data_ptr()), self.nbytes,
                                              _stream(stream)), "f4_filter_transform")

    def __call__(self, x, out=None, stream=None):
        import torch
        if tuple(x.shape) != (self.n, self.c, self.h, self.wd):
            raise WinoError(WINO_EINVAL, "ConvF4: input shape")
        y = out if out is not None else torch.empty((self.n, self.k, self.h, self.wd), dtype=torch.float16,
                                                   device=x.device)
        _check(lib().wino_conv2d_f4(ctypes.c_void_p(x.data_ptr()), ctypes.c_void_p(y.data_ptr()), self.n,
                                    self.c, self.h, self.wd, self.k, self.hilo,
                                    ctypes.c_void_p(self.ws.data_ptr()), self.nbytes, _stream(stream)),
               "conv2d_f4")
        return y


def conv2d_f4(x, w, hilo=True, out=None, stream=None):
    """One F(4x4,3x3) conv (filter transform included)."""
    n, c, h, wd = x.shape
    return ConvF4(w, n, h, wd, hilo, stream)(x, out, stream)


def cfg_workspace_bytes(n, c, h, w, k, cfg) -> int:
    return int(lib().wino_fused_cfg_workspace_bytes(n, c, h, w, k, cfg))


def tune_workspace_bytes(n, c, h, w, k) -> int:
    return int(lib().wino_fused_tune_workspace_bytes(n, c, h, w, k))


def conv2d_fused_cfg(x, ucache, k, cfg, workspace=None, out=None, stream=None):
    """Fused fp16 conv on a cached U with a schedule configuration (CFG_* bits)."""
    import torch
    n, c, h, wd = x.shape
    y = out if out is not None else torch.empty((n, k, h, wd), dtype=torch.float16, device=x.device)
    if workspace is None:
        workspace = _aligned_ws(cfg_workspace_bytes(n, c, h, wd, k, cfg), x.device)
    _check(lib().wino_conv2d_fused_cfg(_p(x), _p(ucache), _p(workspace), _p(y), n, c, h, wd, k, cfg,
                                       _stream(stream)), "conv2d_fused_cfg")
    return y


def tune_layer(x, ucache, k, workspace, out, reps=3, stream=None):
    """Exhaustive tuning of one layer: (per-config mean us list, -1 outside
    the tuning space; best cfg).  workspace: tune_workspace_bytes() bytes,
    256-byte aligned (see _aligned_ws), or None for the direct configurations."""
    n, c, h, wd = x.shape
    us = (ctypes.c_float * NCFG)()
    best = ctypes.c_int(-1)
    _check(lib().wino_tune_layer(_p(x), _p(ucache), _p(workspace), _p(out), n, c, h, wd, k, reps, us,
                                 ctypes.byref(best), _stream(stream)), "tune_layer")
    return [float(v) for v in us], best.value


class Batch:
    """Uneven fp16 layers run as one persistent launch (optionally a CUDA graph).

    Each layer owns its input, U cache (filter_transform), output and pre-pass
    workspace; the Python object keeps references so they outlive the batch."""

    def __init__(self):
        self._h = ctypes.c_void_p(0)
        _check(lib().wino_batch_create(ctypes.byref(self._h)), "batch_create")
        self._keep = []

    def add(self, x, ucache, k, out, workspace=None):
        n, c, h, wd = x.shape
        _check(lib().wino_batch_add_layer(self._h, _p(x), _p(ucache), _p(workspace), _p(out), n, c, h,
                                          wd, k), "batch_add_layer")
        self._keep.append((x, ucache, out, workspace))

    def __len__(self):
        return lib().wino_batch_num_layers(self._h)

    def set_config(self, layer, cfg):
        _check(lib().wino_batch_set_config(self._h, layer, cfg), "batch_set_config")

    def config(self, layer):
        v = ctypes.c_int(0)
        _check(lib().wino_batch_get_config(self._h, layer, ctypes.byref(v)), "batch_get_config")
        return v.value

    def set_route(self, layer, route):
        """0: the layer runs inside the persistent fused launch; 1: the
        two-stage route (128 x 256 tap-GEMM units) launched before it."""
        _check(lib().wino_batch_set_route(self._h, layer, route), "batch_set_route")

    def route(self, layer):
        """(route, fastest fused us, two-stage us) -- the timings from tune()."""
        r, f, t = ctypes.c_int(0), ctypes.c_float(0), ctypes.c_float(0)
        _check(lib().wino_batch_get_route(self._h, layer, ctypes.byref(r), ctypes.byref(f), ctypes.byref(t)),
               "batch_get_route")
        return r.value, f.value, t.value

    def set_order(self, order):
        arr = (ctypes.c_int * len(order))(*order)
        _check(lib().wino_batch_set_order(self._h, arr, len(order)), "batch_set_order")

    def order(self):
        n = len(self)
        arr = (ctypes.c_int * n)()
        _check(lib().wino_batch_get_order(self._h, arr, n), "batch_get_order")
        return list(arr)

    def run(self, stream=None):
        _check(lib().wino_batch_run(self._h, _stream(stream)), "batch_run")

    def tune(self, reps=3, stream=None):
        n = len(self)
        lu = (ctypes.c_float * (n * NCFG))()
        ou = (ctypes.c_float * 3)()
        _check(lib().wino_batch_tune(self._h, reps, lu, ou, _stream(stream)), "batch_tune")
        return [list(lu[i * NCFG:(i + 1) * NCFG]) for i in range(n)], list(ou)

    def tuning_state(self):
        """The autotuner's choices, to be saved (JSON-able) and restored later."""
        return {"version": 2, "configs": [self.config(i) for i in range(len(self))],
                "routes": [self.route(i)[0] for i in range(len(self))], "order": self.order()}

    def restore(self, state):
        """Re-applies tuning_state() output (the same layer list) without re-tuning
        (version 1 states carry no routes: every layer fused)."""
        if state.get("version") not in (1, 2) or len(state["configs"]) != len(self):
            raise ValueError("tuning state of another version or layer list")
        for i, c in enumerate(state["configs"]):
            self.set_config(i, c)
        for i, r in enumerate(state.get("routes", [0] * len(self))):
            self.set_route(i, r)
        self.set_order(state["order"])

    def capture(self, stream=None):
        _check(lib().wino_batch_graph_capture(self._h, _stream(stream)), "batch_graph_capture")

    def launch(self, stream=None):
        _check(lib().wino_batch_graph_launch(self._h, _stream(stream)), "batch_graph_launch")

    def close(self):
        if self._h:
            lib().wino_batch_destroy(self._h)
            self._h = ctypes.c_void_p(0)

    def __del__(self):
        try:
            self.close()
        except Exception:  # noqa: BLE001 - interpreter shutdown
            pass


def error_read_clear() -> int:
    code = ctypes.c_uint32(0)
    _check(lib().wino_error_read_clear(ctypes.byref(code)), "error_read_clear")
    return code.value
