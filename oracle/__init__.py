"""Test-only checkers for the Winograd F(2x2,3x3) conv2d path.

TEST INFRASTRUCTURE: only tests/, __graft_entry__.smoke() and bench.py's
CPU-baseline / reference legs import this package, and only as the checker.
Nothing on the product path (the CUDA library in 2024pra_conv_b200/) imports,
links or calls anything here.

Contents
  conv2d_f64        FP64 direct convolution (conv_oracle.c, a restatement of
                    the reference's conv2dcpu, include/verfiy.h:5-43, with
                    exact double products and a double result).
  ref_conv2dcpu     the reference's own conv2dcpu compiled unmodified from
                    include/verfiy.h (oracle/_ref); fp16 output as it stores it.
  make_inputs       seeded synthetic tensors with the distributions of the
                    benchmark workloads.
  rel_l2, max_norm  error metrics against the FP64 result.
  winograd          NumPy restatement of the reference's Winograd stages.
"""
from __future__ import annotations

import ctypes
import os
import subprocess
import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
_BUILD = os.path.join(HERE, "_build", "liboracle.so")
_REF_PORTABLE = os.path.join(HERE, "_ref", "libverfiy_ref.so")
_REF_FP16 = os.path.join(HERE, "_ref", "libverfiy_ref_fp16.so")

_lib = None
_ref = {}


def build():
    """Compile the C oracle (and the reference CPU path when the environment
    variable WINO_REFERENCE_DIR names the reference tree)."""
    ref = os.environ.get("WINO_REFERENCE_DIR")
    subprocess.run(["make", "-s", "-C", HERE] + ([f"REF={ref}"] if ref else []), check=True)


def _oracle_lib():
    global _lib
    if _lib is None:
        if not os.path.exists(_BUILD):
            build()
        lib = ctypes.CDLL(_BUILD)
        lib.oracle_conv2d_f64.argtypes = [ctypes.c_void_p] * 3 + [ctypes.c_int] * 11
        lib.oracle_conv2d_f64.restype = None
        _lib = lib
    return _lib


def _cpu_flags():
    try:
        with open("/proc/cpuinfo") as f:
            for line in f:
                if line.startswith("flags"):
                    return set(line.split(":", 1)[1].split())
    except OSError:
        pass
    return set()


_V4_FP16_FLAGS = {"avx512f", "avx512bw", "avx512cd", "avx512dq", "avx512vl", "avx512_fp16"}


def ref_variants():
    """Reference CPU builds usable on this host: name -> path."""
    out = {}
    if os.path.exists(_REF_PORTABLE):
        out["portable"] = _REF_PORTABLE
    if os.path.exists(_REF_FP16) and _V4_FP16_FLAGS <= _cpu_flags():
        out["avx512fp16"] = _REF_FP16
    return out


def _ref_lib(variant="portable"):
    if variant not in _ref:
        paths = ref_variants()
        if variant not in paths:
            raise FileNotFoundError(
                f"reference conv2dcpu build '{variant}' not available (run make -C oracle "
                "where the reference tree exists)")
        lib = ctypes.CDLL(paths[variant])
        lib.ref_conv2dcpu.argtypes = [ctypes.c_void_p] * 3 + [ctypes.c_int] * 11
        lib.ref_conv2dcpu.restype = None
        lib.ref_conv2dcpu_omp.argtypes = [ctypes.c_void_p] * 3 + [ctypes.c_int] * 12
        lib.ref_conv2dcpu_omp.restype = None
        lib.ref_max_threads.restype = ctypes.c_int
        _ref[variant] = lib
    return _ref[variant]


def out_hw(h, w, r=3, s=3, u=1, v=1, p=1, q=1):
    """Output size, readme.txt:17-19 of the reference."""
    return (h - r + 2 * p) // u + 1, (w - s + 2 * q) // v + 1


def conv2d_f64(x16, w16, u=1, v=1, p=1, q=1):
    """FP64 direct conv of fp16 NCHW input and KCRS weights -> float64 NKPQ."""
    x = np.ascontiguousarray(x16.astype(np.float32))
    wt = np.ascontiguousarray(w16.astype(np.float32))
    n, c, h, w = x.shape
    k, c2, r, s = wt.shape
    assert c == c2
    oh, ow = out_hw(h, w, r, s, u, v, p, q)
    out = np.empty((n, k, oh, ow), np.float64)
    _oracle_lib().oracle_conv2d_f64(x.ctypes.data, wt.ctypes.data, out.ctypes.data,
                                    n, c, h, w, k, r, s, u, v, p, q)
    return out


def ref_conv2dcpu(x16, w16, u=1, v=1, p=1, q=1, threads=1, variant="portable"):
    """Run the reference's unmodified conv2dcpu; returns its fp16 output."""
    x = np.ascontiguousarray(x16.astype(np.float16))
    wt = np.ascontiguousarray(w16.astype(np.float16))
    n, c, h, w = x.shape
    k, _, r, s = wt.shape
    oh, ow = out_hw(h, w, r, s, u, v, p, q)
    out = np.zeros((n, k, oh, ow), np.float16)
    lib = _ref_lib(variant)
    if threads == 1:
        lib.ref_conv2dcpu(x.ctypes.data, wt.ctypes.data, out.ctypes.data,
                          n, c, h, w, k, r, s, u, v, p, q)
    else:
        lib.ref_conv2dcpu_omp(x.ctypes.data, wt.ctypes.data, out.ctypes.data,
                              n, c, h, w, k, r, s, u, v, p, q, int(threads))
    return out


def ref_max_threads(variant="portable"):
    return int(_ref_lib(variant).ref_max_threads())


# ---------------------------------------------------------------- inputs ----
DISTS = ("uniform", "relu_normal", "normal", "student_t3")


def make_inputs(n, c, h, w, k, seed=0, x_dist="uniform", w_std=None, r=3, s=3):
    """Seeded fp16 NCHW input and KCRS weights.

    x_dist: 'uniform' U[-1,1]; 'relu_normal' max(N(0,1),0); 'normal' N(0,1);
            'student_t3' Student-t with 3 dof clipped to +-60.
    w_std : weight std-dev; default sqrt(1/(9C)).  Weights are N(0, w_std^2).
    Values are sampled in float64 and rounded to fp16.
    """
    rng = np.random.default_rng(seed)
    shape = (n, c, h, w)
    if x_dist == "uniform":
        x = rng.uniform(-1.0, 1.0, shape)
    elif x_dist == "relu_normal":
        x = np.maximum(rng.standard_normal(shape), 0.0)
    elif x_dist == "normal":
        x = rng.standard_normal(shape)
    elif x_dist == "student_t3":
        x = np.clip(rng.standard_t(3, shape), -60.0, 60.0)
    else:
        raise ValueError(x_dist)
    if w_std is None:
        w_std = np.sqrt(1.0 / (9.0 * c))
    wt = rng.standard_normal((k, c, r, s)) * w_std
    return x.astype(np.float16), wt.astype(np.float16)


def make_reference_style_inputs(n, c, h, w, k, seed=0, r=3, s=3):
    """Inputs shaped like the reference harness's (rand()%255)/255 data
    (src/main.cpp:40-48): values in [0, 254/255], so every output is >= 0."""
    rng = np.random.default_rng(seed)
    x = rng.integers(0, 255, (n, c, h, w)) / 255.0
    wt = rng.integers(0, 255, (k, c, r, s)) / 255.0
    return x.astype(np.float16), wt.astype(np.float16)


# ---------------------------------------------------------------- metrics ---
def rel_l2(y, y64):
    y = np.asarray(y, np.float64)
    y64 = np.asarray(y64, np.float64)
    den = np.linalg.norm(y64.ravel())
    return float(np.linalg.norm((y - y64).ravel()) / (den if den > 0 else 1.0))


def max_norm(y, y64):
    y = np.asarray(y, np.float64)
    y64 = np.asarray(y64, np.float64)
    den = np.max(np.abs(y64)) if y64.size else 0.0
    return float(np.max(np.abs(y - y64)) / (den if den > 0 else 1.0)) if y.size else 0.0


def reference_check(gpu_out16, cpu_out16):
    """The reference harness's own pass/fail rule (src/main.cpp:137-151):
    the first element with |gpu-cpu|/gpu > 0.01, or a NaN/Inf GPU value,
    counts as one error.  The difference is formed in fp16 as there."""
    g = np.asarray(gpu_out16, np.float16).ravel()
    c = np.asarray(cpu_out16, np.float16).ravel()
    with np.errstate(divide="ignore", invalid="ignore"):
        diff = np.abs((g - c).astype(np.float16)).astype(np.float32)
        rel = diff / g.astype(np.float32)
        bad = (rel > 0.01) | np.isnan(g.astype(np.float32)) | np.isinf(g.astype(np.float32))
    return 1 if bool(np.any(bad)) else 0
