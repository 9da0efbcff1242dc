"""NumPy restatement of the reference's Winograd F(2x2,3x3) stages.

TEST INFRASTRUCTURE ONLY (see oracle/__init__.py).

Tap index t = 4*a + b (row a, column b of the 4x4 Winograd tile), as in the
reference's filter transform (src/preprocessing.cuh:93-108), input transform
(src/preprocessing.cuh:56-71) and output transform (src/conv2d.cpp:33-40).

  G  = [[1,0,0],[1/2,1/2,1/2],[1/2,-1/2,1/2],[0,0,1]]      preprocessing.cuh:77-81
  Bt = [[1,0,-1,0],[0,1,1,0],[0,-1,1,0],[0,1,0,-1]]       preprocessing.cuh:50-54
  At = [[1,1,1,0],[0,1,-1,-1]]                            conv2d.cpp:18-22

Tiles: output tile (ty, tx) covers outputs (2ty..2ty+1, 2tx..2tx+1); its
input window is rows 2ty-1..2ty+2 and columns 2tx-1..2tx+2 with zeros
outside the image (pad 1, the init_mask/prefetch_input semantics of
preprocessing.cuh:6-46).  Tiles per image: ceil(P/2) * ceil(Q/2); outputs of
a tile that fall outside P x Q are dropped.
"""
from __future__ import annotations

import numpy as np

G = np.array([[1, 0, 0], [0.5, 0.5, 0.5], [0.5, -0.5, 0.5], [0, 0, 1]], np.float64)
BT = np.array([[1, 0, -1, 0], [0, 1, 1, 0], [0, -1, 1, 0], [0, 1, 0, -1]], np.float64)
AT = np.array([[1, 1, 1, 0], [0, 1, -1, -1]], np.float64)


def tiles_hw(h, w):
    return (h + 1) // 2, (w + 1) // 2


def filter_transform(w):
    """KCRS 3x3 -> U[16][K][C] = (G g G^T) flattened row-major over the tap."""
    w = np.asarray(w, np.float64)
    u = np.einsum("ai,kcij,bj->abkc", G, w, G)
    return u.reshape(16, w.shape[0], w.shape[1])


def input_windows(x):
    """NCHW -> d[N][C][TP][TQ][4][4] zero-padded 4x4 windows."""
    x = np.asarray(x, np.float64)
    n, c, h, w = x.shape
    tp, tq = tiles_hw(h, w)
    pad = np.zeros((n, c, 2 * tp + 2, 2 * tq + 2), np.float64)
    pad[:, :, 1:h + 1, 1:w + 1] = x
    d = np.empty((n, c, tp, tq, 4, 4), np.float64)
    for i in range(4):
        for j in range(4):
            d[..., i, j] = pad[:, :, i:i + 2 * tp:2, j:j + 2 * tq:2]
    return d


def input_transform(x):
    """NCHW -> V[16][N*TP*TQ][C] = (B^T d B) flattened over the tap."""
    d = input_windows(x)
    n, c, tp, tq = d.shape[:4]
    v = np.einsum("ai,nctqij,bj->abntqc", BT, d, BT)
    return v.reshape(16, n * tp * tq, c)


def gemm(u, v):
    """M[t][tile][k] = sum_c V[t][tile][c] * U[t][k][c]."""
    return np.einsum("tpc,tkc->tpk", v, u)


def output_transform(m, n, k, p, q):
    """M[16][N*TP*TQ][K] -> Y[N][K][P][Q] with Y tile = A^T m A."""
    tp, tq = tiles_hw(p, q)
    mm = np.asarray(m, np.float64).reshape(4, 4, n, tp, tq, k)
    y = np.einsum("ia,abntqk,jb->nktiqj", AT, mm, AT)
    y = y.reshape(n, k, 2 * tp, 2 * tq)
    return y[:, :, :p, :q]


def conv2d_winograd_f64(x, w):
    """Exact-arithmetic Winograd result (equals the direct conv up to fp64 rounding)."""
    n, c, h, wd = x.shape
    k = w.shape[0]
    return output_transform(gemm(filter_transform(w), input_transform(x)), n, k, h, wd)


def _f16(a):
    return np.asarray(a, np.float64).astype(np.float16).astype(np.float64)


def _bf16(a):
    a32 = np.asarray(a, np.float32)
    b = a32.view(np.uint32).astype(np.uint64)
    b = ((b + 0x7FFF + ((b >> 16) & 1)) >> 16) << 16
    return b.astype(np.uint32).view(np.float32).astype(np.float64)


def input_transform_f16(x):
    """B^T d B as the fused kernel's producers compute it: packed fp16
    arithmetic, each two-term +- sum rounded to fp16 once (rows of B^T d,
    then the columns of that times B)."""
    d = input_windows(x)
    n, c, tp, tq = d.shape[:4]
    e = _f16(np.einsum("ai,nctqij->nctqaj", BT, d))
    v = _f16(np.einsum("nctqaj,bj->abntqc", e, BT))
    return v.reshape(16, n * tp * tq, c)


def _e4m3(a):
    """Round to fp8 e4m3 (3 mantissa bits, min normal 2^-6, subnormal step
    2^-9), nearest-even, saturating at 448 (the .satfinite conversion)."""
    a = np.asarray(a, np.float64)
    mag = np.abs(a)
    e = np.floor(np.log2(np.maximum(mag, 2.0 ** -6)))
    step = np.where(mag < 2.0 ** -6, 2.0 ** -9, 2.0 ** (e - 3))
    r = np.round(mag / step) * step
    return np.sign(a) * np.minimum(r, 448.0)


def conv2d_winograd_f8_emulated(x, w):
    """The fp8 e4m3 variant's quantization, step by step (a model of the
    fused kernel's fp8 path, not of the reference, which has no fp8 path):
    per input channel c, inv_c = fp16(min(448 / (4 max|x_c|), 65504)) and
    sv_c = 1 / inv_c (|V| <= 4 max|x_c|); V8 = e4m3(fp16(V) * inv_c);
    U'[t][k][c] = U * sv_c, su[t][k] = max_c |U'| / 448, U8 = e4m3(U' / su);
    M = su * sum_c U8 V8 (wide accumulation); output transform in wide
    precision."""
    n, c, h, wd = x.shape
    k = w.shape[0]
    amax = np.abs(np.asarray(x, np.float64)).max(axis=(0, 2, 3))
    inv = np.where(amax > 0, 448.0 / (4.0 * np.where(amax > 0, amax, 1.0)), 1.0)
    inv = _f16(np.minimum(inv, 65504.0))
    sv = 1.0 / inv
    v8 = _e4m3(_f16(input_transform_f16(x) * inv[None, None, :]))
    u1 = filter_transform(w) * sv[None, None, :]
    su = np.abs(u1).max(axis=2) / 448.0
    su = np.where(su > 0, su, 1.0)
    u8 = _e4m3(u1 / su[:, :, None])
    m = gemm(u8, v8) * su[:, None, :]
    return output_transform(m, n, k, h, wd)


def conv2d_winograd_f8_twostage_emulated(x, w, hilo=True):
    """The two-stage fp8 path's rounding points (a model of that path; the
    reference has no fp8 path): inv_c as in the fp8 variant above;
    V' = fp16(fp16(V) * inv_c), V_hi = e4m3(V'), V_lo = e4m3(V' - V_hi);
    U' = fp16(U) / inv_c, su[t][k] = max_c |U'| / 448, U_hi / U_lo the same
    split of U' / su; M = fp16(su * (U_hi V_hi + U_lo V_hi + U_hi V_lo))
    (hilo) or fp16(su * U_hi V_hi) (single terms), wide accumulation; output
    transform in wide precision."""
    n, c, h, wd = x.shape
    k = w.shape[0]
    amax = np.abs(np.asarray(x, np.float64)).max(axis=(0, 2, 3))
    inv = np.where(amax > 0, 448.0 / (4.0 * np.where(amax > 0, amax, 1.0)), 1.0)
    inv = _f16(np.minimum(inv, 65504.0))
    vp = _f16(input_transform_f16(x) * inv[None, None, :])
    vh = _e4m3(vp)
    vl = _e4m3(vp - vh)
    u1 = _f16(filter_transform(w)) / inv[None, None, :]
    su = np.abs(u1).max(axis=2) / 448.0
    su = np.where(su > 0, su, 1.0)
    a = u1 / su[:, :, None]
    uh = _e4m3(a)
    ul = _e4m3(a - uh)
    if hilo:
        m = _f16((gemm(uh, vh) + gemm(ul, vh) + gemm(uh, vl)) * su[:, None, :])
    else:
        m = _f16(gemm(uh, vh) * su[:, None, :])
    return output_transform(m, n, k, h, wd)


def conv2d_winograd_emulated(x, w, operand="f16"):
    """Winograd with the rounding points of the fused fp16/bf16 kernels.

    U is formed exactly (fp32 is exact for these +-1/2 combinations of fp16
    values up to one rounding) and rounded once to the operand type; V is
    formed in packed fp16 arithmetic (input_transform_f16) and, for bf16,
    rounded once more; M is accumulated in wide precision (the tensor core
    accumulates in fp32); the output transform is done before the single fp16
    rounding of Y.
    """
    rnd = _f16 if operand == "f16" else _bf16
    n, c, h, wd = x.shape
    k = w.shape[0]
    u = rnd(filter_transform(w))
    v = rnd(input_transform_f16(x))
    m = gemm(u, v).astype(np.float32).astype(np.float64)
    return output_transform(m, n, k, h, wd)
