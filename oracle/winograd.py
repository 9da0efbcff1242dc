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


def conv2d_winograd_emulated(x, w, operand="f16"):
    """Winograd with the rounding points of the fused fp16/bf16 kernels.

    U and V are formed exactly (fp32 is exact for these +-1/2 combinations of
    fp16 values up to one rounding) and rounded once to the GEMM operand type;
    M is accumulated in wide precision (the tensor core accumulates in fp32);
    the output transform is done before the single fp16 rounding of Y.
    """
    rnd = _f16 if operand == "f16" else _bf16
    n, c, h, wd = x.shape
    k = w.shape[0]
    u = rnd(filter_transform(w))
    v = rnd(input_transform(x))
    m = gemm(u, v).astype(np.float32).astype(np.float64)
    return output_transform(m, n, k, h, wd)
