"""NumPy model of the Winograd F(4x4,3x3) variant.

TEST INFRASTRUCTURE ONLY (see oracle/__init__.py).

The reference has F(2x2,3x3) only (src/preprocessing.cuh:75-424,
src/conv2d.cpp:17-250); F(4x4,3x3) is the larger-tile member of the same
family.  The matrices are the published ones of Lavin & Gray, "Fast
Algorithms for Convolutional Neural Networks" (CVPR 2016), interpolation
points 0, 1, -1, 2, -2 and infinity:

  G  (6x3)  rows  [1/4,0,0] [-1/6,-1/6,-1/6] [-1/6,1/6,-1/6]
                  [1/24,1/12,1/6] [1/24,-1/12,1/6] [0,0,1]
  Bt (6x6)  rows  [4,0,-5,0,1,0] [0,-4,-4,1,1,0] [0,4,-4,-1,1,0]
                  [0,-2,-1,2,1,0] [0,2,-1,-2,1,0] [0,4,0,-5,0,1]
  At (4x6)  rows  [1,1,1,1,1,0] [0,1,-1,2,-2,0] [0,1,1,4,4,0] [0,1,-1,8,-8,1]

Tiles follow the reference's pad-1 window semantics (the init_mask /
prefetch_input zeroing of src/preprocessing.cuh:6-46) with a 4-output step:
output tile (ty, tx) covers outputs 4ty..4ty+3 x 4tx..4tx+3; its input window
is rows 4ty-1..4ty+4 and columns 4tx-1..4tx+4, zero outside the image.  Tiles
per image: ceil(P/4) * ceil(Q/4); tap index t = 6*a + b.

Rounding model of the CUDA path (winograd_f4.cu): U and V are formed in fp32
and stored as fp16 -- one piece (plain) or a hi + lo pair, hi = fp16(v),
lo = fp16(v - hi) -- the tap GEMM accumulates the products of the pieces
(hi*hi + lo*hi + hi*lo for hi+lo) in fp32, M is kept in fp32, and the output
transform runs in fp32 before the one fp16 rounding of Y.
"""
from __future__ import annotations

import numpy as np

G4 = np.array([[1 / 4, 0, 0],
               [-1 / 6, -1 / 6, -1 / 6],
               [-1 / 6, 1 / 6, -1 / 6],
               [1 / 24, 1 / 12, 1 / 6],
               [1 / 24, -1 / 12, 1 / 6],
               [0, 0, 1]], np.float64)
BT4 = np.array([[4, 0, -5, 0, 1, 0],
                [0, -4, -4, 1, 1, 0],
                [0, 4, -4, -1, 1, 0],
                [0, -2, -1, 2, 1, 0],
                [0, 2, -1, -2, 1, 0],
                [0, 4, 0, -5, 0, 1]], np.float64)
AT4 = np.array([[1, 1, 1, 1, 1, 0],
                [0, 1, -1, 2, -2, 0],
                [0, 1, 1, 4, 4, 0],
                [0, 1, -1, 8, -8, 1]], np.float64)


def tiles_hw(h, w):
    return (h + 3) // 4, (w + 3) // 4


def filter_transform(w):
    """KCRS 3x3 -> U[36][K][C] = (G g G^T), tap t = 6a + b."""
    w = np.asarray(w, np.float64)
    u = np.einsum("ai,kcij,bj->abkc", G4, w, G4)
    return u.reshape(36, w.shape[0], w.shape[1])


def input_windows(x):
    """NCHW -> d[N][C][TP][TQ][6][6] zero-padded 6x6 windows at stride 4."""
    x = np.asarray(x, np.float64)
    n, c, h, w = x.shape
    tp, tq = tiles_hw(h, w)
    pad = np.zeros((n, c, 4 * tp + 2, 4 * tq + 2), np.float64)
    pad[:, :, 1:h + 1, 1:w + 1] = x
    d = np.empty((n, c, tp, tq, 6, 6), np.float64)
    for i in range(6):
        for j in range(6):
            d[..., i, j] = pad[:, :, i:i + 4 * tp:4, j:j + 4 * tq:4]
    return d


def input_transform(x):
    """NCHW -> V[36][N*TP*TQ][C] = (B^T d B)."""
    d = input_windows(x)
    n, c, tp, tq = d.shape[:4]
    v = np.einsum("ai,nctqij,bj->abntqc", BT4, d, BT4)
    return v.reshape(36, n * tp * tq, c)


def gemm(u, v):
    """M[t][tile][k] = sum_c V[t][tile][c] * U[t][k][c]."""
    return np.einsum("tpc,tkc->tpk", v, u)


def output_transform(m, n, k, p, q):
    """M[36][N*TP*TQ][K] -> Y[N][K][P][Q], Y tile = A^T m A."""
    tp, tq = tiles_hw(p, q)
    mm = np.asarray(m, np.float64).reshape(6, 6, n, tp, tq, k)
    y = np.einsum("ia,abntqk,jb->nktiqj", AT4, mm, AT4)
    y = y.reshape(n, k, 4 * tp, 4 * tq)
    return y[:, :, :p, :q]


def conv2d_f4_f64(x, w):
    """Exact-arithmetic F(4x4,3x3) (equals the direct conv up to fp64 rounding)."""
    n, c, h, wd = x.shape
    return output_transform(gemm(filter_transform(w), input_transform(x)), n, w.shape[0], h, wd)


def _f32(a):
    return np.asarray(a, np.float64).astype(np.float32).astype(np.float64)


def _f16(a):
    return np.asarray(a, np.float64).astype(np.float16).astype(np.float64)


def split_hilo(a):
    """fp32 value -> (hi, lo) fp16 pair, hi = fp16(a), lo = fp16(a - hi)."""
    a = _f32(a)
    hi = _f16(a)
    return hi, _f16(a - hi)


def conv2d_f4_emulated(x, w, hilo=True):
    """The CUDA F(4x4,3x3) path's rounding points (module docstring)."""
    n, c, h, wd = x.shape
    k = w.shape[0]
    u = _f32(filter_transform(w))
    v = _f32(input_transform(x))
    if hilo:
        uh, ul = split_hilo(u)
        vh, vl = split_hilo(v)
        m = gemm(uh, vh) + gemm(uh, vl) + gemm(ul, vh)
    else:
        m = gemm(_f16(u), _f16(v))
    return output_transform(_f32(m), n, k, h, wd)
