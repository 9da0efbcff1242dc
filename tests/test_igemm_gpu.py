"""Tensor-core implicit-GEMM convolution (igemm_conv.cu) for the shapes the
Winograd path does not take: 1x1 projections, stride-2 3x3 downsampling,
ragged channel counts, larger filters.  Through the extension API and behind
the drop-in ABI (route 4), against FP64 (rel-L2 <= 2e-3, max-normalised
<= 1e-2, as the direct kernel's tests) computed by the oracle."""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _inputs(n, c, h, w, k, r, s, seed):
    rng = np.random.default_rng(seed)
    x = rng.standard_normal((n, c, h, w)).astype(np.float16)
    wt = (rng.standard_normal((k, c, r, s)) / np.sqrt(c * r * s)).astype(np.float16)
    return x, wt


def _check(y, x, wt, stride, pad):
    """Against the oracle's FP64 direct convolution (oracle/conv_oracle.c)."""
    import oracle
    y64 = oracle.conv2d_f64(x.cpu().numpy(), wt.cpu().numpy(), u=stride, v=stride, p=pad, q=pad)
    yh = y.cpu().numpy().astype(np.float64)
    assert yh.shape == y64.shape
    d = yh - y64
    rl2 = float(np.linalg.norm(d) / np.linalg.norm(y64))
    mxn = float(np.abs(d).max() / np.abs(y64).max())
    assert rl2 <= 2e-3 and mxn <= 1e-2, (rl2, mxn)


SHAPES = [  # n, c, h, w, k, r, s, stride, pad
    (2, 64, 14, 14, 256, 1, 1, 1, 0),     # 1x1 expansion, one 256-row k-block
    (3, 256, 14, 14, 64, 1, 1, 2, 0),     # 1x1 stride-2 projection, two pixel halves (K <= 128)
    (4, 64, 28, 28, 128, 3, 3, 2, 1),     # stride-2 3x3 downsampling
    (2, 128, 15, 15, 320, 3, 3, 2, 1),    # odd input, two k-blocks (256 + 64 rows)
    (3, 24, 11, 7, 40, 3, 3, 1, 1),       # C, K not multiples of 16 (zero-padded K-steps and rows)
    (2, 48, 10, 12, 24, 5, 5, 1, 2),      # 5x5 (extension API only: its weights exceed transform_filter)
    (2, 3, 32, 32, 64, 7, 7, 2, 3),       # stem 7x7 stride 2, C = 3
    (1, 16, 9, 9, 16, 3, 3, 1, 0),        # pad 0, one unit, one K-step a tap
    (3, 32, 7, 7, 48, 1, 3, 1, 0),        # 1x3 filter, 147 pixels (a partial unit)
    # 1x1 / stride 1 / pad 0 with H * W % 8 == 0: pixel octets by 16-byte loads
    (2, 24, 16, 16, 40, 1, 1, 1, 0),      # ragged C and K, two pixel halves
    (3, 64, 28, 28, 320, 1, 1, 1, 0),     # two k-blocks, 2352 pixels (a partial unit)
    (1, 512, 8, 12, 128, 1, 1, 1, 0),     # 32 K-steps, one partial unit
    (2, 32, 16, 16, 160, 1, 1, 1, 0),     # H * W % 64 == 0, K > 128: TMA boxes (map in transform_pin)
    # more 2-byte-gather cases: strides, paddings and row lengths
    (2, 64, 16, 16, 128, 3, 3, 2, 1),     # stride-2 3x3, 8-column output rows
    (2, 32, 8, 24, 48, 1, 1, 2, 0),       # stride-2 1x1, 12-column output rows
    (1, 24, 10, 16, 40, 3, 3, 1, 1),      # stride 1, ragged C and K
    (3, 16, 9, 8, 16, 3, 3, 1, 0),        # pad 0, 6-column output rows, odd H
    (2, 48, 16, 16, 24, 5, 5, 1, 2),      # 5x5 (extension API only)
    (2, 32, 16, 40, 320, 3, 3, 2, 1),     # two k-blocks, 20-column output rows
]


@pytest.mark.parametrize("shape", SHAPES)
def test_igemm_conv(wino, cuda, shape):
    import torch
    n, c, h, w, k, r, s, stride, pad = shape
    x16, w16 = _inputs(n, c, h, w, k, r, s, seed=sum(shape))
    x, wt = torch.from_numpy(x16).to(cuda), torch.from_numpy(w16).to(cuda)
    y = wino.conv2d_igemm(x, wt, stride=stride, pad=pad)
    torch.cuda.synchronize()
    assert wino.error_read_clear() == 0
    _check(y, x, wt, stride, pad)


def _weights_layout_np(w16):
    """The implicit GEMM's weight operand as igemm_weight_kernel writes it:
    k-blocks of 256 output channels, then K-steps (tap-major, 16 channels
    each), each K-step rows x 32 bytes with output channel row, channel cc at
    (row >> 3) * 256 + (cc >> 3) * 128 + (row & 7) * 16 + (cc & 7) * 2; zeros
    past K and C."""
    K, C, R, S = w16.shape
    CB = (C + 15) // 16
    NKS = R * S * CB
    Kp = (K + 15) // 16 * 16
    out = np.zeros(Kp * NKS * 16, np.float16)
    k, ks, cc = np.meshgrid(np.arange(Kp), np.arange(NKS), np.arange(16), indexing="ij")
    kb, row = k // 256, k % 256
    rows = np.minimum(256, Kp - kb * 256)
    tap, cb = ks // CB, ks % CB
    r, s_ = tap // S, tap % S
    c = cb * 16 + cc
    byte = (kb * 256 * NKS * 32 + ks * rows * 32 + (row >> 3) * 256 + (cc >> 3) * 128
            + (row & 7) * 16 + (cc & 7) * 2)
    ok = (k < K) & (c < C)
    wpad = np.zeros((Kp, max(C, CB * 16), R, S), np.float16)
    wpad[:K, :C] = w16
    out[byte // 2] = np.where(ok, wpad[np.minimum(k, Kp - 1), np.minimum(c, wpad.shape[1] - 1), r, s_], 0)
    return out


@pytest.mark.parametrize("k,c,r,s", [(40, 24, 3, 3), (320, 64, 1, 1), (48, 3, 7, 7), (16, 16, 1, 3)])
def test_igemm_weight_layout_bit_exact(wino, cuda, k, c, r, s):
    """igemm_weight_transform writes exactly the documented operand layout."""
    import torch
    rng = np.random.default_rng(k * 7 + c)
    w16 = rng.standard_normal((k, c, r, s)).astype(np.float16)
    wp = wino.igemm_weight_transform(torch.from_numpy(w16).to(cuda))
    torch.cuda.synchronize()
    want = _weights_layout_np(w16)
    got = wp.cpu().numpy()[:want.size * 2].view(np.float16)   # the operand, before the map slot
    assert got.shape == want.shape
    assert np.array_equal(got.view(np.uint16), want.view(np.uint16))


def _route(wino, x, wt, y, ws, stride, pad):
    r, s = wt.shape[2:]
    pr = wino.make_problem(x, wt, y, ws.transform_pin, ws.transform_filter, ws.mid_result,
                           r=r, s=s, u=stride, v=stride, p=pad, q=pad)
    return wino.lib().wino_dropin_route(ctypes.byref(pr))


@pytest.mark.parametrize("shape", [sh for sh in SHAPES if sh[5] * sh[6] * ((sh[1] + 15) // 16) * ((sh[4] + 15) // 16 * 16)
                                   <= sh[4] * sh[1]])
def test_dropin_takes_igemm(wino, cuda, shape):
    """getkernelInfo routes these shapes to the implicit GEMM (route 4) with
    the caller's workspaces sized as the reference harness sizes them."""
    import torch
    n, c, h, w, k, r, s, stride, pad = shape
    x16, w16 = _inputs(n, c, h, w, k, r, s, seed=11 + sum(shape))
    x, wt = torch.from_numpy(x16).to(cuda), torch.from_numpy(w16).to(cuda)
    ws = wino.DropinWorkspaces(n, c, h, w, k, x.device, True)
    oh, ow = (h - r + 2 * pad) // stride + 1, (w - s + 2 * pad) // stride + 1
    probe = torch.empty((n, k, oh, ow), dtype=torch.float16, device=cuda)
    assert _route(wino, x, wt, probe, ws, stride, pad) == 4
    y = wino.dropin_conv2d(x, wt, ws=ws, stride=stride, pad=pad)
    torch.cuda.synchronize()
    assert wino.error_read_clear() == 0
    _check(y, x, wt, stride, pad)


def test_igemm_persistent_many_units(wino, cuda):
    """784 units of 128 pixels on at most 148 CTAs: every CTA runs several
    units, so the stage ring and both accumulator buffers wrap."""
    import torch
    n, c, h, w, k = 32, 64, 56, 56, 256
    x16, w16 = _inputs(n, c, h, w, k, 1, 1, seed=5)
    x, wt = torch.from_numpy(x16).to(cuda), torch.from_numpy(w16).to(cuda)
    y = wino.conv2d_igemm(x, wt, stride=1, pad=0)
    torch.cuda.synchronize()
    assert wino.error_read_clear() == 0
    _check(y, x, wt, 1, 0)


def test_igemm_stride2_persistent_many_units(wino, cuda):
    """Stride-2 3x3 on 56x56 at N64 (K <= 128: two pixel halves a unit): 196
    units of 256 pixels on at most 148 CTAs."""
    import torch
    n, c, h, w, k = 64, 64, 56, 56, 64
    x16, w16 = _inputs(n, c, h, w, k, 3, 3, seed=6)
    x, wt = torch.from_numpy(x16).to(cuda), torch.from_numpy(w16).to(cuda)
    y = wino.conv2d_igemm(x, wt, stride=2, pad=1)
    torch.cuda.synchronize()
    assert wino.error_read_clear() == 0
    _check(y, x, wt, 2, 1)


def test_igemm_weights_reused_and_matches_direct(wino, cuda):
    """One weight re-layout serves repeated calls; the result agrees with the
    CUDA-core direct kernel to fp16 rounding."""
    import torch
    n, c, h, w, k = 4, 128, 28, 28, 128
    x16, w16 = _inputs(n, c, h, w, k, 3, 3, seed=9)
    x, wt = torch.from_numpy(x16).to(cuda), torch.from_numpy(w16).to(cuda)
    wp = wino.igemm_weight_transform(wt)
    y1 = wino.conv2d_igemm(x, wt, stride=2, pad=1, wprep=wp)
    y2 = wino.conv2d_igemm(x, wt, stride=2, pad=1, wprep=wp)
    yd = wino.conv2d_direct(x, wt, stride=2, pad=1)
    torch.cuda.synchronize()
    assert wino.error_read_clear() == 0
    assert torch.equal(y1, y2)
    d = (y1.double() - yd.double()).norm() / yd.double().norm()
    assert float(d) <= 2e-3
    _check(y1, x, wt, 2, 1)
