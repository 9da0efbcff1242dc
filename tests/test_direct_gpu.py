"""General shapes (any filter size, stride, padding, channel count) through
the CUDA-core direct kernel, and behind the drop-in ABI (which runs them on
the tensor-core implicit GEMM when its weights fit transform_filter, else on
the direct kernel), against FP64 (rel-L2 <= 2e-3, max-normalised <= 1e-2)."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _inputs(oracle_mod, n, c, h, w, k, r, seed):
    rng = np.random.default_rng(seed)
    x = rng.standard_normal((n, c, h, w)).astype(np.float16)
    wt = (rng.standard_normal((k, c, r, r)) / np.sqrt(c * r * r)).astype(np.float16)
    return x, wt


def _check(y, x, wt, stride, pad):
    import torch
    y64 = torch.nn.functional.conv2d(x.double(), wt.double(), stride=stride, padding=pad)
    assert tuple(y.shape) == tuple(y64.shape)
    d = y.double() - y64
    rl2 = float(torch.linalg.vector_norm(d) / torch.linalg.vector_norm(y64))
    mxn = float(d.abs().max() / y64.abs().max())
    assert rl2 <= 2e-3 and mxn <= 1e-2, (rl2, mxn)


SHAPES = [  # n, c, h, w, k, r, stride, pad
    (2, 3, 32, 32, 16, 7, 2, 3),      # stem-style 7x7 stride 2
    (4, 64, 28, 28, 128, 3, 2, 1),    # stride-2 downsampling
    (2, 32, 14, 14, 64, 1, 1, 0),     # 1x1
    (2, 16, 10, 12, 24, 5, 1, 2),     # 5x5, K not a multiple of 16
    (1, 8, 9, 9, 8, 3, 1, 0),         # pad 0
    (3, 24, 11, 7, 40, 3, 1, 1),      # 3x3 s1 p1 but C, K not multiples of 16
]


@pytest.mark.parametrize("shape", SHAPES)
def test_direct_conv(wino, cuda, oracle_mod, shape):
    import torch
    n, c, h, w, k, r, stride, pad = shape
    x16, w16 = _inputs(oracle_mod, n, c, h, w, k, r, seed=sum(shape))
    x, wt = torch.from_numpy(x16).to(cuda), torch.from_numpy(w16).to(cuda)
    y = wino.conv2d_direct(x, wt, stride=stride, pad=pad)
    torch.cuda.synchronize()
    _check(y, x, wt, stride, pad)


@pytest.mark.parametrize("shape", SHAPES)
def test_dropin_general_shapes(wino, cuda, oracle_mod, shape):
    """getkernelInfo accepts these shapes and its four slots compute them
    (route 4 or the direct route, whichever it picks)."""
    import torch
    n, c, h, w, k, r, stride, pad = shape
    x16, w16 = _inputs(oracle_mod, n, c, h, w, k, r, seed=7 + sum(shape))
    x, wt = torch.from_numpy(x16).to(cuda), torch.from_numpy(w16).to(cuda)
    y = wino.dropin_conv2d(x, wt, stride=stride, pad=pad)
    torch.cuda.synchronize()
    _check(y, x, wt, stride, pad)


def test_direct_matches_winograd_shape(wino, cuda, oracle_mod):
    import torch
    x16, w16 = oracle_mod.make_inputs(2, 64, 14, 14, 64, seed=3, x_dist="normal")
    x, wt = torch.from_numpy(x16).to(cuda), torch.from_numpy(w16).to(cuda)
    yd = wino.conv2d_direct(x, wt)
    yw = wino.conv2d(x, wt)
    torch.cuda.synchronize()
    _check(yd, x, wt, 1, 1)
    d = (yd.double() - yw.double()).norm() / yw.double().norm()
    assert float(d) <= 2e-3
    assert wino.error_read_clear() == 0
