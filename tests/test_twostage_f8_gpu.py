"""fp8 two-stage path (wino_conv2d_twostage_f8).  hilo: U and V each split
into e4m3 hi + lo, the tap GEMM on kind::f8f6f4 accumulating hi.hi + lo.hi +
hi.lo -- checked against FP64 within the 2e-2 an fp8 GEMM stage is held to
(the split keeps it near the fp16 path's ~1e-3); single terms: one e4m3 MMA
per step -- within single-term fp8's 8e-2.  Both against the NumPy model of
their rounding points (oracle/winograd.py
conv2d_winograd_f8_twostage_emulated) on odd sizes, partial tile blocks, a
partial k pair, K beyond one k pair and several input distributions."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

FP64_TOL = {True: 2e-2, False: 8e-2}
MODEL_TOL = {True: 2e-3, False: 1e-2}


def _run(wino, cuda, x16, w16, hilo=True):
    import torch
    k = w16.shape[0]
    x = torch.from_numpy(x16).to(cuda)
    wt = torch.from_numpy(w16).to(cuda)
    u2 = wino.filter_transform_unfused(wt)
    y = wino.conv2d_twostage_f8(x, u2, k, hilo=hilo)
    torch.cuda.synchronize()
    assert wino.error_read_clear() == 0
    return y.cpu().numpy()


@pytest.mark.parametrize("hilo", [True, False])
@pytest.mark.parametrize("shape", [(2, 32, 12, 10, 32), (3, 64, 9, 7, 48), (1, 96, 6, 8, 272),
                                   (2, 256, 14, 14, 256), (1, 32, 1, 1, 16)])
def test_twostage_f8_against_fp64_and_model(wino, cuda, oracle_mod, shape, hilo):
    from oracle import winograd as W
    n, c, h, w, k = shape
    x16, w16 = oracle_mod.make_inputs(n, c, h, w, k, seed=11, x_dist="normal", w_std=np.sqrt(2.0 / (9 * c)))
    y = _run(wino, cuda, x16, w16, hilo)
    assert np.isfinite(y.astype(np.float32)).all()
    y64 = oracle_mod.conv2d_f64(x16, w16)
    assert oracle_mod.rel_l2(y, y64) <= FP64_TOL[hilo], oracle_mod.rel_l2(y, y64)
    assert oracle_mod.max_norm(y, y64) <= FP64_TOL[hilo], oracle_mod.max_norm(y, y64)
    ym = W.conv2d_winograd_f8_twostage_emulated(x16, w16, hilo)
    assert oracle_mod.rel_l2(y, ym) <= MODEL_TOL[hilo], oracle_mod.rel_l2(y, ym)


@pytest.mark.parametrize("dist", ["uniform", "normal", "student_t3"])
def test_twostage_f8_precision_sweep(wino, cuda, oracle_mod, dist):
    """The precision sweep's distributions (N64 C=K256 H14 in the bench; a
    smaller batch here): the fp8 hi+lo path stays within 2e-2 of FP64."""
    x16, w16 = oracle_mod.make_inputs(8, 256, 14, 14, 256, seed=0, x_dist=dist, w_std=np.sqrt(2.0 / (9 * 256)))
    y = _run(wino, cuda, x16, w16)
    y64 = oracle_mod.conv2d_f64(x16, w16)
    assert oracle_mod.rel_l2(y, y64) <= FP64_TOL[True]
    assert oracle_mod.max_norm(y, y64) <= FP64_TOL[True]


