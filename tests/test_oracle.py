"""CPU tests of the oracle: pinned against the reference's own conv2dcpu
outputs (tests/golden), cross-checked against torch fp64, and the NumPy
Winograd restatement checked against the direct convolution."""
import numpy as np
import pytest

from conftest import golden_cases, load_golden


@pytest.mark.parametrize("path", golden_cases(), ids=lambda p: p.rsplit("/", 1)[-1])
def test_oracle_matches_reference_golden_bit_exact(oracle_mod, path):
    x, w, y_ref = load_golden(path)
    y64 = oracle_mod.conv2d_f64(x, w)
    # The reference stores (_Float16)sum of the same double sum: bit-exact.
    assert np.array_equal(y64.astype(np.float16), y_ref)


def test_oracle_agrees_with_torch_float64(oracle_mod):
    import torch
    x, w = oracle_mod.make_inputs(2, 32, 9, 11, 48, seed=11, x_dist="normal")
    y64 = oracle_mod.conv2d_f64(x, w)
    yt = torch.nn.functional.conv2d(torch.from_numpy(x.astype(np.float64)),
                                    torch.from_numpy(w.astype(np.float64)), padding=1).numpy()
    assert np.max(np.abs(yt - y64)) <= 1e-12 * max(1.0, np.max(np.abs(y64)))


@pytest.mark.parametrize("shape", [(1, 16, 7, 7, 16), (2, 32, 8, 6, 16), (1, 16, 1, 3, 32)])
def test_winograd_restatement_is_exact(oracle_mod, shape):
    from oracle import winograd as W
    n, c, h, w, k = shape
    x, wt = oracle_mod.make_inputs(n, c, h, w, k, seed=3)
    y64 = oracle_mod.conv2d_f64(x, wt)
    yw = W.conv2d_winograd_f64(x, wt)
    assert np.max(np.abs(yw - y64)) <= 1e-12 * np.max(np.abs(y64))


@pytest.mark.parametrize("dist", ["uniform", "normal", "student_t3", "relu_normal"])
def test_fp16_winograd_error_budget(oracle_mod, dist):
    """The rounding points of the fp16 kernel (U, V rounded once to fp16, fp32
    accumulation, fp16 output) stay inside the rel-L2 <= 2e-3 target."""
    from oracle import winograd as W
    x, w = oracle_mod.make_inputs(2, 64, 14, 14, 32, seed=5, x_dist=dist)
    y64 = oracle_mod.conv2d_f64(x, w)
    ye = W.conv2d_winograd_emulated(x, w, "f16").astype(np.float16)
    assert oracle_mod.rel_l2(ye, y64) < 2e-3


def test_reference_check_rule_detects_planted_error(oracle_mod):
    x, w = oracle_mod.make_reference_style_inputs(1, 16, 6, 6, 16, seed=2)
    y = oracle_mod.conv2d_f64(x, w).astype(np.float16)
    assert oracle_mod.reference_check(y, y) == 0
    bad = y.copy()
    bad.flat[17] = np.float16(float(bad.flat[17]) * 1.05)  # planted 5% error
    assert oracle_mod.reference_check(bad, y) == 1


@pytest.mark.parametrize("n,c,h,w,k,r,s,u,v,p,q", [
    (2, 16, 9, 9, 16, 3, 3, 2, 2, 1, 1),      # stride-2 3x3
    (2, 24, 8, 10, 16, 1, 1, 2, 2, 0, 0),     # stride-2 1x1 projection
    (1, 3, 16, 16, 8, 7, 7, 2, 2, 3, 3),      # 7x7 stem
    (1, 16, 7, 9, 8, 5, 5, 1, 1, 2, 2),       # 5x5
    (2, 16, 6, 8, 8, 1, 3, 1, 1, 0, 1),       # 1x3, different row / column padding
])
def test_oracle_matches_reference_general_shapes_bit_exact(oracle_mod, n, c, h, w, k, r, s, u, v, p, q):
    """The implicit GEMM's and the direct kernel's checker: the oracle equals
    the reference's own conv2dcpu (built unmodified) bit for bit on filter
    sizes, strides and paddings outside the Winograd contract as well."""
    x, wt = oracle_mod.make_inputs(n, c, h, w, k, seed=n + c + h + k, x_dist="normal", r=r, s=s)
    y64 = oracle_mod.conv2d_f64(x, wt, u=u, v=v, p=p, q=q)
    y_ref = oracle_mod.ref_conv2dcpu(x, wt, u=u, v=v, p=p, q=q, threads=1)
    assert y64.shape == y_ref.shape
    assert np.array_equal(y64.astype(np.float16), y_ref)


def test_reference_cpu_multithreaded_matches_single(oracle_mod):
    x, w = oracle_mod.make_inputs(4, 16, 6, 6, 16, seed=9)
    a = oracle_mod.ref_conv2dcpu(x, w, threads=1)
    b = oracle_mod.ref_conv2dcpu(x, w, threads=4)
    assert np.array_equal(a, b)


def test_e4m3_rounding_known_values():
    """fp8 e4m3 rounding of the variant model: nearest-even on a 3-bit
    mantissa, subnormal step 2^-9, saturation at 448."""
    from oracle.winograd import _e4m3
    vals = np.array([1.0, 1.0625, 1.1875, -1.0625, 448.0, 500.0, 2.0 ** -9, 2.0 ** -10 * 1.5,
                     0.0, 240.0, 0.017578125])
    want = np.array([1.0, 1.0, 1.25, -1.0, 448.0, 448.0, 2.0 ** -9, 2.0 ** -9, 0.0, 240.0, 0.017578125])
    assert np.array_equal(_e4m3(vals), want)


@pytest.mark.parametrize("shape", [(1, 16, 9, 7, 16), (2, 16, 4, 5, 32), (1, 32, 1, 1, 16), (1, 16, 13, 12, 16)])
def test_winograd_f4_restatement_is_exact(oracle_mod, shape):
    """F(4x4,3x3) in fp64 equals the direct conv, ragged tiles included."""
    from oracle import winograd_f4 as F4
    n, c, h, w, k = shape
    x, wt = oracle_mod.make_inputs(n, c, h, w, k, seed=4)
    y64 = oracle_mod.conv2d_f64(x, wt)
    assert np.max(np.abs(F4.conv2d_f4_f64(x, wt) - y64)) <= 1e-12 * np.max(np.abs(y64))


@pytest.mark.parametrize("dist", ["uniform", "relu_normal", "student_t3"])
def test_winograd_f4_error_columns(oracle_mod, dist):
    """F(4x4) with single fp16 U and V misses the 2e-3 target (transform
    coefficients up to 5, 1/24 and 8); the hi+lo pieces bring it to the fp16
    output-rounding floor, below F(2x2)'s fp16 error."""
    from oracle import winograd as W, winograd_f4 as F4
    x, w = oracle_mod.make_inputs(2, 64, 20, 20, 32, seed=6, x_dist=dist)
    y64 = oracle_mod.conv2d_f64(x, w)
    plain = oracle_mod.rel_l2(F4.conv2d_f4_emulated(x, w, hilo=False).astype(np.float16), y64)
    hilo = oracle_mod.rel_l2(F4.conv2d_f4_emulated(x, w, hilo=True).astype(np.float16), y64)
    f2 = oracle_mod.rel_l2(W.conv2d_winograd_emulated(x, w, "f16").astype(np.float16), y64)
    floor = oracle_mod.rel_l2(y64.astype(np.float16), y64)
    assert plain > 2e-3
    assert hilo < 1.2 * floor < f2


def test_winograd_f4_hilo_split():
    from oracle import winograd_f4 as F4
    a = np.array([1 / 3, -1 / 6, 1e-3 / 7, 1234.567, 0.0])
    hi, lo = F4.split_hilo(a)
    assert np.all(hi.astype(np.float16).astype(np.float64) == hi)
    # lo's own rounding: half an fp16 step of |a - hi| <= 2^-12 |a|, or half
    # the fp16 subnormal step 2^-24 where lo is subnormal
    assert np.all(np.abs(hi + lo - a.astype(np.float32)) <= np.maximum(2.0 ** -22 * np.abs(a), 2.0 ** -25))


@pytest.mark.parametrize("shape", [(1, 16, 6, 6), (2, 32, 5, 7), (1, 16, 9, 4)])
def test_blocked_input_window_words_give_v(oracle_mod, shape):
    """Layout contract of the two-stage producers: tap (a, b) of tile (n, ty,
    tx) reads, from the blocked input XB[n][c/16][r][par][hh][e][8], the words
    at rows 2ty + i (i in the tap row's pair) and columns 2tx - 1 + jc (jc in
    the tap column's pair; parity (jc & 1) ^ 1, entry tx + (jc >> 1)), and
    two fp16 +- steps (rows, then columns) give the fused kernel's V bit for
    bit."""
    from oracle import winograd as W
    from test_fused_gpu import _xb_layout_np
    n, c, h, w = shape
    x, _ = oracle_mod.make_inputs(n, c, h, w, 16, seed=7, x_dist="normal")
    xb = _xb_layout_np(x)                                      # [n][cb][r][par][hh][e][8]
    tp, tq = (h + 1) // 2, (w + 1) // 2
    pick = {0: (0, 2, 0), 1: (1, 2, 1), 2: (1, 2, 2), 3: (1, 3, 0)}   # (i0, i1, op)

    def op(o, x0, x1):
        r = x0 - x1 if o == 0 else (x0 + x1 if o == 1 else x1 - x0)
        return r.astype(np.float16).astype(np.float32)

    vref = W.input_transform_f16(x).astype(np.float16)        # [16][tiles][C]
    for tile in range(n * tp * tq):
        nn, r = divmod(tile, tp * tq)
        ty, tx = divmod(r, tq)
        for t in range(16):
            i0, i1, opa = pick[t >> 2]
            j0, j1, opb = pick[t & 3]
            word = lambda i, jc: xb[nn, :, 2 * ty + i, (jc & 1) ^ 1, :, tx + (jc >> 1), :].astype(np.float32)
            e0 = op(opa, word(i0, j0), word(i1, j0))
            e1 = op(opa, word(i0, j1), word(i1, j1))
            v = op(opb, e0, e1).astype(np.float16).reshape(-1)   # channel order cb, hh, 8
            assert np.array_equal(v.view(np.uint16), vref[t, tile].view(np.uint16)), (tile, t)
