"""Two-stage F(2x2,3x3) path (input transform fused into the tap GEMMs, fp16
M, separate output transform) against the oracle.

Bars: rel-L2 <= 2e-3 and max-normalised <= 1e-2 against FP64, the fp16 bar of
the path.  The path's rounding points are those of the unfused comparator
(U and V rounded to fp16 as in the fused kernel, fp32 accumulation, M rounded
to fp16, fp32 output transform), so its output is also compared with the
NumPy model of those steps and with the unfused comparator itself.
"""
import numpy as np
import pytest

from conftest import golden_cases, load_golden

pytestmark = pytest.mark.gpu

REL_L2 = 2e-3
MAX_NORM = 1e-2


def _t(a, dev):
    import torch
    return torch.from_numpy(np.ascontiguousarray(a)).to(dev)


def _twostage(wino, x16, w16, dev):
    import torch
    x, w = _t(x16, dev), _t(w16, dev)
    u2 = wino.filter_transform_unfused(w)
    y = wino.conv2d_twostage(x, u2, w.shape[0])
    torch.cuda.synchronize()
    assert wino.error_read_clear() == 0
    return y.cpu().numpy()


def _model(x16, w16):
    """U rounded once, V in packed fp16 (oracle.winograd.input_transform_f16),
    fp32 accumulation, M rounded to fp16, output transform, fp16 Y."""
    from oracle import winograd as W
    n, c, h, wd = x16.shape
    k = w16.shape[0]
    u = W._f16(W.filter_transform(w16))
    v = W.input_transform_f16(x16)
    m = W._f16(W.gemm(u, v).astype(np.float32))
    return W.output_transform(m, n, k, h, wd).astype(np.float16)


def _check(oracle_mod, y, y64, what):
    rl2, mxn = oracle_mod.rel_l2(y, y64), oracle_mod.max_norm(y, y64)
    assert np.isfinite(y.astype(np.float32)).all(), what
    assert rl2 <= REL_L2, f"{what} rel_l2={rl2:.3e}"
    assert mxn <= MAX_NORM, f"{what} max_norm={mxn:.3e}"


@pytest.mark.parametrize("shape", [
    (1, 16, 3, 5, 16),      # tiny, odd width
    (2, 32, 12, 10, 32),
    (3, 48, 9, 7, 144),     # C = 48 (3 K-steps), K = 128 + 16: a short second k-block
    (1, 16, 1, 1, 16),      # one pixel
    (2, 64, 14, 14, 256),   # two full k-blocks per unit
    (1, 32, 30, 2, 16),     # tall and narrow
    (5, 16, 40, 40, 48),    # several tile blocks, last one partial
    (1, 80, 8, 8, 384),     # C = 80 (5 K-steps: a partial stage), three k-blocks
    (2, 256, 10, 6, 64),    # C = 256: the largest U the tap-pair kernel keeps resident
    (2, 272, 6, 8, 48),     # C = 272: the streamed-U kernel
    (1, 512, 5, 4, 272),    # C = 512, K = 272 on the streamed-U kernel
])
def test_twostage_shapes(wino, cuda, oracle_mod, shape):
    n, c, h, w, k = shape
    x, wt = oracle_mod.make_inputs(n, c, h, w, k, seed=sum(shape) + 1, x_dist="normal")
    y = _twostage(wino, x, wt, cuda)
    _check(oracle_mod, y, oracle_mod.conv2d_f64(x, wt), str(shape))
    ym = _model(x, wt).astype(np.float64)
    assert oracle_mod.rel_l2(y, ym) <= 2e-4, shape


@pytest.mark.parametrize("path", golden_cases(), ids=lambda p: p.rsplit("/", 1)[-1])
def test_twostage_vs_reference_golden(wino, cuda, oracle_mod, path):
    x, w, y_ref = load_golden(path)
    y = _twostage(wino, x, w, cuda)
    _check(oracle_mod, y, oracle_mod.conv2d_f64(x, w), path)
    assert oracle_mod.rel_l2(y, y_ref.astype(np.float64)) <= REL_L2


@pytest.mark.parametrize("c", [64, 288])
def test_twostage_matches_unfused_comparator(wino, cuda, oracle_mod, c):
    """Same operands (V formed with the same fp16 operations), the same
    K-step accumulation order and the same rounding points as the unfused
    comparator: the outputs are bit-identical, on the GEMM the build routes
    C = 64 to and on the streamed-U kernel (C = 288)."""
    import torch
    n, h, w, k = 4, 14, 14, 128
    x16, w16 = oracle_mod.make_inputs(n, c, h, w, k, seed=9, x_dist="relu_normal")
    x, wt = _t(x16, cuda), _t(w16, cuda)
    u2 = wino.filter_transform_unfused(wt)
    ys = wino.conv2d_twostage(x, u2, k)
    ws = wino.UnfusedWorkspace(n, c, h, w, k, cuda)
    yu = wino.conv2d_unfused(x, u2, k, ws=ws)
    torch.cuda.synchronize()
    assert torch.equal(ys, yu)


def test_twostage_large_layer(wino, cuda, oracle_mod):
    """N=128 C=K=256 H=W=28, x = ReLU(N(0,1)), w ~ N(0, 2/(9C))."""
    import torch
    x16, w16 = oracle_mod.make_inputs(128, 256, 28, 28, 256, seed=0, x_dist="relu_normal",
                                      w_std=np.sqrt(2.0 / (9 * 256)))
    x, wt = _t(x16, cuda), _t(w16, cuda)
    y = wino.conv2d_twostage(x, wino.filter_transform_unfused(wt), 256)
    torch.cuda.synchronize()
    assert wino.error_read_clear() == 0
    y64 = torch.nn.functional.conv2d(x.double(), wt.double(), padding=1)
    rl2 = float(torch.linalg.vector_norm(y.double() - y64) / torch.linalg.vector_norm(y64))
    mxn = float((y.double() - y64).abs().max() / y64.abs().max())
    assert rl2 <= REL_L2 and mxn <= MAX_NORM, (rl2, mxn)


def test_dropin_large_layer_two_stage_route(wino, cuda, oracle_mod):
    """N=128 C=K=256 H=W=28 through the drop-in ABI, which takes the
    two-stage route for this shape."""
    import torch
    x16, w16 = oracle_mod.make_inputs(128, 256, 28, 28, 256, seed=1, x_dist="relu_normal",
                                      w_std=np.sqrt(2.0 / (9 * 256)))
    x, wt = _t(x16, cuda), _t(w16, cuda)
    y = wino.dropin_conv2d(x, wt)
    torch.cuda.synchronize()
    assert wino.error_read_clear() == 0
    y64 = torch.nn.functional.conv2d(x.double(), wt.double(), padding=1)
    rl2 = float(torch.linalg.vector_norm(y.double() - y64) / torch.linalg.vector_norm(y64))
    mxn = float((y.double() - y64).abs().max() / y64.abs().max())
    assert rl2 <= REL_L2 and mxn <= MAX_NORM, (rl2, mxn)


@pytest.mark.parametrize("shape", [(2, 32, 12, 10, 32), (1, 16, 2, 2, 16), (3, 48, 16, 6, 144)])
def test_dropin_two_stage_route(wino, cuda, oracle_mod, shape):
    """Even H and W: getkernelInfo fills the four slots with the U2 filter
    transform, the pre-pass, the two-stage GEMM and the output transform
    (M in the caller's mid_result), and the result equals the extension
    entry point's.  The 2x2 image has one tile: its transformed tiles (V2,
    tiles rounded up to 8) do not fit the harness's transform_pin when the
    build reads V2, and getkernelInfo takes the fused route after the
    pre-pass instead."""
    import ctypes
    import torch
    n, c, h, w, k = shape
    x, wt = oracle_mod.make_inputs(n, c, h, w, k, seed=3, x_dist="uniform")
    xt, wtt = _t(x, cuda), _t(wt, cuda)
    ws = wino.DropinWorkspaces(n, c, h, w, k, cuda)
    y = torch.empty((n, k, h, w), dtype=torch.float16, device=cuda)
    pr = wino.make_problem(xt, wtt, y, ws.transform_pin, ws.transform_filter, ws.mid_result)
    param = (ctypes.c_char * 80)()
    rc, ki = wino.get_kernel_info(pr, param)
    assert rc == 0
    L = wino.lib()
    fits = L.wino_twostage_prepass_bytes(n, c, h, w) <= 4 * h * h * n * c * 2
    if not fits:
        assert L.wino_dropin_route(ctypes.byref(pr)) == 2
        y2 = wino.dropin_conv2d(xt, wtt, ws=ws)
        torch.cuda.synchronize()
        assert wino.error_read_clear() == 0
        _check(oracle_mod, y2.cpu().numpy(), oracle_mod.conv2d_f64(x, wt), str(shape))
        return
    assert ki.slot(3)["kernel"] == L.wino_twostage_gemm_kernel_ptr_for(c)
    assert ki.slot(4)["kernel"] == L.wino_twostage_output_kernel_ptr()
    y2 = wino.dropin_conv2d(xt, wtt, ws=ws)
    y3 = wino.conv2d_twostage(xt, wino.filter_transform_unfused(wtt), k)
    torch.cuda.synchronize()
    assert wino.error_read_clear() == 0
    assert torch.equal(y2, y3)
    _check(oracle_mod, y2.cpu().numpy(), oracle_mod.conv2d_f64(x, wt), str(shape))


def _xr_layout_np(x16):
    """NumPy statement of the row-transformed records the pre-pass of the
    resident-U and tap-pair kernels writes: XR[n][c/16][ty][a][par][hh][e][8] with
    R_a(ty, x) = fp16(s0 * X(2ty - 1 + i0, x) + s1 * X(2ty - 1 + i1, x)) for
    B^T row a = s0 * d_i0 + s1 * d_i1 (one rounding of the exact two-term
    sum), par 0 entry e = column 2e, par 1 entry e = column 2e - 1, zero
    outside the image."""
    from oracle import winograd as W
    n, c, h, w = x16.shape
    tp, tq = (h + 1) // 2, (w + 1) // 2
    e = tq + 1
    pad = np.zeros((n, c, 2 * tp + 2, 2 * e + 1), np.float64)   # rows -1 .. 2tp, cols -1 .. 2e-1
    pad[:, :, 1:h + 1, 1:w + 1] = x16.astype(np.float64)
    win = np.stack([pad[:, :, 2 * t:2 * t + 4] for t in range(tp)], axis=2)   # n c ty i col
    r = np.einsum("ai,nctix->nctax", W.BT, win).astype(np.float16)            # n c ty a col
    out = np.zeros((n, c // 16, tp, 4, 2, 2, e, 8), np.float16)
    v = r.reshape(n, c // 16, 2, 8, tp, 4, 2 * e + 1)                         # n cb hh ci ty a col
    out[:, :, :, :, 0] = v[..., 2 * np.arange(e) + 1].transpose(0, 1, 4, 5, 2, 6, 3)
    out[:, :, :, :, 1] = v[..., 2 * np.arange(e)].transpose(0, 1, 4, 5, 2, 6, 3)
    return out


@pytest.mark.parametrize("shape", [(2, 32, 12, 10), (1, 16, 9, 7), (3, 48, 1, 1), (1, 16, 28, 28)])
def test_twostage_row_prepass_bit_exact(wino, cuda, oracle_mod, shape):
    """The row-transformed pre-pass (stage 0 of conv2d_twostage when the
    build routes C to the resident-U or tap-pair kernel) writes exactly the
    NumPy statement of its records."""
    import torch
    n, c, h, w = shape
    L = wino.lib()
    if L.wino_twostage_gemm_kernel_ptr_for(c) not in (L.wino_twostage_pair_kernel_ptr(),
                                                      L.wino_twostage_res_kernel_ptr()):
        pytest.skip("this build routes C to the streamed-U kernel")
    k = 16
    x16, _ = oracle_mod.make_inputs(n, c, h, w, k, seed=5, x_dist="normal")
    ref = _xr_layout_np(x16)
    nb = wino.twostage_workspace_bytes(n, c, h, w, k)
    ws = wino._aligned_ws(nb, cuda)
    ws.fill_(0xA5)                                                 # poison
    x = _t(x16, cuda)
    u2 = torch.zeros(16 * k * c, dtype=torch.float16, device=cuda)
    y = torch.empty((n, k, h, w), dtype=torch.float16, device=cuda)
    wino.twostage_stage(0, x, u2, k, y, ws)
    torch.cuda.synchronize()
    got = ws[:ref.nbytes].cpu().numpy().view(np.uint16)
    assert np.array_equal(got, ref.view(np.uint16).reshape(-1))


def _v2_layout_np(x16):
    """NumPy statement of the transformed tiles V2 that the bulk-copy-fed
    resident-U kernel reads: V = B^T d B of each tile's 4x4 window (rows
    first: R = fp16(s0 d_i0 + s1 d_i1), then columns: V = fp16(s0 R_j0 + s1
    R_j1)), stored per tap in 128-tile blocks (tiles rounded up to 8), per
    16-channel step in the K-major core-matrix interleave: tile i, channel c
    at byte (i >> 3) * 256 + (c >> 3) * 128 + (i & 7) * 16 + (c & 7) * 2."""
    from oracle import winograd as W
    n, c, h, w = x16.shape
    tp, tq = (h + 1) // 2, (w + 1) // 2
    pad = np.zeros((n, c, 2 * tp + 2, 2 * tq + 2), np.float64)
    pad[:, :, 1:h + 1, 1:w + 1] = x16.astype(np.float64)
    win = np.stack([np.stack([pad[:, :, 2 * a:2 * a + 4, 2 * b:2 * b + 4] for b in range(tq)], axis=2)
                    for a in range(tp)], axis=2)                               # n c ty tx i j
    r = np.einsum("ai,ncyxij->ncyxaj", W.BT, win).astype(np.float16).astype(np.float64)
    v = np.einsum("bj,ncyxaj->ncyxab", W.BT, r).astype(np.float16)            # n c ty tx a b
    nt = n * tp * tq
    nt8 = (nt + 7) // 8 * 8
    vt = v.transpose(4, 5, 0, 2, 3, 1).reshape(16, nt, c)                      # tap, tile, channel
    vt = np.concatenate([vt, np.zeros((16, nt8 - nt, c), np.float16)], axis=1)
    out = []
    for t in range(16):
        for tb in range((nt8 + 127) // 128):
            rows = min(128, nt8 - 128 * tb)
            blk = vt[t, 128 * tb:128 * tb + rows]                              # rows x c
            for cs in range(c // 16):
                piece = blk[:, 16 * cs:16 * cs + 16].reshape(rows // 8, 8, 2, 8)    # grp, i&7, hh, c&7
                out.append(piece.transpose(0, 2, 1, 3).reshape(-1))            # grp, hh, i&7, c&7
    return np.concatenate(out)


@pytest.mark.parametrize("shape", [(2, 32, 12, 10), (1, 16, 9, 7), (3, 48, 1, 1), (1, 16, 28, 28)])
def test_twostage_tile_prepass_bit_exact(wino, cuda, oracle_mod, shape):
    """The transformed-tile pre-pass (stage 0 of conv2d_twostage when the
    build routes C to the bulk-copy-fed resident-U kernel) writes exactly the
    NumPy statement of V2, partial last tile blocks included."""
    import torch
    n, c, h, w = shape
    L = wino.lib()
    if L.wino_twostage_gemm_kernel_ptr_for(c) != L.wino_twostage_resv_kernel_ptr():
        pytest.skip("this build does not route C to the bulk-copy-fed resident-U kernel")
    k = 16
    x16, _ = oracle_mod.make_inputs(n, c, h, w, k, seed=6, x_dist="normal")
    ref = _v2_layout_np(x16)
    nb = wino.twostage_workspace_bytes(n, c, h, w, k)
    ws = wino._aligned_ws(nb, cuda)
    ws.fill_(0xA5)                                                 # poison
    x = _t(x16, cuda)
    u2 = torch.zeros(16 * k * c, dtype=torch.float16, device=cuda)
    y = torch.empty((n, k, h, w), dtype=torch.float16, device=cuda)
    wino.twostage_stage(0, x, u2, k, y, ws)
    torch.cuda.synchronize()
    got = ws[:ref.nbytes].cpu().numpy().view(np.uint16)
    assert np.array_equal(got, ref.view(np.uint16))
