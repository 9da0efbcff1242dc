"""The conv entry point for callers that cannot allocate device memory.

Some callers (plugin hosts that hand the operator only its input and output,
runtimes with device memory fixed at start-up) cannot provide the U-cache
workspace the regular entry points take.  wino_conv2d_noalloc keeps U in a
fixed array inside the library instead.  This file checks, through the C-ABI,
that two consecutive calls give the regular entry point's result within the
fp16 parity tolerance, and that filters too large for the array are refused.
It sits last in collection order so a failure here cannot hide other tests.
"""
import ctypes

import numpy as np
import pytest

REL_L2 = 2e-3
WINO_ESCRATCH = 5


def _noalloc(wino):
    lib = wino.lib()
    fn = lib.wino_conv2d_noalloc
    fn.argtypes = [ctypes.c_void_p] * 3 + [ctypes.c_int] * 5 + [ctypes.c_void_p]
    fn.restype = ctypes.c_int
    lib.wino_noalloc_max_kc.restype = ctypes.c_longlong
    return fn, int(lib.wino_noalloc_max_kc())


def test_noalloc_symbol_is_exported(wino):
    fn, max_kc = _noalloc(wino)
    assert max_kc == 512 * 512


def test_noalloc_rejects_filter_beyond_scratch(wino):
    fn, max_kc = _noalloc(wino)
    # rejected before any CUDA call: the pointers are never dereferenced
    rc = fn(ctypes.c_void_p(0x1000), ctypes.c_void_p(0x2000), ctypes.c_void_p(0x3000),
            1, 1024, 8, 8, 512, None)
    assert rc == WINO_ESCRATCH
    assert 1024 * 512 > max_kc


@pytest.mark.gpu
def test_noalloc_matches_regular_entry_on_two_calls(wino, cuda, oracle_mod):
    import torch
    fn, _ = _noalloc(wino)
    stream = torch.cuda.current_stream()
    cases = [((4, 64, 14, 14, 96), "uniform", 1), ((2, 128, 9, 12, 64), "student_t3", 2)]
    for (n, c, h, w, k), dist, seed in cases:
        x16, w16 = oracle_mod.make_inputs(n, c, h, w, k, seed=seed, x_dist=dist)
        x = torch.from_numpy(x16).to(cuda)
        wt = torch.from_numpy(w16).to(cuda)
        y = torch.full((n, k, h, w), float("nan"), dtype=torch.float16, device=cuda)
        rc = fn(ctypes.c_void_p(x.data_ptr()), ctypes.c_void_p(wt.data_ptr()),
                ctypes.c_void_p(y.data_ptr()), n, c, h, w, k, ctypes.c_void_p(stream.cuda_stream))
        assert rc == 0
        y_ref = wino.conv2d(x, wt)  # regular path: caller-owned U cache + fused conv
        torch.cuda.synchronize()
        a = y.double().cpu().numpy()
        b = y_ref.double().cpu().numpy()
        assert np.isfinite(a).all()
        rel = np.linalg.norm(a - b) / np.linalg.norm(b)
        assert rel <= REL_L2, rel
        # and against the FP64 oracle, like every other parity test
        assert oracle_mod.rel_l2(a, oracle_mod.conv2d_f64(x16, w16)) <= REL_L2
    assert wino.error_read_clear() == 0
