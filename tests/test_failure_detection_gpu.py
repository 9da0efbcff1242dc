"""Failure detection without a GPU fault: a kernel's bounded waits on
mbarriers that nothing signals run out after their one-second limit, record
their codes in the kernel's error word and return; the context stays usable
(a conv runs correctly right after)."""
import ctypes
import time

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def test_bounded_waits_report_and_context_survives(wino, cuda, oracle_mod):
    import torch
    L = wino.lib()
    codes = (ctypes.c_uint32 * 2)()
    t0 = time.time()
    assert L.wino_selftest_wait_timeout(codes) == 0          # cudaSuccess: no fault
    dt = time.time() - t0
    assert list(codes) == [1, 2]                             # ERR_WAIT_FULL, ERR_WAIT_EMPTY
    assert 0.9 <= dt <= 30.0                                  # the waits' time limit, ~1 s
    x16, w16 = oracle_mod.make_inputs(2, 32, 10, 10, 32, seed=4, x_dist="normal")
    y = wino.conv2d(torch.from_numpy(x16).to(cuda), torch.from_numpy(w16).to(cuda))
    torch.cuda.synchronize()
    y64 = oracle_mod.conv2d_f64(x16, w16)
    assert oracle_mod.rel_l2(y.cpu().numpy(), y64) <= 2e-3
    assert wino.error_read_clear() == 0
