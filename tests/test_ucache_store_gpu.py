"""Persisted U cache: content tag of the weights, save/load round trip,
refusal of stale files (other weights, shape, layout)."""
import ctypes
import os

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def test_weight_tag_tracks_contents(wino, cuda, oracle_mod):
    import torch
    _, w16 = oracle_mod.make_inputs(1, 64, 4, 4, 32, seed=1)
    w = torch.from_numpy(w16).to(cuda)
    t1, t2 = wino.weight_tag(w), wino.weight_tag(w.clone())
    assert t1 == t2 and t1 != 0
    w2 = w.clone()
    w2.view(-1)[12345] = w2.view(-1)[12345] + 1.0
    assert wino.weight_tag(w2) != t1
    w3 = w.clone()
    w3.view(-1)[[0, 1]] = w3.view(-1)[[1, 0]]     # a swap of two different values
    if float(w.view(-1)[0]) != float(w.view(-1)[1]):
        assert wino.weight_tag(w3) != t1


def test_persistent_u_cache_round_trip_and_invalidation(wino, cuda, oracle_mod, tmp_path):
    import torch
    x16, w16 = oracle_mod.make_inputs(2, 64, 14, 14, 48, seed=2, x_dist="normal")
    x, w = torch.from_numpy(x16).to(cuda), torch.from_numpy(w16).to(cuda)
    path = str(tmp_path / "u.bin")
    u1, loaded = wino.filter_transform_persistent(w, path)
    assert not loaded and os.path.getsize(path) > 16 * 48 * 64 * 2
    u2, loaded = wino.filter_transform_persistent(w, path)
    assert loaded
    fresh = wino.filter_transform(w)
    torch.cuda.synchronize()
    assert torch.equal(u2.view(torch.int16), fresh.view(torch.int16))
    y1, y2 = wino.conv2d_fused(x, fresh, 48), wino.conv2d_fused(x, u2, 48)
    torch.cuda.synchronize()
    assert torch.equal(y1.view(torch.int16), y2.view(torch.int16))
    # changed weights: the file is stale, U is recomputed and the file rewritten
    w2 = w.clone()
    w2[3, 5, 1, 1] += 0.25
    u3, loaded = wino.filter_transform_persistent(w2, path)
    assert not loaded
    assert torch.equal(u3.view(torch.int16), wino.filter_transform(w2).view(torch.int16))
    # direct C-ABI: stale tag or shape -> WINO_ESTALE, buffer untouched
    L = wino.lib()
    buf = torch.full((16 * 48 * 64,), 7.0, dtype=torch.float16, device=cuda)
    assert L.wino_ucache_load(os.fsencode(path), ctypes.c_void_p(buf.data_ptr()), 48, 64,
                              wino.weight_tag(w)) == wino.WINO_ESTALE
    assert L.wino_ucache_load(os.fsencode(path), ctypes.c_void_p(buf.data_ptr()), 32, 64,
                              wino.weight_tag(w2)) == wino.WINO_ESTALE
    assert bool((buf == 7.0).all())
    assert L.wino_ucache_load(os.fsencode(path), ctypes.c_void_p(buf.data_ptr()), 48, 64,
                              wino.weight_tag(w2)) == wino.WINO_OK
    assert torch.equal(buf.view(torch.int16), u3.view(torch.int16))
