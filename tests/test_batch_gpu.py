"""Schedule configurations, the batched persistent launch, its CUDA graph
and the autotuner.

Every configuration and every layer order computes the same arithmetic, so
outputs must be bit-identical to the single-layer default path; each layer
is also checked against FP64 (rel-L2 <= 2e-3, max-normalised <= 1e-2).
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _fp64_check(x, w, y):
    import torch
    y64 = torch.nn.functional.conv2d(x.double(), w.double(), padding=1)
    yd = y.double()
    rl2 = float(torch.linalg.vector_norm(yd - y64) / torch.linalg.vector_norm(y64))
    mxn = float((yd - y64).abs().max() / y64.abs().max())
    assert rl2 <= 2e-3 and mxn <= 1e-2, (rl2, mxn)


@pytest.mark.parametrize("shape", [(4, 64, 20, 20, 144), (2, 32, 7, 7, 32), (1, 16, 6, 224, 16),
                                   (1, 256, 10, 10, 64)])
def test_configs(wino, cuda, oracle_mod, shape):
    """Unsplit configurations: bit-identical to the default path.  Split
    ones (fp32 partial sums added in another order): FP64 parity."""
    import torch
    n, c, h, w, k = shape
    x16, w16 = oracle_mod.make_inputs(n, c, h, w, k, seed=7, x_dist="normal")
    x = torch.from_numpy(x16).to(cuda)
    wt = torch.from_numpy(w16).to(cuda)
    u = wino.filter_transform(wt)
    ref = wino.conv2d_fused(x, u, k)
    for cfg in range(wino.NCFG):
        y = wino.conv2d_fused_cfg(x, u, k, cfg)
        torch.cuda.synchronize()
        if (cfg >> wino.CFG_SPLIT_SHIFT) == 0 or c == 16:
            assert torch.equal(y.view(torch.int16), ref.view(torch.int16)), cfg
        else:
            _fp64_check(x, wt, y)
    _fp64_check(x, wt, ref)
    assert wino.error_read_clear() == 0


def test_tune_layer_space(wino, cuda, oracle_mod):
    import torch
    n, c, h, w, k = 1, 512, 14, 14, 128
    x16, w16 = oracle_mod.make_inputs(n, c, h, w, k, seed=9, x_dist="uniform")
    x = torch.from_numpy(x16).to(cuda)
    u = wino.filter_transform(torch.from_numpy(w16).to(cuda))
    y = torch.empty((n, k, h, w), dtype=torch.float16, device=cuda)
    ws = wino._aligned_ws(wino.tune_workspace_bytes(n, c, h, w, k), cuda)
    us, best = wino.tune_layer(x, u, k, ws, y, reps=1)
    timed = [i for i, t in enumerate(us) if t > 0]
    assert all(not (i & wino.CFG_DIRECT) for i in timed)
    assert {0, 1, wino.cfg_split(1), wino.cfg_split(2), wino.cfg_split(3)} <= set(timed)
    assert best in timed and us[best] == min(us[i] for i in timed)
    us2, best2 = wino.tune_layer(x, u, k, None, y, reps=1)
    assert [i for i, t in enumerate(us2) if t > 0] == [wino.CFG_DIRECT, wino.CFG_DIRECT | 1]
    assert wino.error_read_clear() == 0


def _layer_set(wino, oracle_mod, cuda, n):
    import torch
    layers = []
    for i, (c, k, h) in enumerate(wino.RESNET_LAYER_SET):
        x16, w16 = oracle_mod.make_inputs(n, c, h, h, k, seed=100 + i, x_dist="uniform",
                                          w_std=np.sqrt(2.0 / (9 * c)))
        x = torch.from_numpy(x16).to(cuda)
        wt = torch.from_numpy(w16).to(cuda)
        u = wino.filter_transform(wt)
        ws = torch.empty(wino.fused_workspace_bytes(n, c, h, h), dtype=torch.uint8, device=cuda)
        y = torch.full((n, k, h, h), float("nan"), dtype=torch.float16, device=cuda)
        layers.append((x, wt, u, ws, y, k))
    return layers


def _refs(wino, layers):
    """Each layer's single-layer outputs on both routes: the fused kernel and
    the two-stage path (U relaid to its layout)."""
    fused = [wino.conv2d_fused(x, u, k) for (x, wt, u, ws, y, k) in layers]
    two = [wino.conv2d_twostage(x, wino.filter_transform_unfused(wt), k) for (x, wt, u, ws, y, k) in layers]
    return fused, two


def _check_routes(wino, b, layers, refs, tag):
    import torch
    torch.cuda.synchronize()
    for i, (x, wt, u, ws, y, k) in enumerate(layers):
        r = refs[b.route(i)[0]][i]
        assert torch.equal(y.view(torch.int16), r.view(torch.int16)), (tag, i, b.route(i))
        y.fill_(float("nan"))


def test_batched_layer_set_one_launch_graph_and_tuner(wino, cuda, oracle_mod):
    """The 12-layer ResNet-style set at N=32 in one persistent launch; after
    tuning, layers the tuner routes to the two-stage path equal that path's
    single-layer output bit for bit."""
    import torch
    layers = _layer_set(wino, oracle_mod, cuda, 32)
    refs = _refs(wino, layers)
    b = wino.Batch()
    for (x, wt, u, ws, y, k) in layers:
        b.add(x, u, k, y, workspace=ws)
    assert len(b) == 12

    def check(tag):
        _check_routes(wino, b, layers, refs, tag)

    b.run()
    check("run")
    for (x, wt, u, ws, y, k), r, r2 in zip(layers, refs[0], refs[1]):
        _fp64_check(x, wt, r)
        _fp64_check(x, wt, r2)
    # mixed configurations and a reversed table order
    for i in range(12):
        b.set_config(i, i % 4)      # unsplit configurations: batch layers run unsplit
    b.set_order(list(range(11, -1, -1)))
    b.run()
    check("mixed configs, reversed order")
    # autotuner: timings for every configuration, then the best order
    layer_us, order_us = b.tune(reps=2)
    assert all(min(t for t in row if t > 0) > 0 for row in layer_us)
    assert all(t > 0 for t in order_us)
    for i in range(12):
        row = layer_us[i]
        assert row[b.config(i)] == min(t for t in row if t > 0)
        route, fused_us, two_us = b.route(i)
        assert fused_us > 0 and two_us > 0          # every layer of the set has both routes
        assert route in (0, 1)
    assert sorted(b.order()) == list(range(12))
    b.run()
    check("tuned")
    # CUDA graph of pre-passes + the persistent launch, replayed twice
    b.capture()
    b.launch()
    check("graph 1")
    b.launch()
    check("graph 2")
    b.close()
    assert wino.error_read_clear() == 0


def test_tuning_state_save_and_restore(wino, cuda, oracle_mod, tmp_path):
    """Tuned choices survive a JSON round trip and re-apply without tuning."""
    import json
    import torch
    layers = _layer_set(wino, oracle_mod, cuda, 4)
    refs = _refs(wino, layers)
    b = wino.Batch()
    for (x, wt, u, ws, y, k) in layers:
        b.add(x, u, k, y, workspace=ws)
    b.tune(reps=1)
    path = tmp_path / "tuning.json"
    path.write_text(json.dumps(b.tuning_state()))
    b.close()
    b2 = wino.Batch()
    for (x, wt, u, ws, y, k) in layers:
        b2.add(x, u, k, y, workspace=ws)
    state = json.loads(path.read_text())
    b2.restore(state)
    assert b2.tuning_state() == state
    b2.run()
    _check_routes(wino, b2, layers, refs, "restored")
    b2.close()
    assert wino.error_read_clear() == 0


def test_batch_routes_mixed(wino, cuda, oracle_mod):
    """Layers set explicitly to the two-stage route run before the persistent
    launch of the rest (also inside the CUDA graph) and equal the two-stage
    path's single-layer outputs; every layer two-stage skips the persistent
    launch altogether."""
    layers = _layer_set(wino, oracle_mod, cuda, 2)
    refs = _refs(wino, layers)
    b = wino.Batch()
    for (x, wt, u, ws, y, k) in layers:
        b.add(x, u, k, y, workspace=ws)
    for i in range(0, 12, 3):
        b.set_route(i, 1)
    b.run()
    _check_routes(wino, b, layers, refs, "mixed")
    assert [b.route(i)[0] for i in range(12)] == [1 if i % 3 == 0 else 0 for i in range(12)]
    b.capture()
    b.launch()
    _check_routes(wino, b, layers, refs, "mixed graph")
    for i in range(12):
        b.set_route(i, 1)
    b.run()
    _check_routes(wino, b, layers, refs, "all two-stage")
    b.close()
    assert wino.error_read_clear() == 0
