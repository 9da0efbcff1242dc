"""The cost model's CUDA kernels against the NumPy oracle, and the trained
model against exhaustive tuning on the committed timings of 400 shapes."""
import importlib
import json
import os

import numpy as np
import pytest

from oracle import mlp as M

pytestmark = pytest.mark.gpu
TIMINGS = os.path.join(os.path.dirname(__file__), "golden", "tuning_timings.json")


def _cm():
    return importlib.import_module("2024pra_conv_b200.costmodel")


def _batch(seed, B=37, F=6, O=4):
    rng = np.random.default_rng(seed)
    p = M.init_params(F, O, seed=seed) + (0.05 * rng.standard_normal(M.nparams(F, O))).astype(np.float32)
    x = rng.standard_normal((B, F)).astype(np.float32)
    t = rng.standard_normal((B, O)).astype(np.float32)
    m = (rng.random((B, O)) > 0.25).astype(np.float32)
    return p, x, t, m


@pytest.mark.parametrize("seed", [0, 1, 2])
def test_mlp_forward_and_gradient_match_cpu_oracle(cuda, seed):
    import torch
    cm = _cm()
    p, x, t, m = _batch(seed)
    T = lambda a: torch.from_numpy(a).to(cuda)
    y = cm.mlp_forward(T(p), T(x), O=4).cpu().numpy()
    y64, _ = M.forward(p.astype(np.float64), x.astype(np.float64), 6, 4)
    assert np.allclose(y, y64, rtol=1e-4, atol=1e-5)
    loss, g = cm.mlp_grad(T(p), T(x), T(t), T(m))
    loss64, g64 = M.loss_and_grad(p.astype(np.float64), x.astype(np.float64), t, m, 6, 4)
    assert abs(loss - loss64) <= 1e-5 * max(1.0, abs(loss64))
    g = g.cpu().numpy()
    assert np.max(np.abs(g - g64)) <= 1e-5 * max(1.0, np.max(np.abs(g64))), np.max(np.abs(g - g64))


def test_mlp_training_on_gpu_reduces_loss(cuda):
    import torch
    cm = _cm()
    p, x, t, m = _batch(5, B=64)
    T = lambda a: torch.from_numpy(a).to(cuda)
    pt = T(p)
    hist = cm.mlp_train(pt, T(x), T(t), T(m), epochs=400, lr=3e-3)
    assert hist[-1] < 0.5 * hist[0]
    loss_end, _ = M.loss_and_grad(pt.cpu().numpy().astype(np.float64), x, t, m, 6, 4)
    assert abs(loss_end - hist[-1]) <= 0.05 * hist[-1] + 1e-4     # one more step apart


@pytest.mark.skipif(not os.path.exists(TIMINGS), reason="timings fixture not generated")
def test_cost_model_picks_within_10pct_of_exhaustive_and_beats_default(cuda, capsys):
    """Trained on 300 shapes' exhaustive timings, evaluated on 100 held out."""
    cm = _cm()
    with open(TIMINGS) as f:
        rows = json.load(f)["rows"]
    r = cm.evaluate(rows)
    with capsys.disabled():
        print("\ncost model:", {k: v for k, v in r.items() if k != "regret"})
    assert r["loss_last"] < r["loss_first"]
    assert r["regret_geomean"] <= 1.10
    assert r["gain_geomean"] >= 1.0


@pytest.mark.skipif(not os.path.exists(TIMINGS), reason="timings fixture not generated")
def test_trained_model_checkpoint_gives_the_same_picks(cuda, tmp_path):
    cm = _cm()
    with open(TIMINGS) as f:
        rows = json.load(f)["rows"]
    model = cm.train(rows, epochs=500)
    shapes = [tuple(r["shape"]) for r in rows[:50]]
    picks = cm.pick(model, shapes)
    assert all(not (p & 2) for p in picks)                   # inside the tuning space
    path = str(tmp_path / "m.npz")
    cm.save_model(model, path)
    assert cm.pick(cm.load_model(path), shapes) == picks
