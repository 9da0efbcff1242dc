"""Cost-model pieces that need no GPU: the NumPy MLP oracle against finite
differences, the shape space, the features, the split."""
import importlib

import numpy as np

from oracle import mlp as M


def test_mlp_oracle_gradient_matches_finite_differences():
    F, O, B = 6, 4, 7
    rng = np.random.default_rng(3)
    p = M.init_params(F, O, seed=1).astype(np.float64) + 0.01 * rng.standard_normal(M.nparams(F, O))
    x = rng.standard_normal((B, F))
    t = rng.standard_normal((B, O))
    m = (rng.random((B, O)) > 0.2).astype(np.float64)
    _, g = M.loss_and_grad(p, x, t, m, F, O)
    idx = rng.choice(len(p), 60, replace=False)
    for i in idx:
        e = np.zeros_like(p)
        e[i] = 1e-6
        num = (M.loss_and_grad(p + e, x, t, m, F, O)[0] - M.loss_and_grad(p - e, x, t, m, F, O)[0]) / 2e-6
        assert abs(num - g[i]) <= 1e-6 + 1e-5 * abs(num), (i, num, g[i])


def test_shape_space_and_split():
    cm = importlib.import_module("2024pra_conv_b200.costmodel")
    shapes = cm.random_shapes()
    assert len(shapes) == 400 and shapes == cm.random_shapes()      # seeded
    for n, c, h, k in shapes:
        assert n in (1, 8, 32, 128)
        for v in (c, k):
            assert 16 <= v <= 1024 and (v % 48 == 0 or (v & (v - 1)) == 0)
        assert 7 <= h <= 112
    tr, te = cm.split(400)
    assert len(tr) == 300 and len(te) == 100 and not set(tr) & set(te)
    f = np.array([cm.raw_features(s) for s in shapes])
    assert f.shape == (400, cm.F) and np.isfinite(f).all()
    p = cm.init_params()
    assert np.array_equal(p, M.init_params(cm.F, cm.NCFG, seed=0))


def test_model_checkpoint_round_trip(tmp_path):
    cm = importlib.import_module("2024pra_conv_b200.costmodel")
    model = {"params": cm.init_params(seed=3), "mu": np.arange(cm.F, dtype=np.float64),
             "sd": np.ones(cm.F)}
    path = str(tmp_path / "model.npz")
    cm.save_model(model, path)
    back = cm.load_model(path)
    assert np.array_equal(back["params"], model["params"]) and np.array_equal(back["mu"], model["mu"])
    np.savez(path, version=99, features=cm.F, outputs=cm.NCFG, params=model["params"], mu=model["mu"],
             sd=model["sd"])
    import pytest
    with pytest.raises(ValueError):
        cm.load_model(path)
