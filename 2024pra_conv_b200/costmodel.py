"""Learned tile-configuration cost model and its data.

For a 3x3 stride-1 pad-1 layer the autotuner (wino_tune_layer) times every
schedule configuration of the fused kernel (CFG_* bits: k-major block order,
split of the channel steps over several CTAs).  A small MLP -- shape features -> 64 ReLU -> 64 ReLU ->
log-time per configuration (16 outputs, masked to the configurations
timed) -- is trained on those timings with the
library's own CUDA kernels (csrc/mlp.cu: forward, backward, Adam) and picks
a configuration for unseen shapes without timing them; exhaustive tuning
stays the fallback and the yardstick of its picks.  The reference has no
counterpart (one hard-wired kernel set per shape, src/conv2d.cpp:458-494).

Shape space (400 seeded shapes, 300 train / 100 held out): N in {1, 8, 32,
128}; C, K in the powers of two and multiples of 48 inside [16, 1024];
H = W in [7, 112].

    python -m 2024pra_conv_b200.costmodel collect OUT.json   # GPU: timings
    python -m 2024pra_conv_b200.costmodel evaluate IN.json   # GPU: train + evaluate
"""
from __future__ import annotations

import ctypes
import importlib
import json
import math
import sys

import numpy as np

NS = (1, 8, 32, 128)
CK = tuple(sorted({v for v in range(16, 1025) if v % 48 == 0} | {1 << e for e in range(4, 11)}))
H_RANGE = (7, 112)
NCFG = 16  # schedule configurations (CFG_* bits); the tuning space uses the non-direct ones
F = 6  # features


def _wino():
    return importlib.import_module("2024pra_conv_b200")


def random_shapes(count=400, seed=0):
    """Seeded shapes (n, c, h, k), h = w."""
    rng = np.random.default_rng(seed)
    out = []
    for _ in range(count):
        out.append((int(rng.choice(NS)), int(rng.choice(CK)), int(rng.integers(H_RANGE[0], H_RANGE[1] + 1)),
                    int(rng.choice(CK))))
    return out


def split(count=400, n_train=300, seed=1):
    """Seeded train / held-out index split."""
    idx = np.random.default_rng(seed).permutation(count)
    return sorted(idx[:n_train].tolist()), sorted(idx[n_train:].tolist())


def raw_features(shape):
    n, c, h, k = shape
    tiles = n * ((h + 1) // 2) ** 2
    flops = 2.0 * n * c * k * h * h * 9
    return [math.log2(n), math.log2(c), math.log2(k), math.log2(h), math.log2(tiles), math.log2(flops)]


class Normaliser:
    def __init__(self, feats):
        a = np.asarray(feats, np.float64)
        self.mu = a.mean(0)
        self.sd = a.std(0) + 1e-6

    def __call__(self, feats):
        return ((np.asarray(feats, np.float64) - self.mu) / self.sd).astype(np.float32)


def collect(shapes, reps=2, log=None):
    """Exhaustive timings (us per configuration) of every shape on cuda:0."""
    import torch
    wino = _wino()
    dev = torch.device("cuda", 0)
    g = torch.Generator(device=dev)
    g.manual_seed(0)
    rows = []
    for i, (n, c, h, k) in enumerate(shapes):
        x = (torch.rand((n, c, h, h), device=dev, generator=g) * 2 - 1).half()
        w = (torch.randn((k, c, 3, 3), device=dev, generator=g) * math.sqrt(2.0 / (9 * c))).half()
        u = wino.filter_transform(w)
        y = torch.empty((n, k, h, h), dtype=torch.float16, device=dev)
        ws = wino._aligned_ws(wino.tune_workspace_bytes(n, c, h, h, k), dev)
        us, best = wino.tune_layer(x, u, k, ws, y, reps=reps)
        rows.append({"shape": [n, c, h, k], "us": us, "best": best})
        if log:
            log(f"{i:3d} N{n} C{c} H{h} K{k}: " + " ".join(f"{t:9.1f}" for t in us) + f"  best {best}")
        del x, w, u, y, ws
    code = wino.error_read_clear()
    if code:
        raise RuntimeError(f"device error word {code}")
    return rows


def _lib():
    L = _wino().lib()
    f, i, vp = ctypes.c_float, ctypes.c_int, ctypes.c_void_p
    for name, args, res in [
        ("wino_mlp_num_params", [i, i], i),
        ("wino_mlp_forward", [vp, vp, vp, i, i, i, vp], i),
        ("wino_mlp_grad", [vp, vp, vp, vp, i, i, i, f, vp, vp, vp, vp], i),
        ("wino_mlp_train", [vp, vp, vp, vp, i, i, i, f, i, f, vp, vp, vp, vp, vp], i),
    ]:
        fn = getattr(L, name)
        fn.argtypes = args
        fn.restype = res
    return L


def init_params(O=NCFG, seed=0):
    """He-style initialisation, identical to the CPU oracle's."""
    rng = np.random.default_rng(seed)
    H = 64
    parts = [rng.standard_normal((H, F)) * np.sqrt(2.0 / F), np.zeros(H),
             rng.standard_normal((H, H)) * np.sqrt(2.0 / H), np.zeros(H),
             rng.standard_normal((O, H)) * np.sqrt(1.0 / H), np.zeros(O)]
    return np.concatenate([a.ravel() for a in parts]).astype(np.float32)


def _ptr(t):
    return ctypes.c_void_p(t.data_ptr())


def _stream():
    import torch
    return ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)


def mlp_forward(params, x, O=NCFG):
    """params, x: cuda float32 tensors -> predictions [B, O]."""
    import torch
    L = _lib()
    B = x.shape[0]
    y = torch.empty((B, O), dtype=torch.float32, device=x.device)
    rc = L.wino_mlp_forward(_ptr(params), _ptr(x), _ptr(y), B, x.shape[1], O, _stream())
    if rc:
        raise RuntimeError(f"wino_mlp_forward {rc}")
    return y


def mlp_grad(params, x, t, m):
    import torch
    L = _lib()
    B, Fx = x.shape
    O = t.shape[1]
    P = L.wino_mlp_num_params(Fx, O)
    grad = torch.empty(P, dtype=torch.float32, device=x.device)
    loss = torch.empty(1, dtype=torch.float32, device=x.device)
    scratch = torch.empty(B * (P + 1), dtype=torch.float32, device=x.device)
    rc = L.wino_mlp_grad(_ptr(params), _ptr(x), _ptr(t), _ptr(m), B, Fx, O, float(m.sum().item()), _ptr(grad),
                         _ptr(loss), _ptr(scratch), _stream())
    if rc:
        raise RuntimeError(f"wino_mlp_grad {rc}")
    return float(loss.item()), grad


def mlp_train(params, x, t, m, epochs=3000, lr=3e-3):
    """Full-batch Adam on the GPU; returns the loss history (before each step)."""
    import torch
    L = _lib()
    B, Fx = x.shape
    O = t.shape[1]
    P = L.wino_mlp_num_params(Fx, O)
    mom = torch.zeros(P, dtype=torch.float32, device=x.device)
    var = torch.zeros(P, dtype=torch.float32, device=x.device)
    scratch = torch.empty(B * (P + 1) + P + 1, dtype=torch.float32, device=x.device)
    hist = torch.empty(max(epochs, 1), dtype=torch.float32, device=x.device)
    rc = L.wino_mlp_train(_ptr(params), _ptr(x), _ptr(t), _ptr(m), B, Fx, O, float(m.sum().item()), epochs, lr,
                          _ptr(mom), _ptr(var), _ptr(scratch), _ptr(hist), _stream())
    if rc:
        raise RuntimeError(f"wino_mlp_train {rc}")
    return hist[:epochs].cpu().numpy()


def dataset(rows, idx, norm=None):
    feats = [raw_features(tuple(rows[i]["shape"])) for i in idx]
    norm = norm or Normaliser(feats)
    x = norm(feats)
    us = np.array([rows[i]["us"] for i in idx], np.float64)
    m = (us > 0).astype(np.float32)
    t = np.where(us > 0, np.log(np.maximum(us, 1e-3)), 0.0).astype(np.float32)
    return x, t, m, us, norm


def evaluate(rows, epochs=3000, lr=3e-3, seed=0, default_cfg=0):
    """Train on the 300 training shapes, pick on the 100 held out.

    Returns a dict: per held-out shape t(pick) / t(best) ("regret"), the
    geometric means of that and of t(default) / t(pick) ("gain" over the
    method without the model: the fixed default configuration), the share
    of exact picks, and the training loss at start and end."""
    import torch
    tr, te = split(len(rows))
    xtr, ttr, mtr, _, norm = dataset(rows, tr)
    xte, _, _, us_te, _ = dataset(rows, te, norm)
    dev = torch.device("cuda", 0)
    p = torch.from_numpy(init_params(seed=seed)).to(dev)
    hist = mlp_train(p, torch.from_numpy(xtr).to(dev), torch.from_numpy(ttr).to(dev),
                     torch.from_numpy(mtr).to(dev), epochs=epochs, lr=lr)
    pred = mlp_forward(p, torch.from_numpy(xte).to(dev)).cpu().numpy()
    pred = np.where(us_te > 0, pred, np.inf)
    pick = pred.argmin(1)
    valid = np.where(us_te > 0, us_te, np.inf)
    best = valid.min(1)
    t_pick = valid[np.arange(len(te)), pick]
    t_def = valid[:, default_cfg]
    regret = t_pick / best
    gain = t_def / t_pick
    return {"regret": regret.tolist(), "regret_geomean": float(np.exp(np.log(regret).mean())),
            "regret_max": float(regret.max()), "gain_geomean": float(np.exp(np.log(gain).mean())),
            "default_regret_geomean": float(np.exp(np.log(t_def / best).mean())),
            "exact_picks": float(np.mean(t_pick == best)), "loss_first": float(hist[0]),
            "loss_last": float(hist[-1]), "held_out": len(te), "train": len(tr)}


def train(rows, idx=None, epochs=3000, lr=3e-3, seed=0):
    """Train on the given rows (default: the training split) with the CUDA
    kernels; returns a model dict {params (float32 numpy), mu, sd}."""
    import torch
    idx = split(len(rows))[0] if idx is None else idx
    x, t, m, _, norm = dataset(rows, idx)
    dev = torch.device("cuda", 0)
    p = torch.from_numpy(init_params(seed=seed)).to(dev)
    mlp_train(p, torch.from_numpy(x).to(dev), torch.from_numpy(t).to(dev), torch.from_numpy(m).to(dev),
              epochs=epochs, lr=lr)
    return {"params": p.cpu().numpy(), "mu": norm.mu, "sd": norm.sd}


def pick(model, shapes, allowed=None):
    """Predicted-fastest configuration per shape (n, c, h, k) with the CUDA
    inference kernel; `allowed`: configurations to choose from (default: the
    tuning space, i.e. every configuration without CFG_DIRECT)."""
    import torch
    allowed = [c for c in range(NCFG) if not (c & 2)] if allowed is None else allowed
    norm = Normaliser([[0.0] * F])
    norm.mu, norm.sd = np.asarray(model["mu"]), np.asarray(model["sd"])
    x = norm([raw_features(tuple(s)) for s in shapes])
    dev = torch.device("cuda", 0)
    pred = mlp_forward(torch.from_numpy(np.asarray(model["params"], np.float32)).to(dev),
                       torch.from_numpy(x).to(dev)).cpu().numpy()
    mask = np.full(NCFG, np.inf)
    mask[allowed] = 0.0
    return [int(v) for v in (pred + mask).argmin(1)]


MODEL_VERSION = 1


def save_model(model, path):
    """Versioned checkpoint of a trained model (NumPy .npz)."""
    np.savez(path, version=MODEL_VERSION, features=F, outputs=NCFG, params=model["params"],
             mu=model["mu"], sd=model["sd"])


def load_model(path):
    """A checkpoint written by save_model; refuses other versions or shapes."""
    d = np.load(path)
    if int(d["version"]) != MODEL_VERSION or int(d["features"]) != F or int(d["outputs"]) != NCFG:
        raise ValueError(f"{path}: cost-model checkpoint of another version or shape")
    return {"params": d["params"].astype(np.float32), "mu": d["mu"], "sd": d["sd"]}


def main(argv):
    if len(argv) >= 2 and argv[0] == "collect":
        rows = collect(random_shapes(), log=lambda s: print(s, flush=True))
        with open(argv[1], "w") as f:
            json.dump({"configs": "index = CFG_* bits: 1 k-major, 2 direct, (level << 2) split "
                                  "16-channel steps over up to 4^level CTAs; -1 = outside the tuning space",
                       "rows": rows}, f)
        return 0
    if len(argv) >= 2 and argv[0] == "evaluate":
        with open(argv[1]) as f:
            rows = json.load(f)["rows"]
        r = evaluate(rows)
        r.pop("regret")
        print(json.dumps(r))
        return 0
    print(__doc__)
    return 2


if __name__ == "__main__":
    sys.exit(main(sys.argv[1:]))
