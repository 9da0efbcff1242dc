import glob
import importlib
import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

GOLDEN = os.path.join(ROOT, "tests", "golden")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a B200 (sm_100a) GPU")


def _build_if_needed():
    pkg_dir = os.path.join(ROOT, "2024pra_conv_b200")
    lib = os.path.join(pkg_dir, "_build", "libwinoconv.so")
    if not os.path.exists(lib):
        sys.path.insert(0, pkg_dir)
        import build as _b  # 2024pra_conv_b200/build.py
        _b.build()
    return lib


@pytest.fixture(scope="session")
def wino():
    """The package (its directory name starts with a digit)."""
    _build_if_needed()
    return importlib.import_module("2024pra_conv_b200")


@pytest.fixture(scope="session")
def oracle_mod():
    import oracle
    oracle.build() if not os.path.exists(os.path.join(ROOT, "oracle", "_build", "liboracle.so")) else None
    return oracle


def golden_cases():
    return sorted(glob.glob(os.path.join(GOLDEN, "*.npz")))


def load_golden(path):
    d = np.load(path)
    return d["x"], d["w"], d["y_ref"]


@pytest.fixture(scope="session")
def cuda():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    return torch.device("cuda:0")
