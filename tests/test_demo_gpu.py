"""The C++ drop-in demo (csrc/conv2d_demo.cpp): a caller compiled only
against include/conv2d.h runs the reference harness flow on the GPU and
passes the harness's 1 % check on sampled outputs."""
import json
import os
import subprocess

import pytest

pytestmark = pytest.mark.gpu
DEMO = os.path.join(os.path.dirname(__file__), "..", "2024pra_conv_b200", "_build", "conv2ddemo")


@pytest.mark.parametrize("shape", [(8, 64, 32, 32, 64), (2, 48, 9, 14, 32)])
def test_cpp_dropin_demo(wino, cuda, shape):
    assert os.path.exists(DEMO), "build the library first (build.py builds the demo)"
    r = subprocess.run([DEMO] + [str(v) for v in shape], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stdout + r.stderr
    line = json.loads(r.stdout.strip().splitlines()[-1])
    assert line["error"] == 0 and line["checked"] == 512 and line["paramsize"] == 80
