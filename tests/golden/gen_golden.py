"""Generate the golden vectors in tests/golden/*.npz.

Inputs are seeded synthetic fp16 tensors; the expected outputs come from the
reference's own CPU convolution, conv2dcpu() of include/verfiy.h, compiled
unmodified by oracle/Makefile (portable build: exact fp16 products).  The
reference ships no test vectors of its own, so these outputs of the reference
itself are what pins the oracle.

Run from the repository root where the reference tree is present:
    make -C oracle && python tests/golden/gen_golden.py
"""
from __future__ import annotations

import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

import oracle  # noqa: E402

# name, (n, c, h, w, k), input distribution, seed
CASES = [
    ("small_uniform", (1, 16, 8, 8, 16), "uniform", 1),
    ("odd_hw_normal", (2, 16, 7, 7, 32), "normal", 2),
    ("rect_h6_w10", (1, 32, 6, 10, 16), "uniform", 3),
    ("odd_both_c48", (3, 48, 5, 9, 48), "student_t3", 4),
    ("one_pixel", (1, 16, 1, 1, 16), "uniform", 5),
    ("h2_w3", (1, 16, 2, 3, 16), "normal", 6),
    ("tall_h17_w4", (1, 16, 17, 4, 32), "relu_normal", 7),
    ("refstyle_c64_h14", (2, 64, 14, 14, 64), "refstyle", 8),
]


def main():
    os.makedirs(HERE, exist_ok=True)
    for name, (n, c, h, w, k), dist, seed in CASES:
        if dist == "refstyle":
            x, wt = oracle.make_reference_style_inputs(n, c, h, w, k, seed=seed)
        else:
            x, wt = oracle.make_inputs(n, c, h, w, k, seed=seed, x_dist=dist)
        y = oracle.ref_conv2dcpu(x, wt)  # the reference's conv2dcpu, one thread
        np.savez_compressed(os.path.join(HERE, f"{name}.npz"), x=x, w=wt, y_ref=y,
                            shape=np.array([n, c, h, w, k]), dist=np.array(dist))
        print(f"{name}: n={n} c={c} h={h} w={w} k={k} -> y {y.shape}")


if __name__ == "__main__":
    main()
