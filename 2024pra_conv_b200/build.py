"""Build recipe for libwinoconv.so and the drop-in demo driver.

Everything is compiled in-tree into 2024pra_conv_b200/_build/ for sm_100a
only (`-gencode arch=compute_100a,code=sm_100a`).  The library links the
shared CUDA runtime: the kernel pointers getkernelInfo() returns are launched
by the caller's own cudaLaunchKernel, which only works when caller and
library share one runtime instance.

    python 2024pra_conv_b200/build.py            # build (incremental)
    python 2024pra_conv_b200/build.py --clean    # rebuild from scratch
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
BUILD = os.path.join(HERE, "_build")
INCLUDE = os.path.join(ROOT, "include")
LIB = os.path.join(BUILD, "libwinoconv.so")
DEMO = os.path.join(BUILD, "conv2ddemo")

CUDA_HOME = os.environ.get("CUDA_HOME", "/usr/local/cuda")
NVCC = os.path.join(CUDA_HOME, "bin", "nvcc")
# The image exports CC/CXX wrappers without the full runtime specs; use the
# system compilers from PATH (nvcc's host compiler is pinned the same way).
CXX = shutil.which("g++") or "g++"

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ARCH + ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC",
                     "-ccbin", CXX, "-I", INCLUDE, "-I", CSRC]
# Extra nvcc flags for tuning builds (e.g. -DWINO_PAIR_LOAD=__ldcg); the
# default build uses none.
NVCC_FLAGS += os.environ.get("WINO_NVCC_EXTRA", "").split()
CXX_FLAGS = ["-O2", "-fPIC", "-std=c++17", "-I", INCLUDE, "-I", CSRC,
             "-I", os.path.join(CUDA_HOME, "include")]

CU_SOURCES = ["filter_transform.cu", "fused_conv.cu", "input_layout.cu", "unfused_conv.cu", "misc.cu", "noalloc.cu",
              "mlp.cu", "direct_conv.cu", "ucache_store.cu", "winograd_f4.cu",
              "twostage_conv.cu", "igemm_conv.cu"]
CPP_SOURCES = ["wino_abi.cpp", "wino_batch.cpp"]
HEADERS = ["tc_sm100.cuh", "wino_common.cuh", "wino_param.h", "vgen.cuh", "wino_batch.h"]


def _newer(src_list, target):
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(s) > t for s in src_list)


def _run(cmd):
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        sys.stderr.write(" ".join(cmd) + "\n" + r.stdout + r.stderr)
        raise RuntimeError(f"build step failed: {os.path.basename(cmd[-1])}")
    return r


def build(clean: bool = False, verbose: bool = False) -> str:
    if clean and os.path.isdir(BUILD):
        shutil.rmtree(BUILD)
    os.makedirs(BUILD, exist_ok=True)
    deps = [os.path.join(CSRC, h) for h in HEADERS] + [
        os.path.join(INCLUDE, f) for f in os.listdir(INCLUDE)]
    objs = []
    for src in CU_SOURCES:
        s = os.path.join(CSRC, src)
        o = os.path.join(BUILD, src + ".o")
        if _newer([s] + deps, o):
            if verbose:
                print("nvcc", src)
            _run([NVCC] + NVCC_FLAGS + ["-c", s, "-o", o])
        objs.append(o)
    for src in CPP_SOURCES:
        s = os.path.join(CSRC, src)
        o = os.path.join(BUILD, src + ".o")
        if _newer([s] + deps, o):
            if verbose:
                print("g++", src)
            _run([CXX] + CXX_FLAGS + ["-c", s, "-o", o])
        objs.append(o)
    if _newer(objs, LIB):
        _run([NVCC] + ARCH + ["-shared", "-cudart", "shared", "-ccbin", CXX, "-o", LIB] + objs)
    demo_src = os.path.join(CSRC, "conv2d_demo.cpp")
    if os.path.exists(demo_src) and _newer([demo_src, LIB] + deps, DEMO):
        _run([CXX] + CXX_FLAGS + ["-o", DEMO, demo_src, "-L", BUILD, "-lwinoconv",
                                  "-Wl,-rpath,$ORIGIN", "-L", os.path.join(CUDA_HOME, "lib64"),
                                  "-lcudart"])
    return LIB


if __name__ == "__main__":
    build(clean="--clean" in sys.argv, verbose=True)
    print(LIB)
