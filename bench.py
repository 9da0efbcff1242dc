#!/usr/bin/env python
"""Benchmark of the B200 Winograd F(2x2,3x3) fp16 conv2d.

One step = one forward conv of the single-large-layer workload
(N=128, C=K=256, H=W=28, 3x3, stride 1, pad 1; x = ReLU(N(0,1)),
w ~ N(0, 2/(9C)), seed 0), run through the drop-in ABI exactly as the
reference harness runs it: getkernelInfo once, then per step the four launch
slots (for this even-sized layer: filter transform, input pre-pass writing
the transformed tiles to transform_pin, tap GEMM writing M to mid_result,
output transform).

Printed (rank 0, one JSON line):
  value      direct-conv-equivalent TFLOP/s (2*N*K*C*P*Q*9 / time), whole job,
             inputs resident in HBM, L2 flushed between steps
  e2e        the same metric through the C-ABI with host buffers: each step
             copies x host->device, runs the four slots, copies y back
  roofline   the step's slowest kernel against its own roofline (the slower
             of Winograd GEMM FLOPs 2*16*K*C*N*ceil(P/2)*ceil(Q/2) over the
             measured bf16 GEMM peak and its compulsory DRAM bytes over the
             measured copy bandwidth, MEASURED_PEAKS.json), each kernel timed
             alone by CUDA events; roofline.kernels lists all three
  cpu_baseline  the reference's own conv2dcpu (oracle/_ref) on this host's
             cores over a bounded sample of images
plus the fused-vs-unfused comparison and the error against FP64.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
Multi-GPU (torchrun): every rank runs an independent replica (the operator
does not shard); value = all ranks' FLOPs / max-over-ranks time.
"""
from __future__ import annotations

import argparse
import ctypes
import importlib
import json
import os
import statistics
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

WORKLOAD = dict(n=128, c=256, h=28, w=28, k=256)
WORKLOAD_NAME = "conv2d N128 C256 H28 W28 K256 3x3 s1 p1 fp16 (single large layer)"
METRIC = "direct-conv-equiv TFLOP/s"
L2_FLUSH_BYTES = 256 << 20  # > 126 MB L2


def direct_flops(n, c, h, w, k):
    return 2.0 * n * k * c * h * w * 9


def wino_flops(n, c, h, w, k):
    return 2.0 * 16 * k * c * n * ((h + 1) // 2) * ((w + 1) // 2)


def replica_throughput(local_ms, flops_per_rank, world, device):
    """Whole-job throughput of `world` independent replicas: every rank did
    `flops_per_rank` in `local_ms`; the job ends with its slowest rank, so the
    time is the max over ranks (all_reduce MAX; every rank calls this) and the
    value all ranks' FLOPs over it.  Returns (max_ms, TFLOP/s)."""
    max_ms = float(local_ms)
    if world > 1:
        import torch
        t = torch.tensor([max_ms], dtype=torch.float64, device=device)
        torch.distributed.all_reduce(t, op=torch.distributed.ReduceOp.MAX)
        max_ms = float(t.item())
    return max_ms, flops_per_rank * world / (max_ms * 1e-3) / 1e12


def measured_peaks():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(path) as f:
            d = json.load(f)
        return dict(hbm_gbs=d["hbm_gbs"], tflops=d["bf16_tflops"],
                    tflops_sustained=d.get("bf16_tflops_sustained"), source="measured")
    except (OSError, KeyError, ValueError):
        return dict(hbm_gbs=6650.0, tflops=1590.0, tflops_sustained=1400.0, source="fallback")


def committed_traffic(kernel):
    """DRAM bytes per launch of `kernel` from the committed ncu summaries, if any."""
    if kernel == "fused_wino_f16_kernel":
        name = "fused_conv_n128_c256_h28.json"
    else:
        name = "twostage_conv_n128_c256_h28.json"
    try:
        with open(os.path.join(ROOT, "profiles", name)) as f:
            d = json.load(f)
        if "kernels" in d:
            return d["kernels"].get(kernel, {}).get("dram_bytes_per_launch")
        return d.get("dram_bytes_per_launch")
    except (OSError, ValueError):
        return None


def kernel_roofline(name, us, flops, nbytes, peaks):
    """One kernel against its roofline: the slower of its tensor time
    (flops / measured bf16 GEMM peak) and its HBM time (compulsory bytes /
    measured copy bandwidth) decides the bound; achieved and peak are in
    that bound's unit."""
    t_tensor = flops / (peaks["tflops"] * 1e12) if flops else 0.0
    t_hbm = nbytes / (peaks["hbm_gbs"] * 1e9)
    if t_tensor >= t_hbm:
        achieved, peak, unit, bound = flops / (us * 1e-6) / 1e12, peaks["tflops"], "TFLOP/s", "tensor"
    else:
        achieved, peak, unit, bound = nbytes / (us * 1e-6) / 1e9, peaks["hbm_gbs"], "GB/s", "hbm"
    return {"kernel": name, "bound": bound, "achieved": achieved, "peak": peak, "unit": unit,
            "frac": achieved / peak, "us": us, "flops": flops, "bytes": nbytes,
            "floor_us": max(t_tensor, t_hbm) * 1e6, "traffic": committed_traffic(name),
            "peak_source": peaks["source"]}


# ------------------------------------------------------------------ clocks --
class ClockSampler:
    """Samples SM clock, power and throttle reasons through NVML."""

    REASONS = {0x8: "hw_slowdown", 0x40: "hw_thermal_slowdown", 0x20: "sw_thermal_slowdown",
               0x4: "sw_power_cap", 0x80: "hw_power_brake_slowdown", 0x1: "gpu_idle"}

    def __init__(self, index, period_s=0.005):
        self.samples = []
        self.period = period_s
        self._stop = threading.Event()
        self._thread = None
        try:
            import pynvml
            pynvml.nvmlInit()
            self.nvml = pynvml
            self.h = pynvml.nvmlDeviceGetHandleByIndex(index)
            self.max_sm = pynvml.nvmlDeviceGetMaxClockInfo(self.h, pynvml.NVML_CLOCK_SM)
        except Exception:  # noqa: BLE001 - NVML absent: report no clocks
            self.nvml = None
            self.max_sm = None

    def _run(self):
        nv = self.nvml
        while not self._stop.is_set():
            try:
                sm = nv.nvmlDeviceGetClockInfo(self.h, nv.NVML_CLOCK_SM)
                rs = nv.nvmlDeviceGetCurrentClocksEventReasons(self.h)
                pw = nv.nvmlDeviceGetPowerUsage(self.h) / 1000.0
                self.samples.append((sm, rs, pw))
            except Exception:  # noqa: BLE001
                pass
            time.sleep(self.period)

    def __enter__(self):
        if self.nvml:
            self._thread = threading.Thread(target=self._run, daemon=True)
            self._thread.start()
        return self

    def __exit__(self, *exc):
        self._stop.set()
        if self._thread:
            self._thread.join()

    def summary(self):
        if not self.samples:
            return {"sm_mhz": None, "sm_max_mhz": self.max_sm, "reasons": [], "samples": 0}
        busy = [s for s in self.samples if not (s[1] & 0x1)] or self.samples
        reasons = set()
        for _, rs, _ in busy:
            for bit, name in self.REASONS.items():
                if rs & bit and name != "gpu_idle":
                    reasons.add(name)
        return {"sm_mhz": statistics.median(s[0] for s in busy), "sm_max_mhz": self.max_sm,
                "reasons": sorted(reasons), "samples": len(busy),
                "power_w_max": max(s[2] for s in busy)}


# ------------------------------------------------------------- CPU legs -----
def cpu_info():
    """CPU model string and logical CPU count of this host (lscpu / nproc)."""
    model = None
    try:
        with open("/proc/cpuinfo") as f:
            for line in f:
                if line.startswith("model name"):
                    model = line.split(":", 1)[1].strip()
                    break
    except OSError:
        pass
    return {"cpu_model": model, "nproc": os.cpu_count()}


BUILD_FLAGS = {"portable": "g++ -O3 -march=x86-64-v3 (fp16 products evaluated exactly in float)",
               "avx512fp16": "g++ -O3 -march=x86-64-v4 -mavx512fp16 (products rounded to fp16)"}


def cpu_reference_sample(seed=0, images=None, threads=None, variant=None):
    """Time the reference's conv2dcpu (oracle/_ref, unmodified verfiy.h) on
    `images` images of the workload.  threads == 1 calls it once over all the
    images, exactly as the reference harness does (src/main.cpp:138);
    otherwise an OpenMP loop calls it once per image."""
    import numpy as np
    import oracle
    variants = oracle.ref_variants()
    if variant is None:
        variant = "avx512fp16" if "avx512fp16" in variants else "portable"
    threads = threads or oracle.ref_max_threads(variant)
    images = images or max(2, threads)
    W = WORKLOAD
    x, w = oracle.make_inputs(images, W["c"], W["h"], W["w"], W["k"], seed=seed,
                              x_dist="relu_normal", w_std=np.sqrt(2.0 / (9 * W["c"])))
    t0 = time.perf_counter()
    oracle.ref_conv2dcpu(x, w, threads=threads, variant=variant)
    dt = time.perf_counter() - t0
    flops = direct_flops(images, W["c"], W["h"], W["w"], W["k"])
    return dict(tflops=flops / dt / 1e12, seconds=dt, images=images, threads=threads,
                variant=variant)


def cpu_baseline_modes():
    """The reference CPU path in every mode this host offers: each build
    (exact products; fp16-rounded products where the CPU has AVX512-FP16)
    with one thread exactly as the reference calls it and with all host
    threads.  Returns (modes, headline) where headline is the fastest mode."""
    import oracle
    modes = []
    for variant in oracle.ref_variants():
        allt = oracle.ref_max_threads(variant)
        for threads, images in ((1, 2), (allt, 2 * allt)):
            r = cpu_reference_sample(seed=0, images=images, threads=threads, variant=variant)
            modes.append({"build": variant, "flags": BUILD_FLAGS.get(variant), "threads": threads,
                          "images": images, "seconds": r["seconds"], "value": r["tflops"],
                          "unit": "TFLOP/s"})
    best = max(modes, key=lambda m: m["value"]) if modes else None
    return modes, best


def run_reference_arm(args, rank):
    """The reference's own CPU implementation (conv2dcpu) on the host cores
    with every thread, on the GPU arm's workload.  Each step runs as many of
    the workload's 128 images as fit a budget of about 150 s for the whole
    run (all 128 when the host is fast enough)."""
    if rank != 0:
        return 0
    import oracle
    variants = oracle.ref_variants()
    variant = "avx512fp16" if "avx512fp16" in variants else "portable"
    threads = oracle.ref_max_threads(variant)
    cal = cpu_reference_sample(seed=0, images=threads, threads=threads, variant=variant)
    per_image = cal["seconds"] / cal["images"]
    budget = 150.0 / max(1, args.steps + args.warmup)
    images = int(budget / per_image) // threads * threads
    images = max(threads, min(WORKLOAD["n"], images))
    samples = []
    for i in range(args.warmup + args.steps):
        r = cpu_reference_sample(seed=i, images=images, threads=threads, variant=variant)
        if i >= args.warmup:
            samples.append(r)
    secs = sum(s["seconds"] for s in samples)
    flops = sum(direct_flops(s["images"], WORKLOAD["c"], WORKLOAD["h"], WORKLOAD["w"],
                             WORKLOAD["k"]) for s in samples)
    value = flops / secs / 1e12
    full = images == WORKLOAD["n"]
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": "TFLOP/s",
        "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": secs / len(samples) * 1e3, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f16", "data": "synthetic (seeded)",
        "config": {"workload": WORKLOAD_NAME, **WORKLOAD,
                   "step": (f"all {images} images of the workload" if full else
                            f"{images} of {WORKLOAD['n']} images of the workload") + " on the host CPU"},
        "cpu_baseline": {"value": value, "unit": "TFLOP/s", "cores": threads,
                         "kind": "reference",
                         "sample": f"{images} of {WORKLOAD['n']} images per step, conv2dcpu build "
                                   f"'{variant}' ({BUILD_FLAGS.get(variant)}), OpenMP over images",
                         **cpu_info()},
        "e2e": {"value": value, "unit": "TFLOP/s", "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)
    return 0


# ------------------------------------------------------------- GPU arm ------
def run_ours(args, rank, world, local_rank):
    import numpy as np
    import torch
    import oracle
    wino = importlib.import_module("2024pra_conv_b200")
    dev = torch.device("cuda", local_rank)
    torch.cuda.set_device(dev)
    W = WORKLOAD
    n, c, h, w, k = W["n"], W["c"], W["h"], W["w"], W["k"]
    x16, w16 = oracle.make_inputs(n, c, h, w, k, seed=rank, x_dist="relu_normal",
                                  w_std=np.sqrt(2.0 / (9 * c)))
    x = torch.from_numpy(x16).to(dev)
    wt = torch.from_numpy(w16).to(dev)
    y = torch.empty((n, k, h, w), dtype=torch.float16, device=dev)
    flush = torch.empty(L2_FLUSH_BYTES, dtype=torch.uint8, device=dev)
    stream = torch.cuda.current_stream()

    # drop-in ABI: problem, getParamsize, getkernelInfo (once, as the harness)
    dws = wino.DropinWorkspaces(n, c, h, w, k, dev)   # the harness's caller buffers
    pr = wino.make_problem(x, wt, y, dws.transform_pin, dws.transform_filter, dws.mid_result)
    param = (ctypes.c_char * wino.get_param_size(pr))()
    code, ki = wino.get_kernel_info(pr, param)
    if code != 0:
        raise SystemExit(f"getkernelInfo failed: {code}")

    def step():
        wino.launch_kernel_info(ki, param, stream)

    ev = lambda: torch.cuda.Event(enable_timing=True)

    def timed(fn, iters, flush_between=True):
        """Sum of per-iteration CUDA-event times (ms) on the current stream."""
        total = 0.0
        times = []
        for _ in range(iters):
            if flush_between:
                flush.zero_()
            a, b = ev(), ev()
            a.record(stream)
            fn()
            b.record(stream)
            b.synchronize()
            dt = a.elapsed_time(b)
            times.append(dt)
            total += dt
        return total, times

    sampler = ClockSampler(local_rank)
    with sampler:
        for _ in range(max(args.warmup, 3)):
            step()
        torch.cuda.synchronize()
        # soak so the clocks under load are steady before the timed steps
        t_end = time.time() + args.soak
        while time.time() < t_end:
            step()
        torch.cuda.synchronize()
        if world > 1:
            torch.distributed.barrier()
        torch.cuda.synchronize()
        total_ms, step_ms = timed(step, args.steps)
        torch.cuda.synchronize()
        if world > 1:
            torch.distributed.barrier()
    clocks = sampler.summary()

    dflops = direct_flops(n, c, h, w, k)
    max_ms, value = replica_throughput(total_ms, dflops * args.steps, world, dev)

    # --- parity of the timed path (outside the timed region)
    y64 = torch.nn.functional.conv2d(x.double(), wt.double(), padding=1)
    yd = y.double()
    rel_l2 = float(torch.linalg.vector_norm(yd - y64) / torch.linalg.vector_norm(y64))
    max_norm = float((yd - y64).abs().max() / y64.abs().max())
    y64_ref = y64                               # kept for the end-to-end check below
    del yd

    # --- per-kernel pieces: filter transform, fused conv on cached U, unfused path
    ucache = wino.filter_transform(wt)
    torch.cuda.synchronize()
    iters = max(args.steps, 10)
    ft_ms, _ = timed(lambda: wino.filter_transform(wt, stream), iters)
    yf = torch.empty_like(y)
    xbws = torch.empty(wino.fused_workspace_bytes(n, c, h, w), dtype=torch.uint8, device=dev)
    fused_ms, fused_times = timed(
        lambda: wino.conv2d_fused(x, ucache, k, out=yf, stream=stream, workspace=xbws), iters)
    layout_ms, _ = timed(lambda: wino.input_layout(x, xbws, stream), iters)
    u2 = wino.filter_transform_unfused(wt)
    # two-stage path on cached U: pre-pass + tap GEMM + output transform
    ts_ws = wino._aligned_ws(wino.twostage_workspace_bytes(n, c, h, w, k), dev)
    yt = torch.empty_like(y)
    ts_ms, _ = timed(lambda: wino.conv2d_twostage(x, u2, k, out=yt, workspace=ts_ws, stream=stream), iters)
    ts_pre_ms, _ = timed(lambda: wino.twostage_stage(0, x, u2, k, yt, ts_ws, stream), iters)
    ts_gemm_ms, _ = timed(lambda: wino.twostage_stage(1, x, u2, k, yt, ts_ws, stream), iters)
    ts_out_ms, _ = timed(lambda: wino.twostage_stage(2, x, u2, k, yt, ts_ws, stream), iters)
    del ts_ws
    ws = wino.UnfusedWorkspace(n, c, h, w, k, dev)
    yu = torch.empty_like(y)
    unf_ms, _ = timed(lambda: wino.conv2d_unfused(x, u2, k, ws=ws, out=yu, stream=stream), iters)
    torch.cuda.synchronize()
    unf_rel = float(torch.linalg.vector_norm(yu.double() - y.double()) /
                    torch.linalg.vector_norm(y.double()))
    del ws
    fused_us = fused_ms / iters * 1e3          # pre-pass + fused kernel
    layout_us = layout_ms / iters * 1e3         # pre-pass alone
    kernel_us = max(fused_us - layout_us, 1e-3)  # the fused kernel
    unfused_us = unf_ms / iters * 1e3
    ft_us = ft_ms / iters * 1e3
    ts_us, ts_pre_us, ts_gemm_us, ts_out_us = (ts_ms / iters * 1e3, ts_pre_ms / iters * 1e3,
                                               ts_gemm_ms / iters * 1e3, ts_out_ms / iters * 1e3)
    # the route getkernelInfo chose for the timed drop-in step
    two_stage = ki.slot(3)["kernel"] == wino.lib().wino_twostage_gemm_kernel_ptr_for(c)

    # --- end to end through the C-ABI with host buffers.  Every step uploads
    # its input from pinned host memory, runs the drop-in slots and downloads
    # its output; consecutive steps are pipelined over two buffer sets and
    # three streams (upload / compute / download), so step i's download
    # overlaps step i+1's upload and compute (PCIe is full duplex).
    xh = torch.empty_like(x, device="cpu").pin_memory()
    xh.copy_(x)
    yh = [torch.empty_like(y, device="cpu").pin_memory() for _ in range(2)]
    xd = [x, torch.empty_like(x)]
    yd = [y, torch.empty_like(y)]
    dws2 = wino.DropinWorkspaces(n, c, h, w, k, dev)
    params, kis = [], []
    for bset in range(2):
        ws_b = dws if bset == 0 else dws2
        pr_b = wino.make_problem(xd[bset], wt, yd[bset], ws_b.transform_pin, ws_b.transform_filter,
                                 ws_b.mid_result)
        prm = (ctypes.c_char * wino.get_param_size(pr_b))()
        code, ki_b = wino.get_kernel_info(pr_b, prm)
        if code != 0:
            raise SystemExit(f"getkernelInfo failed: {code}")
        params.append(prm)
        kis.append(ki_b)
    s_up, s_comp, s_down = torch.cuda.Stream(), torch.cuda.Stream(), torch.cuda.Stream()
    up_done = [torch.cuda.Event() for _ in range(2)]
    comp_done = [torch.cuda.Event() for _ in range(2)]
    down_done = [torch.cuda.Event() for _ in range(2)]
    started = [False, False]

    def e2e_run(steps_):
        for i in range(steps_):
            bset = i % 2
            with torch.cuda.stream(s_up):
                if started[bset]:
                    s_up.wait_event(comp_done[bset])       # the compute has read xd[bset]
                xd[bset].copy_(xh, non_blocking=True)
                up_done[bset].record(s_up)
            s_comp.wait_event(up_done[bset])
            if started[bset]:
                s_comp.wait_event(down_done[bset])         # the download has read yd[bset]
            wino.launch_kernel_info(kis[bset], params[bset], s_comp)
            comp_done[bset].record(s_comp)
            with torch.cuda.stream(s_down):
                s_down.wait_event(comp_done[bset])
                yh[bset].copy_(yd[bset], non_blocking=True)
                down_done[bset].record(s_down)
            started[bset] = True

    e2e_run(2)
    torch.cuda.synchronize()
    a_ev, b_ev = ev(), ev()
    a_ev.record(s_up)
    e2e_run(args.steps)
    s_down.wait_stream(s_up)
    s_down.wait_stream(s_comp)
    b_ev.record(s_down)
    b_ev.synchronize()
    e2e_ms = a_ev.elapsed_time(b_ev)
    torch.cuda.synchronize()
    e2e_err = float((yh[(args.steps - 1) % 2].to(dev).double() - y64_ref).norm() / y64_ref.norm())
    _, e2e_value = replica_throughput(e2e_ms, dflops * args.steps, world, dev)
    del dws2, xd, yd

    errcode = wino.error_read_clear()
    if errcode:
        raise SystemExit(f"device error word {errcode}")

    if rank != 0:
        return 0
    peaks = measured_peaks()
    wflops = wino_flops(n, c, h, w, k)
    L = wino.lib()
    tiles = n * ((h + 1) // 2) * ((w + 1) // 2)
    x_bytes, y_bytes = n * c * h * w * 2, n * k * h * w * 2
    m_bytes, u_bytes = 16 * k * tiles * 2, 16 * k * c * 2
    if two_stage:
        pre_bytes = L.wino_twostage_prepass_bytes(n, c, h, w)
        gk = L.wino_twostage_gemm_kernel_ptr_for(c)
        gname = ("twostage_res_kernel_t<1>" if gk == L.wino_twostage_resv_kernel_ptr() else
                 "twostage_res_kernel_t<0>" if gk == L.wino_twostage_res_kernel_ptr() else
                 "twostage_pair_kernel" if gk == L.wino_twostage_pair_kernel_ptr() else "twostage_stream_kernel")
        pname = "v2_layout_kernel" if gk == L.wino_twostage_resv_kernel_ptr() else "prepass"
        kern = [kernel_roofline(pname, ts_pre_us, 0, x_bytes + pre_bytes, peaks),
                kernel_roofline(gname, ts_gemm_us, wflops, pre_bytes + u_bytes + m_bytes, peaks),
                kernel_roofline("twostage_output_kernel", ts_out_us, 0, m_bytes + y_bytes, peaks)]
    else:
        kern = [kernel_roofline("fused_wino_f16_kernel", kernel_us, wflops, x_bytes + y_bytes + u_bytes, peaks)]
    dom = max(kern, key=lambda r: r["us"])
    roofline = {k2: dom[k2] for k2 in ("bound", "achieved", "peak", "unit", "frac", "traffic", "peak_source",
                                       "kernel")}
    roofline["algorithmic"] = (f"{dom['bytes'] / 1e6:.1f} MB compulsory DRAM bytes and {dom['flops'] / 1e9:.2f} "
                               "Winograd GEMM GFLOP per launch; the bound is the slower of the two")
    roofline["kernels"] = kern
    roofline["step_floor_us"] = sum(r["floor_us"] for r in kern)
    roofline["step_frac_of_kernel_floors"] = roofline["step_floor_us"] / (max_ms / args.steps * 1e3)
    cpu = None
    if world == 1 and not args.no_cpu:
        try:
            modes, best = cpu_baseline_modes()
            cpu = {"value": best["value"], "unit": "TFLOP/s", "cores": best["threads"],
                   "kind": "reference",
                   "sample": f"{best['images']} of {n} images of the workload, reference conv2dcpu "
                             f"build '{best['build']}' on {best['threads']} threads, "
                             f"{best['seconds']:.1f} s (fastest of the modes below)",
                   "modes": modes, **cpu_info()}
        except Exception as e:  # noqa: BLE001 - report, do not fail the GPU numbers
            cpu = {"value": None, "unit": "TFLOP/s", "cores": None, "kind": "reference",
                   "sample": f"unavailable: {e}", **cpu_info()}
    line = {
        "metric": METRIC, "value": value, "unit": "TFLOP/s", "n_gpus": world,
        "steps": args.steps, "warmup": max(args.warmup, 3), "ms_per_step": max_ms / args.steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f16",
        "data": "synthetic (seeded ReLU(N(0,1)) input, N(0,2/(9C)) weights)",
        "config": {"workload": WORKLOAD_NAME, **W, "parallelism": f"replicas x{world}",
                   "step": ("drop-in ABI: filter transform + input pre-pass (transformed tiles) + tap GEMM + "
                            "output transform" if two_stage else
                            "drop-in ABI: filter transform + input re-layout + fused conv + 1 empty slot"),
                   "l2": "flushed between steps (256 MB write)"},
        "us_per_layer": max_ms / args.steps * 1e3,
        "fused_us_cached_u": fused_us,
        "input_layout_us": layout_us,
        "fused_kernel_us": kernel_us,
        "fused_direct_equiv_tflops": dflops / (fused_us * 1e-6) / 1e12,
        "filter_transform_us": ft_us,
        "two_stage_us_cached_u": ts_us,
        "two_stage_prepass_us": ts_pre_us,
        "two_stage_gemm_us": ts_gemm_us,
        "two_stage_output_us": ts_out_us,
        "unfused_us": unfused_us,
        "speedup_vs_unfused": unfused_us / (ts_us if two_stage else fused_us),
        "rel_l2": rel_l2, "max_norm": max_norm, "unfused_rel_diff": unf_rel,
        "roofline": roofline,
        "cpu_baseline": cpu,
        "e2e": {"value": e2e_value, "unit": "TFLOP/s", "h2d_bytes_per_step": x.numel() * 2,
                "d2h_bytes_per_step": y.numel() * 2, "rel_l2_of_downloaded_output": e2e_err,
                "pipelining": "2 buffer sets, upload / compute / download streams"},
        "gpu_launches": 4 * args.steps,
        "clocks": clocks,
    }
    if world == 1 and not args.no_extras:
        line["extensions"] = extension_legs(wino, dev, flush, ev, peaks, max(args.steps, 5))
    print(json.dumps(line), flush=True)
    return 0


def extension_legs(wino, dev, flush, ev, peaks, steps):
    """Rank-0 extras on the other workloads: the batched 12-layer ResNet-style
    set (autotuned, one persistent launch, CUDA graph), the precision
    variants on N64 C=K256 H14 with their errors against FP64, Winograd
    F(4x4,3x3) beside F(2x2) on N128 C256 H28, the fused epilogue, and the
    learned cost model measured against exhaustive tuning on the committed
    timings.  Not part of `value`."""
    import numpy as np
    import torch
    import oracle
    out = {}
    stream = torch.cuda.current_stream()

    def timed(fn, iters, do_flush=True):
        ts = []
        for _ in range(iters):
            if do_flush:
                flush.zero_()
            a, b = ev(), ev()
            a.record(stream)
            fn()
            b.record(stream)
            b.synchronize()
            ts.append(a.elapsed_time(b))
        return statistics.median(ts) * 1e3  # us

    # --- batched layer set, N=32
    n = 32
    layers = []
    dfl = 0.0
    t_roof = 0.0          # sum over layers of max(t_HBM, t_tensor)
    n_tc = 0
    for i, (c, k, h) in enumerate(wino.RESNET_LAYER_SET):
        x16, w16 = oracle.make_inputs(n, c, h, h, k, seed=100 + i, x_dist="uniform",
                                      w_std=np.sqrt(2.0 / (9 * c)))
        x = torch.from_numpy(x16).to(dev)
        wt = torch.from_numpy(w16).to(dev)
        u = wino.filter_transform(wt)
        ws = torch.empty(wino.fused_workspace_bytes(n, c, h, h), dtype=torch.uint8, device=dev)
        y = torch.empty((n, k, h, h), dtype=torch.float16, device=dev)
        layers.append((x, wt, u, ws, y, c, k, h))
        dfl += direct_flops(n, c, h, h, k)
        byt = 2.0 * (n * c * h * h + n * k * h * h + 16 * k * c)
        t_hbm = byt / (peaks["hbm_gbs"] * 1e9)
        t_tc = wino_flops(n, c, h, h, k) / (peaks["tflops"] * 1e12)
        t_roof += max(t_hbm, t_tc)
        n_tc += t_tc > t_hbm
    seq_us = timed(lambda: [wino.conv2d_fused(x, u, k, out=y, workspace=ws)
                            for (x, wt, u, ws, y, c, k, h) in layers], steps)
    b = wino.Batch()
    for (x, wt, u, ws, y, c, k, h) in layers:
        b.add(x, u, k, y, workspace=ws)
    b.run()
    untuned_us = timed(b.run, steps)
    layer_us, order_us = b.tune(reps=3)
    b.capture()
    b.launch()
    torch.cuda.synchronize()
    graph_us = timed(b.launch, steps)
    worst = 0.0
    for (x, wt, u, ws, y, c, k, h) in layers:
        y64 = torch.nn.functional.conv2d(x.double(), wt.double(), padding=1)
        worst = max(worst, float(torch.linalg.vector_norm(y.double() - y64) / torch.linalg.vector_norm(y64)))
    # each layer alone with its tuned configuration (pre-pass + fused kernel),
    # against its own roofline, to show which layer classes lose the time
    per_layer = []
    for i, (x, wt, u, ws, y, c, k, h) in enumerate(layers):
        cfg = b.config(i)
        cws = wino._aligned_ws(wino.cfg_workspace_bytes(n, c, h, h, k, cfg), dev)
        us = timed(lambda: wino.conv2d_fused_cfg(x, u, k, cfg, workspace=cws, out=y), steps)
        byt = 2.0 * (n * c * h * h + n * k * h * h + 16 * k * c)
        t_hbm = byt / (peaks["hbm_gbs"] * 1e9) * 1e6
        t_tc = wino_flops(n, c, h, h, k) / (peaks["tflops"] * 1e12) * 1e6
        per_layer.append({"c": c, "k": k, "h": h, "cfg": cfg, "us": us, "bound_us": max(t_hbm, t_tc),
                          "bound": "tensor" if t_tc > t_hbm else "hbm",
                          "frac": max(t_hbm, t_tc) / us})
        del cws
    out["layer_set"] = {
        "workload": "12 ResNet-style 3x3 s1 p1 layers at N=32, (C,K,H): " +
                    ", ".join(f"({c},{k},{h})" for (c, k, h) in wino.RESNET_LAYER_SET),
        "us_graph_tuned": graph_us, "us_persistent_untuned": untuned_us, "us_sequential_launches": seq_us,
        "direct_equiv_tflops": dfl / (graph_us * 1e-6) / 1e12,
        "configs": [b.config(i) for i in range(len(layers))], "order": b.order(),
        # the tuner's route per layer (0 fused tile blocks of 128 k x 32 tiles, 1 two-stage
        # tap-GEMM units of 128 tiles x 256 k) with each layer's time alone on both routes
        "routes": [b.route(i)[0] for i in range(len(layers))],
        "alone_us_fused_twostage": [[round(b.route(i)[1], 1), round(b.route(i)[2], 1)] for i in range(len(layers))],
        "order_us": order_us, "worst_rel_l2": worst, "per_layer_alone": per_layer,
        "roofline": {"per_layer_bound": f"{n_tc} of 12 layers tensor-bound, the rest HBM-bound",
                     "target_us": t_roof * 1e6, "frac": t_roof * 1e6 / graph_us,
                     "definition": "sum over layers of max(HBM bytes / hbm_gbs, Winograd FLOPs / "
                                   "bf16_tflops) over the measured time"},
        "l2": "flushed between steps"}
    b.close()
    del layers

    # --- precision variants, N64 C=K256 H14 (uniform inputs)
    x16, w16 = oracle.make_inputs(64, 256, 14, 14, 256, seed=0, x_dist="uniform",
                                  w_std=np.sqrt(2.0 / (9 * 256)))
    x = torch.from_numpy(x16).to(dev)
    wt = torch.from_numpy(w16).to(dev)
    y64 = torch.nn.functional.conv2d(x.double(), wt.double(), padding=1)
    var = {}
    for name, v in [("f16", wino.VAR_F16), ("bf16", wino.VAR_BF16), ("f8_e4m3", wino.VAR_F8),
                    ("f16_hilo", wino.VAR_F16_HILO)]:
        ws = torch.empty(wino.variant_workspace_bytes(v, 64, 256, 14, 14, 256) + 256, dtype=torch.uint8,
                         device=dev)
        y = torch.empty((64, 256, 14, 14), dtype=torch.float16, device=dev)
        wino.conv2d_variant(x, wt, v, out=y, workspace=ws)
        torch.cuda.synchronize()
        d = y.double() - y64
        us = timed(lambda: wino.conv2d_variant(x, wt, v, out=y, workspace=ws), steps)
        var[name] = {"us_per_call": us, "rel_l2": float(torch.linalg.vector_norm(d) / torch.linalg.vector_norm(y64)),
                     "max_norm": float(d.abs().max() / y64.abs().max()),
                     "direct_equiv_tflops": direct_flops(64, 256, 14, 14, 256) / (us * 1e-6) / 1e12}
    # the two-stage route's fp16 and fp8 GEMMs on a cached fp16 U (per call:
    # for fp8 the channel maxima, the U and V splits, GEMM, output transform)
    u2 = wino.filter_transform_unfused(wt)
    for name, run in [("two_stage_f16", lambda y: wino.conv2d_twostage(x, u2, 256, out=y)),
                      ("two_stage_f8_hilo", lambda y: wino.conv2d_twostage_f8(x, u2, 256, hilo=True, out=y)),
                      ("two_stage_f8", lambda y: wino.conv2d_twostage_f8(x, u2, 256, hilo=False, out=y))]:
        y = torch.empty((64, 256, 14, 14), dtype=torch.float16, device=dev)
        run(y)
        torch.cuda.synchronize()
        d = y.double() - y64
        us = timed(lambda: run(y), steps)
        var[name] = {"us_per_call": us, "rel_l2": float(torch.linalg.vector_norm(d) / torch.linalg.vector_norm(y64)),
                     "max_norm": float(d.abs().max() / y64.abs().max()),
                     "direct_equiv_tflops": direct_flops(64, 256, 14, 14, 256) / (us * 1e-6) / 1e12}
    out["variants"] = {"workload": "N64 C256 H14 W14 K256, x ~ U[-1,1]; per call: filter transform "
                                   "+ input pre-pass + fused kernel (f16 .. f16_hilo); pre-pass + tap GEMM "
                                   "+ output transform on a cached fp16 U (two_stage_*)", **var}

    # --- Winograd F(4x4,3x3), hi+lo and plain, on N128 C256 H28 K256 against F(2x2) fused
    n, c, h, k = 128, 256, 28, 256
    x16, w16 = oracle.make_inputs(n, c, h, h, k, seed=0, x_dist="relu_normal", w_std=np.sqrt(2.0 / (9 * c)))
    x = torch.from_numpy(x16).to(dev)
    wt = torch.from_numpy(w16).to(dev)
    y64 = torch.nn.functional.conv2d(x.double(), wt.double(), padding=1)
    y = torch.empty((n, k, h, h), dtype=torch.float16, device=dev)
    f4 = {}
    for name, hilo in [("f4_hilo", True), ("f4_f16", False)]:
        conv = wino.ConvF4(wt, n, h, h, hilo=hilo)
        conv(x, out=y)
        torch.cuda.synchronize()
        d = y.double() - y64
        us = timed(lambda: conv(x, out=y), steps)
        f4[name] = {"us_per_call": us,
                    "rel_l2": float(torch.linalg.vector_norm(d) / torch.linalg.vector_norm(y64)),
                    "max_norm": float(d.abs().max() / y64.abs().max()),
                    "direct_equiv_tflops": direct_flops(n, c, h, h, k) / (us * 1e-6) / 1e12,
                    "workspace_bytes": conv.nbytes}
        del conv
    u = wino.filter_transform(wt)
    ws = torch.empty(wino.fused_workspace_bytes(n, c, h, h), dtype=torch.uint8, device=dev)
    wino.conv2d_fused(x, u, k, out=y, workspace=ws)
    torch.cuda.synchronize()
    d = y.double() - y64
    us = timed(lambda: wino.conv2d_fused(x, u, k, out=y, workspace=ws), steps)
    f4["f2_fused_f16"] = {"us_per_call": us,
                          "rel_l2": float(torch.linalg.vector_norm(d) / torch.linalg.vector_norm(y64)),
                          "max_norm": float(d.abs().max() / y64.abs().max()),
                          "direct_equiv_tflops": direct_flops(n, c, h, h, k) / (us * 1e-6) / 1e12}
    u2 = wino.filter_transform_unfused(wt)
    ws2 = wino._aligned_ws(wino.twostage_workspace_bytes(n, c, h, h, k), dev)
    wino.conv2d_twostage(x, u2, k, out=y, workspace=ws2)
    torch.cuda.synchronize()
    d = y.double() - y64
    us = timed(lambda: wino.conv2d_twostage(x, u2, k, out=y, workspace=ws2), steps)
    f4["f2_two_stage_f16"] = {"us_per_call": us,
                              "rel_l2": float(torch.linalg.vector_norm(d) / torch.linalg.vector_norm(y64)),
                              "direct_equiv_tflops": direct_flops(n, c, h, h, k) / (us * 1e-6) / 1e12}
    del u2, ws2
    out["winograd_f4"] = {"workload": "N128 C256 H28 K256, x = relu(N(0,1)); transformed filter cached; "
                                      "per call: input transform + 36-tap GEMM + output transform (F4), "
                                      "pre-pass + fused kernel (F2), pre-pass + tap GEMM + "
                                      "output transform (F2 two-stage)", **f4}
    del x, wt, y64, y, u, ws

    # --- fused epilogue (bias + residual + ReLU) vs the conv then separate elementwise ops
    n, c, h, k = 128, 256, 28, 256
    x16, w16 = oracle.make_inputs(n, c, h, h, k, seed=0, x_dist="relu_normal", w_std=np.sqrt(2.0 / (9 * c)))
    x = torch.from_numpy(x16).to(dev)
    wt = torch.from_numpy(w16).to(dev)
    u = wino.filter_transform(wt)
    ws = torch.empty(wino.fused_workspace_bytes(n, c, h, h), dtype=torch.uint8, device=dev)
    bias = torch.randn(k, device=dev) * 0.1
    res = torch.randn((n, k, h, h), device=dev).half()
    y = torch.empty((n, k, h, h), dtype=torch.float16, device=dev)
    bias16 = bias.half().view(1, k, 1, 1)
    fused_ep = timed(lambda: wino.conv2d_fused_epilogue(x, u, k, bias=bias, residual=res, relu=True, out=y,
                                                        workspace=ws), steps)

    def separate():
        wino.conv2d_fused(x, u, k, out=y, workspace=ws)
        torch.relu_(y.add_(bias16).add_(res))

    sep = timed(separate, steps)
    out["fused_epilogue"] = {"workload": "N128 C256 H28 K256: relu(conv + bias + residual)",
                             "us_fused": fused_ep, "us_conv_then_torch_elementwise": sep}
    del x, wt, u, ws, res, y

    # --- tensor-core implicit GEMM on the shapes outside the Winograd contract
    out["implicit_gemm"] = implicit_gemm_leg(wino, dev, timed, peaks, steps)

    # --- learned cost model vs exhaustive tuning (committed timings)
    path = os.path.join(ROOT, "tests", "golden", "tuning_timings.json")
    if os.path.exists(path):
        cm = importlib.import_module("2024pra_conv_b200.costmodel")
        with open(path) as f:
            rows = json.load(f)["rows"]
        r = cm.evaluate(rows)
        r.pop("regret")
        out["cost_model"] = {"data": "exhaustive tuning timings of 400 seeded shapes "
                                     "(tests/golden/tuning_timings.json), 300 train / 100 held out", **r}
    err = wino.error_read_clear()
    if err:
        raise SystemExit(f"device error word {err}")
    return out


# ResNet-50 layers at N = 128 that the Winograd path does not take (1x1
# projections and expansions, stride-2 3x3 downsampling): name, c, h, k, r,
# stride, pad.
IGEMM_LAYERS = [
    ("1x1 64->256 h56", 64, 56, 256, 1, 1, 0),
    ("1x1 256->64 h56", 256, 56, 64, 1, 1, 0),
    ("1x1 256->128 h56 s2", 256, 56, 128, 1, 2, 0),
    ("3x3 128 s2 h56", 128, 56, 128, 3, 2, 1),
    ("1x1 512->128 h28", 512, 28, 128, 1, 1, 0),
    ("1x1 128->512 h28", 128, 28, 512, 1, 1, 0),
    ("3x3 256 s2 h28", 256, 28, 256, 3, 2, 1),
    ("1x1 1024->256 h14", 1024, 14, 256, 1, 1, 0),
    ("3x3 512 s2 h14", 512, 14, 512, 3, 2, 1),
]


def implicit_gemm_leg(wino, dev, timed, peaks, steps):
    """Each IGEMM_LAYERS layer at N = 128 through the tcgen05 implicit GEMM
    (weights re-laid out once, L2 flushed before every call) beside the
    CUDA-core direct kernel it replaces and the library convolution
    (torch / cuDNN, fp16), with its roofline: floor = max(input + output +
    weight bytes / HBM peak, direct FLOPs / bf16 peak).  rel-L2 against FP64
    on the first 4 images."""
    import torch
    n = 128
    rows = []
    t_sum = floor_sum = 0.0
    for name, c, h, k, r, st, pd in IGEMM_LAYERS:
        g = torch.Generator(device=dev).manual_seed(c * 131 + h * 7 + k)
        x = torch.randn((n, c, h, h), device=dev, generator=g).half()
        wt = (torch.randn((k, c, r, r), device=dev, generator=g) / (c * r * r) ** 0.5).half()
        oh = (h - r + 2 * pd) // st + 1
        y = torch.empty((n, k, oh, oh), dtype=torch.float16, device=dev)
        wp = wino.igemm_weight_transform(wt)
        us = timed(lambda: wino.conv2d_igemm(x, wt, stride=st, pad=pd, wprep=wp, out=y), steps)
        us_direct = timed(lambda: wino.conv2d_direct(x, wt, stride=st, pad=pd, out=y), max(3, steps // 4))
        us_lib = timed(lambda: torch.nn.functional.conv2d(x, wt, stride=st, padding=pd), steps)
        xs = x[:4].contiguous()
        ys = wino.conv2d_igemm(xs, wt, stride=st, pad=pd, wprep=wp)
        y64 = torch.nn.functional.conv2d(xs.double(), wt.double(), stride=st, padding=pd)
        rl2 = float(torch.linalg.vector_norm(ys.double() - y64) / torch.linalg.vector_norm(y64))
        flops = 2.0 * n * oh * oh * k * c * r * r
        nbytes = 2.0 * (x.numel() + y.numel() + wt.numel())
        floor = max(nbytes / (peaks["hbm_gbs"] * 1e9), flops / (peaks["tflops"] * 1e12)) * 1e6
        t_sum += us
        floor_sum += floor
        rows.append({"layer": name, "us": round(us, 1), "us_direct_cuda_cores": round(us_direct, 1),
                     "us_library_cudnn": round(us_lib, 1), "tflops": round(flops / (us * 1e-6) / 1e12, 1),
                     "floor_us": round(floor, 1), "frac_of_floor": round(floor / us, 3),
                     "bound": "hbm" if nbytes / (peaks["hbm_gbs"] * 1e9) > flops / (peaks["tflops"] * 1e12)
                     else "tensor",
                     "flat_octet_loads": bool(r == 1 and st == 1 and pd == 0 and (h * h) % 8 == 0),
                     "rel_l2_fp64": rl2})
        del x, wt, y, wp, xs, ys, y64
    return {"workload": "ResNet-50 layers outside the Winograd contract, N128, x ~ N(0,1), "
                        "weights ~ N(0, 1/(c r s)); drop-in route 4 runs the same kernels",
            "layers": rows, "sum_us": round(t_sum, 1), "sum_floor_us": round(floor_sum, 1),
            "frac_of_floor": round(floor_sum / t_sum, 3)}


def run_only(args):
    """Launch one kernel family `args.steps` times on the workload with batch
    `args.n` (for profiler captures; prints nothing measured)."""
    import numpy as np
    import torch
    import oracle
    wino = importlib.import_module("2024pra_conv_b200")
    dev = torch.device("cuda", 0)
    W = dict(WORKLOAD, n=args.n or WORKLOAD["n"])
    n, c, h, w, k = W["n"], W["c"], W["h"], W["w"], W["k"]
    x16, w16 = oracle.make_inputs(n, c, h, w, k, seed=0, x_dist="relu_normal",
                                  w_std=np.sqrt(2.0 / (9 * c)))
    x = torch.from_numpy(x16).to(dev)
    wt = torch.from_numpy(w16).to(dev)
    if args.only == "fused":
        u = wino.filter_transform(wt)
        for _ in range(args.steps):
            wino.conv2d_fused(x, u, k)
    elif args.only == "unfused":
        u2 = wino.filter_transform_unfused(wt)
        ws = wino.UnfusedWorkspace(n, c, h, w, k, dev)
        for _ in range(args.steps):
            wino.conv2d_unfused(x, u2, k, ws=ws)
    elif args.only == "twostage":
        u2 = wino.filter_transform_unfused(wt)
        ws = wino._aligned_ws(wino.twostage_workspace_bytes(n, c, h, w, k), dev)
        y = torch.empty((n, k, h, w), dtype=torch.float16, device=dev)
        for _ in range(args.steps):
            wino.conv2d_twostage(x, u2, k, out=y, workspace=ws)
    elif args.only == "f4":
        conv = wino.ConvF4(wt, n, h, w, hilo=True)
        for _ in range(args.steps):
            conv(x)
    elif args.only == "igemm":
        # the 1x1 512->128 layer at 28x28 (octet loads) and the stride-2
        # 3x3 128 layer at 56x56 (2-byte gather), batch n
        for (c2, h2, k2, r2, st2, pd2) in ((512, 28, 128, 1, 1, 0), (128, 56, 128, 3, 2, 1)):
            x2 = torch.randn((n, c2, h2, h2), device=dev).half()
            w2 = (torch.randn((k2, c2, r2, r2), device=dev) / (c2 * r2 * r2) ** 0.5).half()
            wp2 = wino.igemm_weight_transform(w2)
            for _ in range(args.steps):
                wino.conv2d_igemm(x2, w2, stride=st2, pad=pd2, wprep=wp2)
    else:
        for _ in range(args.steps):
            wino.dropin_conv2d(x, wt)
    torch.cuda.synchronize()
    code = wino.error_read_clear()
    print(json.dumps({"only": args.only, "n": n, "launches": args.steps, "device_error": code}))
    return 1 if code else 0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--soak", type=float, default=1.0, help="seconds of untimed load before timing")
    ap.add_argument("--no-cpu", action="store_true", help="skip the CPU baseline leg")
    ap.add_argument("--no-extras", action="store_true",
                    help="skip the layer-set / variants / cost-model legs")
    ap.add_argument("--only", choices=["fused", "unfused", "dropin", "f4", "twostage", "igemm"],
                    help="only launch this path (profiler captures)")
    ap.add_argument("--n", type=int, default=0, help="batch size for --only")
    args = ap.parse_args()
    if args.only:
        return run_only(args)
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        return run_reference_arm(args, rank)
    if world > 1:
        import datetime
        import torch
        torch.cuda.set_device(local_rank)
        torch.distributed.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    try:
        return run_ours(args, rank, world, local_rank)
    finally:
        if world > 1:
            import torch
            torch.distributed.destroy_process_group()


if __name__ == "__main__":
    sys.exit(main())
