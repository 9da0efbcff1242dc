"""Multi-GPU is replicas only: the whole-job time is the max over ranks of
independent replicas.  The reduction runs here on CPU with two gloo ranks;
the reference arm's extra ranks exit without work."""
import importlib.util
import os
import socket

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _bench():
    spec = importlib.util.spec_from_file_location("bench_mod", os.path.join(ROOT, "bench.py"))
    m = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(m)
    return m


def _worker(rank, world, port, q):
    import datetime
    import torch
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    torch.distributed.init_process_group("gloo", rank=rank, world_size=world,
                                         timeout=datetime.timedelta(seconds=60))
    try:
        b = _bench()
        local_ms = [3.0, 5.0][rank]
        q.put((rank, b.replica_throughput(local_ms, 2e12, world, "cpu")))
    finally:
        torch.distributed.destroy_process_group()


def test_replica_throughput_two_gloo_ranks():
    import torch.multiprocessing as mp
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    out = dict(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    for r in (0, 1):
        max_ms, tflops = out[r]
        assert max_ms == 5.0                                # the slowest replica
        assert tflops == pytest.approx(2 * 2e12 / 5e-3 / 1e12)


def test_single_rank_and_reference_arm_extra_ranks():
    b = _bench()
    assert b.replica_throughput(4.0, 1e12, 1, "cpu") == (4.0, pytest.approx(250.0))

    class A:
        steps, warmup, gpus = 1, 0, 2
    assert b.run_reference_arm(A(), 1) == 0                # rank 1: no work, exit 0
