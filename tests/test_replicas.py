"""Replica plumbing of bench.py on CPU: two gloo ranks, as torchrun would
start them (127.0.0.1 rendezvous).  The box does not shard (one box per GPU,
no exchange), so the only collectives are the barrier and the max over ranks
of the timed region; the reference arm runs on rank 0 alone."""
import importlib.util
import os
import socket

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _bench():
    spec = importlib.util.spec_from_file_location("bench", os.path.join(ROOT, "bench.py"))
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, times, out):
    import datetime
    import torch.distributed as dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    b = _bench()
    dist.barrier()
    ms = b.reduce_max_ms(times[rank], dist, "cpu")
    out.put((rank, ms, b.aggregate_rate(world, 64, ms)))
    dist.barrier()
    dist.destroy_process_group()


def test_max_over_ranks_with_gloo():
    import torch.multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    times = [12.5, 17.0]
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, times, q)) for r in range(2)]
    for p in procs:
        p.start()
    got = sorted(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    # every rank sees the slowest replica's time; the job rate counts both boxes
    assert [g[1] for g in got] == [17.0, 17.0]
    assert got[0][2] == pytest.approx(2 * 64 ** 3 / 17.0e-3 / 1e9)


def test_single_process_needs_no_collective():
    b = _bench()
    assert b.reduce_max_ms(3.25, None, "cpu") == 3.25
    assert b.aggregate_rate(1, 1024, 100.0) == pytest.approx(1024 ** 3 / 0.1 / 1e9)


def test_reference_arm_runs_on_rank_zero_only(monkeypatch):
    b = _bench()
    monkeypatch.setenv("RANK", "1")
    import argparse
    ns = argparse.Namespace(cpu_n=256, steps=1, warmup=0, gpus=2, n=1024)
    # a non-zero rank returns at once, before touching the oracle
    assert b.run_reference(ns) == 0
