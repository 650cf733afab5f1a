"""CPU, world size 2 over gloo: the multi-GPU plumbing of bench.py.

Shots are independent, so N GPUs run N shot batches with no data-path collective (weak
scaling); the only collectives are the barrier and the max over ranks of each timing.
These tests run that host logic on two gloo ranks: each rank's batch, the max-over-ranks
reduction, the aggregate, and that the reference arm lets only rank 0 work."""
import os
import socket
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, q):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world),
                      LOCAL_RANK=str(rank))
    sys.path.insert(0, ROOT)
    from datetime import timedelta

    import numpy as np
    import torch.distributed as dist

    import bench

    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=timedelta(seconds=60))
    try:
        r, w, local = bench.rank_info()
        sv = bench.workload(r, shots=8)
        ms = 10.0 + 5.0 * r  # this rank's step time
        ms_max = bench.max_over_ranks(ms, dist, "cpu")
        value = w * len(sv.shots) / (ms_max / 1000.0)
        dist.barrier()
        q.put((r, w, local, float(np.asarray(sv.shots).sum()), ms_max, value))
    finally:
        dist.destroy_process_group()


@pytest.mark.timeout(300)
def test_two_gloo_ranks_shard_and_take_the_max():
    import torch.multiprocessing as mp

    world, port = 2, _free_port()
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_rank_main, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(240)
    assert all(p.exitcode == 0 for p in procs), [p.exitcode for p in procs]
    res = sorted(q.get(timeout=10) for _ in range(world))
    assert [r[0] for r in res] == [0, 1] and all(r[1] == 2 for r in res)
    # each rank solves its own batch (different seeded shots), no data exchange
    assert res[0][3] != res[1][3]
    # every rank sees the slowest rank's time; the aggregate counts both batches
    assert all(abs(r[4] - 15.0) < 1e-12 for r in res)
    assert all(abs(r[5] - 2 * 8 / 0.015) < 1e-6 for r in res)


def test_reference_arm_runs_on_rank_zero_only(monkeypatch):
    sys.path.insert(0, ROOT)
    import bench

    monkeypatch.setenv("RANK", "1")
    monkeypatch.setenv("WORLD_SIZE", "2")
    args = type("A", (), dict(gpus=2, steps=1, warmup=0))()
    assert bench.run_reference(args) == 0  # returns at once, no work, no output


def test_max_over_ranks_without_process_group():
    sys.path.insert(0, ROOT)
    import bench

    assert bench.max_over_ranks(3.5, None, "cpu") == 3.5
