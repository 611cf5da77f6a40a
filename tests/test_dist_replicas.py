"""The N-GPU bench path on CPU: two gloo ranks on 127.0.0.1.

The force path does not shard (one system per GPU), so `bench.py --gpus N`
runs N independent replicas; the only cross-rank operations are the
barrier around each timed region, the max of the timed durations and the
sum of the steps all ranks did.  The reference arm runs on rank 0 alone."""
from __future__ import annotations

import os
import socket
import sys
from pathlib import Path

import pytest
import torch.multiprocessing as mp

ROOT = Path(__file__).resolve().parents[1]


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank: int, world: int, port: int, q):
    os.environ.update(RANK=str(rank), WORLD_SIZE=str(world), LOCAL_RANK=str(rank),
                      MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    sys.path.insert(0, str(ROOT))
    import torch.distributed as dist

    import bench

    ws, r, local = bench.dist_setup()
    try:
        bench.barrier(ws)
        t = bench.max_over_ranks(ws, 10.0 + r)     # this rank's timed milliseconds
        steps = bench.sum_over_ranks(ws, 5)        # each replica did 5 steps
        # --impl reference: rank 0 runs and prints, the others return at once
        args = type("A", (), {"n": 64, "warmup": 0, "steps": 1, "gpus": ws})()
        if r != 0:
            bench.run_reference(args, ws, r)
        q.put((r, ws, t, steps))
    finally:
        dist.destroy_process_group()


def test_two_replicas_reduce_time_and_steps():
    world, port = 2, _free_port()
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_rank, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=120)
    assert all(p.exitcode == 0 for p in procs), [p.exitcode for p in procs]
    got = sorted(q.get(timeout=10) for _ in range(world))
    for r, (rank, ws, t, steps) in enumerate(got):
        assert rank == r and ws == world
        assert t == pytest.approx(11.0)   # max over ranks of 10 + rank
        assert steps == pytest.approx(10.0)
