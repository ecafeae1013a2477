"""The multi-rank plumbing of bench.py on the CPU (gloo, two ranks over
127.0.0.1): the bench runs one independent solve per GPU (replicas, no
collective on the data path), times them together and reports the slowest
rank; the reference arm runs on rank 0 only."""
import os
import socket
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, out):
    import torch.distributed as dist

    sys.path.insert(0, ROOT)
    import bench

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        # each replica took its own time; every rank gets the slowest one
        got = bench.max_over_ranks(10.0 + 5.0 * rank, dist, "cpu")
        out.put((rank, got))
    finally:
        dist.destroy_process_group()


def test_max_over_ranks_with_two_gloo_ranks():
    import torch.multiprocessing as mp

    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=120)
    assert all(p.exitcode == 0 for p in procs)
    res = dict(q.get(timeout=5) for _ in range(2))
    assert res == {0: 15.0, 1: 15.0}


def test_single_rank_is_the_identity():
    sys.path.insert(0, ROOT)
    import bench

    assert bench.max_over_ranks(3.25, None, "cpu") == 3.25


def test_reference_arm_runs_on_rank_zero_only(capsys):
    sys.path.insert(0, ROOT)
    import argparse

    import bench

    args = argparse.Namespace(size=8, steps=1, warmup=0, gpus=2)
    bench.run_reference_arm(args, 1, 2)  # another rank: no work, no line
    assert capsys.readouterr().out == ""
