"""The multi-rank plumbing of bench.py on CPU: two gloo ranks (the path runs
replicas only -- no data-path collective), max-over-ranks timing and the
rank-0-only report."""
import os
import socket

import pytest
import torch.multiprocessing as mp

from conftest import ROOT


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, out):
    import sys

    sys.path.insert(0, ROOT)
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank),
                      WORLD_SIZE=str(world), LOCAL_RANK=str(rank))
    import torch

    torch.cuda.is_available = lambda: False  # force the CPU (gloo) backend
    import bench

    r, w, local = bench.dist_setup()
    try:
        bench.barrier(w)
        t = bench.max_over_ranks(10.0 + r, w)
        s = bench.sum_over_ranks(1.0, w)
        out.put((r, t, s))
    finally:
        bench.dist_teardown(w)


def test_two_rank_timing_reduction():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = sorted(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert [r for r, _, _ in res] == [0, 1]
    assert all(t == 11.0 for _, t, _ in res)  # max over ranks
    assert all(s == 2.0 for _, _, s in res)


def test_single_rank_is_identity():
    import bench

    assert bench.max_over_ranks(3.5, 1) == 3.5 and bench.sum_over_ranks(2.0, 1) == 2.0


def test_workload_name():
    import bench

    assert bench.workload_name(1 << 20).startswith("plummer N=2^20")
    assert "4097" in bench.workload_name(4097)
