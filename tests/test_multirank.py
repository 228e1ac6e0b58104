"""The multi-rank path of bench.py on CPU: two gloo ranks (replicas only) reduce their
timings to the slowest rank and report the whole-job rate; a rank that leaves early
makes the others fail within the process-group timeout instead of hanging."""
import datetime
import os
import socket
import sys

import pytest
import torch.multiprocessing as mp

from conftest import ROOT


def _port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, mode, out):
    import torch
    import torch.distributed as dist

    sys.path.insert(0, ROOT)
    import bench

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=10))
    try:
        if mode == "reduce":
            # per-rank seconds of the timed region and of the e2e region
            mine = [0.5 + 0.25 * rank, 2.0 - rank]
            total_s, e2e_s = bench.max_over_ranks(torch, dist, mine, "cpu")
            out[rank] = (total_s, e2e_s, bench.replica_throughput(world, 10_000 * 100, total_s))
        else:  # "leave": rank 1 exits before the collective, rank 0 must fail, not hang
            if rank == 1:
                out[rank] = "left"
                return
            try:
                bench.max_over_ranks(torch, dist, [1.0], "cpu")
                out[rank] = "no error"
            except Exception as e:  # gloo reports the missing peer
                out[rank] = "error: " + type(e).__name__
    finally:
        if not (mode == "leave" and rank == 1):
            try:
                dist.destroy_process_group()
            except Exception:
                pass


def _run(mode):
    ctx = mp.get_context("spawn")
    out = ctx.Manager().dict()
    port = _port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, mode, out)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=120)
        assert not p.is_alive()
    return dict(out)


def test_two_gloo_ranks_reduce_to_the_slowest():
    out = _run("reduce")
    assert out[0] == out[1]
    total_s, e2e_s, rate = out[0]
    assert total_s == 0.75 and e2e_s == 2.0
    assert rate == pytest.approx(2 * 10_000 * 100 / 0.75)


def test_rank_that_leaves_fails_the_others_within_the_timeout():
    out = _run("leave")
    assert out[1] == "left"
    assert out[0].startswith("error")
