"""Multi-rank plumbing of bench.py on CPU (gloo, world size 2): the solves
are independent replicas, so the only collectives are the timing barrier and
the max over ranks of the device time; the job value counts every rank's
cells over the slowest rank's time."""

from __future__ import annotations

import os
import socket
import sys

import pytest
import torch.multiprocessing as mp

from conftest import ROOT


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank: int, world: int, port: int, q):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), WORLD_SIZE=str(world), RANK=str(rank),
                      LOCAL_RANK=str(rank))
    sys.path.insert(0, str(ROOT))
    import bench
    import torch.distributed as dist
    w, r, _ = bench.dist_setup("gloo")
    bench.barrier(w)
    ms = 100.0 + 25.0 * r  # rank 1 is the slow one
    m = bench.max_over_ranks(ms, w)
    bench.barrier(w)
    parts = bench.gather_objects(_part(r), w)
    q.put((r, w, m, bench.replica_value(1000, 10, m, w), parts))
    dist.destroy_process_group()


def _part(rank: int) -> dict:
    """A batch-leg part as one rank reports it (instances k = rank, rank + 2, ...)."""
    return {"instances": 3 - rank, "cells": 1000 * (3 - rank), "wall_split": 2.0 + rank, "wall_ref": 5.0 - rank,
            "plain_m": 2 if rank == 0 else 0, "plain_wall": 4.0 if rank == 0 else 0.0,
            "cell_steps": 10_000 * (3 - rank), "steps": 30 - 10 * rank, "converged": 1, "nonphysical": rank,
            "within": 3 - 2 * rank, "dcl_max": 1e-6 * (rank + 1), "dcd_max": None if rank else 2e-7,
            "latencies": [1.0 + rank, 2.0 + rank]}


def test_two_rank_barrier_and_max_over_ranks():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    ps = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in ps:
        p.start()
    out = sorted(q.get(timeout=120) for _ in ps)
    for p in ps:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert [o[0] for o in out] == [0, 1]
    for r, w, m, v, parts in out:
        assert w == 2 and m == 125.0
        assert v == pytest.approx(2 * 1000 * 5 * 10 / 0.125 / 1e6)
        assert parts == [_part(0), _part(1)]  # every rank sees every part, in rank order


def test_batch_parts_combine_to_job_figures():
    """5 instances dealt over 2 ranks: the job takes the slowest rank's wall
    time, counts add, errors take the maximum, and the plain one-at-a-time
    rate measured on rank 0 counts once per GPU."""
    sys.path.insert(0, str(ROOT))
    import bench
    b = bench.combine_batch_parts([_part(0), _part(1)], 1000)
    assert b["instances"] == 5 and b["ranks"] == 2 and b["cells"] == 5000
    assert b["wall_s"] == 3.0 and b["solves_per_s"] == pytest.approx(5 / 3.0, abs=1e-3)
    assert b["fp64_batch_solves_per_s"] == pytest.approx(1.0)
    assert b["mcell_stage_per_s"] == pytest.approx(50_000 * 5 / 3.0 / 1e6, abs=0.1)
    assert b["converged"] == 2 and b["nonphysical"] == 1 and b["mean_steps"] == pytest.approx(10.0)
    assert b["cl_err_max"] == pytest.approx(2e-6) and b["cd_err_max"] == pytest.approx(2e-7)
    assert b["within_1e-4"] == "4/5"
    plain = b["plain_fp64_one_at_a_time"]
    assert plain["solves_per_s_per_gpu"] == pytest.approx(0.5) and plain["solves_per_s_job"] == pytest.approx(1.0)
    assert b["speedup_vs_plain"] == pytest.approx((5 / 3.0) / 1.0, abs=0.01)
    assert b["p50_s"] == pytest.approx(2.0) and b["p99_s"] <= 3.0


def test_single_rank_needs_no_process_group():
    sys.path.insert(0, str(ROOT))
    import bench
    assert bench.max_over_ranks(3.5, 1) == 3.5
    bench.barrier(1)
    assert bench.replica_value(100, 2, 1.0, 1) == pytest.approx(100 * 5 * 2 / 1e-3 / 1e6)


def test_serve_parts_combine_to_job_figures():
    """Two ranks serving 3 + 2 requests: counts add, the slowest rank's wall
    time is the job's, percentiles run over every request."""
    sys.path.insert(0, str(ROOT))
    import bench
    parts = [{"rate": 50.0, "requests": 3, "completed": 3, "converged": 1, "nonphysical": 0, "wall_s": 2.0,
              "latencies": [0.1, 0.2, 0.3], "steps": [100, 200, 300]},
             {"rate": 50.0, "requests": 2, "completed": 2, "converged": 2, "nonphysical": 1, "wall_s": 2.5,
              "latencies": [0.4, 0.5], "steps": [400, 500]}]
    j = bench.combine_serve_parts(parts)
    assert j["ranks"] == 2 and j["requests"] == 5 and j["completed"] == 5
    assert j["converged"] == 3 and j["nonphysical"] == 1
    assert j["wall_s"] == 2.5 and j["solves_per_s"] == pytest.approx(2.0)
    assert j["p50_s"] == pytest.approx(0.3) and 0.45 < j["p99_s"] <= 0.5
    assert j["mean_steps"] == pytest.approx(300.0)
