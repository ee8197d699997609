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
    from purinecfd_b200.shard import Group
    w, r, _ = bench.dist_setup("gloo")
    bench.barrier(w)
    ms = 100.0 + 25.0 * r  # rank 1 is the slow one
    m = bench.max_over_ranks(ms, w)
    bench.barrier(w)
    parts = Group().gather({"rank": r})
    q.put((r, w, m, bench.replica_value(1000, 10, m, w), parts))
    dist.destroy_process_group()


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
        assert parts == [{"rank": 0}, {"rank": 1}]  # every rank sees every part, in rank order


def test_single_rank_needs_no_process_group():
    sys.path.insert(0, str(ROOT))
    import bench
    assert bench.max_over_ranks(3.5, 1) == 3.5
    bench.barrier(1)
    assert bench.replica_value(100, 2, 1.0, 1) == pytest.approx(100 * 5 * 2 / 1e-3 / 1e6)


def test_stratified_sample_keeps_the_class_mix():
    sys.path.insert(0, str(ROOT))
    import bench
    classes = ["a"] * 80 + ["b"] * 90 + ["c"] * 86
    idx = bench.stratified_sample(classes, 24)
    counts = {c: sum(1 for k in idx if classes[k] == c) for c in "abc"}
    assert counts == {"a": 8, "b": 8, "c": 8}
    assert idx == sorted(idx) and len(set(idx)) == len(idx)
    assert bench.stratified_sample(["x"] * 3 + ["y"], 2) == [0, 1, 3]


def test_thread_sweep_counts():
    sys.path.insert(0, str(ROOT))
    import bench
    assert bench.thread_counts(16) == [1, 2, 4, 8, 16]
    assert bench.thread_counts(12) == [1, 2, 4, 8, 12]
    assert bench.thread_counts(1) == [1]
