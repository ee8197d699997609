"""Instance sharding over ranks (purinecfd_b200.shard) on CPU: two gloo ranks
run the real dispatcher — plan, local share, gather, combine — with the
per-GPU solver replaced by a stand-in that records what it was given, so no
GPU is needed.  Checks that every instance is solved exactly once, by the
rank the plan names, and that results come back in submission order with
the job figures combined over both ranks."""

from __future__ import annotations

import os
import socket
import sys
from dataclasses import dataclass

import numpy as np
import torch.multiprocessing as mp

from conftest import ROOT


@dataclass
class FakeResult:
    k: int
    steps: int
    status: int


@dataclass
class FakeStats:
    wall_s: float


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _sizes():
    """(n_rings, n_theta) of the instances: mixed sizes, in submission order."""
    return [(17, 40), (65, 128), (129, 256), (33, 64), (257, 512), (17, 40), (65, 128), (129, 256), (41, 96)]


def _rank(rank: int, world: int, port: int, q):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), WORLD_SIZE=str(world), RANK=str(rank),
                      LOCAL_RANK=str(rank))
    sys.path.insert(0, str(ROOT))
    from datetime import timedelta

    import torch.distributed as dist
    from purinecfd_b200 import shard
    from purinecfd_b200.serve import Request
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=timedelta(seconds=60))
    g = shard.Group()
    cases = [({"k": k}, None, nr, nt) for k, (nr, nt) in enumerate(_sizes())]
    solved = []

    def fake_solve(sub, precision, device=0, **kw):
        assert device == rank
        solved.extend(c[0]["k"] for c in sub)
        return [FakeResult(c[0]["k"], c[2], 10) for c in sub], 1.0 + rank

    out, wall, plan = shard.solve_sharded(cases, 0, group=g, solve_fn=fake_solve, max_steps=100)

    reqs = [Request({"k": k}, np.zeros((nr * nt, 2)), nr, nt, 200) for k, (nr, nt) in enumerate(_sizes())]
    served = []

    def fake_serve(sub, rate, arrivals=None, device=0, **kw):
        assert device == rank and len(arrivals) == len(sub)
        assert all(np.diff(arrivals) >= 0)
        served.extend(r.config["k"] for r in sub)
        res = [(i, FakeResult(r.config["k"], r.n_rings, 0 if r.n_rings < 100 else 8), 0.1 * (i + 1))
               for i, r in enumerate(sub)]
        return FakeStats(2.0 + rank), res

    st, results = shard.serve_sharded(reqs, 50.0, seed=3, group=g, serve_fn=fake_serve)
    q.put((rank, solved, [r.k for r in out], wall, plan, served, st, [(i, r.k) for i, r, _ in results]))
    dist.destroy_process_group()


def test_plan_balances_work_and_is_deterministic():
    from purinecfd_b200.shard import instance_work, shard_plan
    works = [instance_work(nr, nt, 100) for nr, nt in _sizes()]
    for world in (1, 2, 3, 4):
        plan = shard_plan(works, world)
        assert plan == shard_plan(works, world) and len(plan) == len(works)
        loads = [sum(w for w, r in zip(works, plan) if r == q) for q in range(world)]
        assert max(loads) - min(loads) <= max(works)


def test_two_ranks_solve_and_serve_every_instance_once():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    ps = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in ps:
        p.start()
    out = sorted((q.get(timeout=120) for _ in ps), key=lambda x: x[0])
    for p in ps:
        p.join(timeout=60)
        assert p.exitcode == 0
    n = len(_sizes())
    (_, solved0, order0, wall0, plan0, served0, st0, res0), (_, solved1, order1, wall1, plan1, served1, st1, res1) = out
    # the same plan on both ranks; each instance solved once, by its owner
    assert plan0 == plan1
    assert sorted(solved0 + solved1) == list(range(n)) and not set(solved0) & set(solved1)
    assert all(plan0[k] == 0 for k in solved0) and all(plan0[k] == 1 for k in solved1)
    assert sorted(served0 + served1) == list(range(n)) and not set(served0) & set(served1)
    # results gathered on every rank, in submission order; job wall = slowest rank
    assert order0 == order1 == list(range(n))
    assert wall0 == wall1 == 2.0
    assert [k for _, k in res0] == [k for _, k in res1] == list(range(n))
    assert [i for i, _ in res0] == list(range(n))
    assert st0 == st1
    assert st0.completed == n and st0.ranks == 2 and st0.wall_s == 3.0
    assert st0.nonphysical == sum(1 for nr, _ in _sizes() if nr >= 100)
    assert abs(st0.solves_per_s - n / 3.0) < 1e-12
