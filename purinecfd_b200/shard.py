"""Instance sharding over GPUs: independent solves dealt to one process per GPU.

Batched cases and serving requests are independent solves, so a job on N GPUs
splits them into N shares and needs no data-path collective: each rank (one
process per GPU, launched by torchrun) solves its share in its own Batch on
its own device, and one gather of host objects at the end combines the
results.  The plan is a pure function of the instance list, so every rank
computes the same plan without communicating.

Plan: instances are taken in submission order and each goes to the rank with
the least work so far, where an instance's work is its cell count times its
step limit (the HBM footprint and the device time of a solve both grow with
the cell count); ties go to the lowest rank.

The collectives (`Group`) go through torch.distributed on whatever backend the
process group was created with (NCCL between GPUs, gloo in the CPU tests);
without a process group the job is one rank and nothing is communicated.
"""

from __future__ import annotations

import os
from dataclasses import dataclass

import numpy as np


def instance_work(n_rings: int, n_theta: int, max_steps: int) -> float:
    """Work estimate of one solve: cells x step limit."""
    return float((n_rings - 1) * n_theta) * float(max(1, max_steps))


def shard_plan(works: list[float], world: int) -> list[int]:
    """Owner rank of each instance (greedy least-loaded in submission order)."""
    load = [0.0] * max(1, world)
    owner = []
    for w in works:
        r = min(range(len(load)), key=lambda q: (load[q], q))
        owner.append(r)
        load[r] += w
    return owner


class Group:
    """The ranks of a job: torch.distributed when a process group exists,
    else a single rank."""

    def __init__(self):
        self.world, self.rank, self.local_rank = 1, 0, 0
        try:
            import torch.distributed as dist
            if dist.is_available() and dist.is_initialized():
                self.world = dist.get_world_size()
                self.rank = dist.get_rank()
                self.local_rank = int(os.environ.get("LOCAL_RANK", self.rank))
        except ImportError:
            pass

    def gather(self, obj) -> list:
        """Every rank's object, in rank order, on every rank."""
        if self.world == 1:
            return [obj]
        import torch.distributed as dist
        out = [None] * self.world
        dist.all_gather_object(out, obj)
        return out

    def barrier(self):
        if self.world > 1:
            import torch.distributed as dist
            dist.barrier()


def solve_sharded(cases, precision: int, group: Group | None = None, solve_fn=None, **kw):
    """Solve every case (config, xy, n_rings, n_theta) with the cases dealt
    over the ranks; each rank runs `solve_fn` (default serve.batch_solve) on
    its share on its own device.  Returns (results in case order, job wall
    seconds = the slowest rank's, plan) on every rank."""
    from .serve import batch_solve
    g = group or Group()
    solve_fn = solve_fn or batch_solve
    max_steps = kw.get("max_steps", 2000)
    plan = shard_plan([instance_work(c[2], c[3], max_steps) for c in cases], g.world)
    mine = [k for k, r in enumerate(plan) if r == g.rank]
    if mine:
        res, wall = solve_fn([cases[k] for k in mine], precision, device=g.local_rank, **kw)
    else:
        res, wall = [], 0.0
    parts = g.gather((mine, res, wall))
    out = [None] * len(cases)
    for idx, rr, _ in parts:
        for k, r in zip(idx, rr):
            out[k] = r
    return out, max(p[2] for p in parts), plan


@dataclass
class JobServeStats:
    rate: float
    ranks: int
    requests: int
    completed: int
    converged: int
    nonphysical: int
    wall_s: float
    solves_per_s: float
    p50_s: float
    p99_s: float
    mean_steps: float


def serve_sharded(requests, rate: float, seed: int = 0, group: Group | None = None, serve_fn=None, **kw):
    """Serve a Poisson request stream over all ranks.  The arrival times are
    drawn once for the whole stream (the same seed on every rank); each
    request is submitted by its owner at its own arrival time, so a rank sees
    the sub-stream of its requests and latency is measured from the real
    arrival.  Returns (job statistics, [(request index, result, latency)] in
    request order) on every rank."""
    from .serve import percentile, poisson_arrivals, serve
    g = group or Group()
    serve_fn = serve_fn or serve
    arrivals = poisson_arrivals(len(requests), rate, seed)
    plan = shard_plan([instance_work(r.n_rings, r.n_theta, r.max_steps) for r in requests], g.world)
    mine = [k for k, r in enumerate(plan) if r == g.rank]
    g.barrier()  # common start
    if mine:
        st, res = serve_fn([requests[k] for k in mine], rate, arrivals=arrivals[mine], device=g.local_rank, **kw)
        wall = st.wall_s
        local = [(mine[k], r, lat) for k, r, lat in res]
    else:
        wall, local = 0.0, []
    parts = g.gather((wall, local))
    results = sorted((x for _, loc in parts for x in loc), key=lambda x: x[0])
    wall = max(p[0] for p in parts)
    lat = [x[2] for x in results]
    steps = [x[1].steps for x in results]
    st = JobServeStats(rate=rate, ranks=g.world, requests=len(requests), completed=len(results),
                       converged=sum(1 for x in results if x[1].status == 0),
                       nonphysical=sum(1 for x in results if x[1].status == 8), wall_s=wall,
                       solves_per_s=len(results) / wall if wall > 0 else float("nan"),
                       p50_s=percentile(lat, 50), p99_s=percentile(lat, 99),
                       mean_steps=float(np.mean(steps)) if steps else float("nan"))
    return st, results

