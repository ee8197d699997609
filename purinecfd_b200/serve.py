"""Continuous-batching solve server over the batched solver.

Requests (a config, an O-mesh and stopping rules) arrive as a Poisson stream;
the server submits each request as it arrives, the batch admits it as soon
as a slot and HBM are free (its state stays device-resident until it
retires), every instance advances in the shared persistent kernel, and
finished instances retire individually while others keep running.  Reported:
solves/s and latency percentiles (arrival -> retirement).
"""

from __future__ import annotations

import math
import time
from dataclasses import dataclass, field

import numpy as np

from . import meshgen, workloads
from .batch import Batch
from .solver import DT_LOCAL, PREC_FP32_SPLIT


@dataclass
class Request:
    config: dict
    xy: np.ndarray
    n_rings: int
    n_theta: int
    max_steps: int
    residual_drop: float = 1e-6
    cl_tol: float = 1e-5
    meta: dict = field(default_factory=dict)


def request_stream(seed: int, n: int, cylinder_fraction: float = 0.2, max_steps: int = 2000) -> list[Request]:
    """Requests drawn like the batch benchmark (NACA 4-digit sections on three
    mesh classes, M, alpha, Re ranges) plus circular-cylinder O-meshes of
    40x17 to 513x129 nodes; instance k uses PCG64(seed, stream k)."""
    out = []
    for k in range(n):
        rng = np.random.Generator(np.random.PCG64([seed, 10_000 + k]))
        if rng.uniform() < cylinder_fraction:
            nt = int(rng.integers(40, 514))
            nr = int(rng.integers(17, 130))
            mach = rng.uniform(0.2, 0.5)
            re = 10.0 ** rng.uniform(4.0, 5.0)
            cfg = workloads.flow_config(mach, 0.0, re, cfl=1.0, nut_ratio=3.0)
            xy = meshgen.cylinder_o_mesh(nr, nt, radius=0.5, r_far=20.0, first_spacing=1e-3)
            out.append(Request(cfg, xy, nr, nt, max_steps, meta={"kind": "cylinder", "mach": mach, "re": re}))
        else:
            cfg, xy, nr, nt, meta = workloads.batch_instance(seed, k)
            cfg["simulation"]["CFL"] = 1.0
            out.append(Request(cfg, xy, nr, nt, max_steps, meta=dict(meta, kind="naca")))
    return out


@dataclass
class ServeStats:
    rate: float
    requests: int
    completed: int
    converged: int
    nonphysical: int
    wall_s: float
    solves_per_s: float
    p50_s: float
    p99_s: float
    mean_steps: float


def poisson_arrivals(n: int, rate: float, seed: int = 0) -> np.ndarray:
    """Arrival offsets (seconds, the first at 0) of n requests of a Poisson
    stream at `rate` requests/s."""
    rng = np.random.default_rng(seed)
    gaps = rng.exponential(1.0 / rate, size=n)
    return np.cumsum(gaps) - gaps[0] if n else gaps


def serve(requests: list[Request], rate: float, seed: int = 0, precision: int = PREC_FP32_SPLIT,
          hbm_budget_gb: float = 150.0, max_instances: int = 512, steps_per_poll: int = 25,
          chunk: int = 25, arrivals: np.ndarray | None = None, device: int = 0) -> tuple[ServeStats, list]:
    """Run the request list with Poisson arrivals at `rate` requests/s (real
    time), or at the given arrival offsets (seconds from the start).  Returns
    (statistics, [(request index, result, latency)] in completion order)."""
    if arrivals is None:
        arrivals = poisson_arrivals(len(requests), rate, seed)
    arrivals = np.asarray(arrivals, dtype=float)
    b = Batch(precision=precision, dt_mode=DT_LOCAL, steps_per_poll=steps_per_poll, hbm_budget_gb=hbm_budget_gb,
              max_instances=max_instances, device=device)
    t0 = time.perf_counter()
    arrival_of = {}
    nxt = 0
    results = []
    while len(results) < len(requests):
        now = time.perf_counter() - t0
        while nxt < len(requests) and arrivals[nxt] <= now:
            r = requests[nxt]
            ident = b.submit(r.config, r.xy, r.n_rings, r.n_theta, r.max_steps, r.residual_drop, r.cl_tol)
            arrival_of[ident] = (t0 + arrivals[nxt], nxt)
            nxt += 1
        active, queued, _ = b.stats()
        if active + queued > 0:
            b.step(chunk)
        elif nxt < len(requests):
            time.sleep(max(0.0, min(0.05, arrivals[nxt] - (time.perf_counter() - t0))))
        done_at = time.perf_counter()
        for ident in b.poll():
            res = b.result(ident)
            t_arr, k = arrival_of[ident]
            results.append((k, res, done_at - t_arr))
    wall = time.perf_counter() - t0
    b.close()
    lat = np.array([x[2] for x in results])
    conv = sum(1 for x in results if x[1].status == 0)
    bad = sum(1 for x in results if x[1].status == 8)
    st = ServeStats(rate, len(requests), len(results), conv, bad, wall, len(results) / wall,
                    float(np.percentile(lat, 50)), float(np.percentile(lat, 99)),
                    float(np.mean([x[1].steps for x in results])))
    return st, results


def batch_solve(cases, precision: int, max_instances: int = 256, max_steps: int = 2000, residual_drop: float = 1e-6,
                cl_tol: float = 0.0, hbm_budget_gb: float = 40.0, steps_per_poll: int = 25, info: dict | None = None,
                device: int = 0):
    """Solve every case (config, xy, n_rings, n_theta) in one batch; returns
    (results in case order, wall seconds).  `info`, when given, receives the
    stage kernel configuration the batch ran with."""
    b = Batch(precision=precision, dt_mode=DT_LOCAL, steps_per_poll=steps_per_poll, hbm_budget_gb=hbm_budget_gb,
              max_instances=max_instances, device=device)
    t0 = time.perf_counter()
    ids = [b.submit(c[0], c[1], c[2], c[3], max_steps, residual_drop, cl_tol) for c in cases]
    res = {r.id: r for r in b.run_all(chunk=max(steps_per_poll, 100))}
    wall = time.perf_counter() - t0
    if info is not None:
        info["kernel"] = "x".join(map(str, b.kernel_config()))
    b.close()
    return [res[i] for i in ids], wall


def solve_alone(case, precision: int, max_steps: int = 2000, residual_drop: float = 1e-6, cl_tol: float = 0.0,
                poll: int = 50, device: int = 0):
    """One solve on its own (the plain one-at-a-time path: a Solver with its
    autotuned stage kernel and a CUDA graph per RK step, local time steps)
    under the batch's stopping rules, checked every `poll` steps: residual
    below residual_drop times the first step's residual, |CL(n) - CL(n-100)|
    below cl_tol (CL sampled every `poll` steps), or the step limit.  Returns
    a BatchResult (status JST_OK converged, JST_ERR_NONPHYSICAL, or
    JST_ERR_TIMEOUT at the limit)."""
    from .batch import BatchResult
    from .solver import NonPhysical, Solver
    cfg, xy, nr, nt = case
    t0 = time.perf_counter()
    s = Solver(cfg, xy, nr, nt, precision=precision, dt_mode=DT_LOCAL, device=device)
    status, steps, first, res = 10, 0, float("nan"), float("nan")
    cl_hist = []
    cl = cd = float("nan")
    try:
        s.run(1)
        steps, first = 1, s.residual()
        res = first
        while steps < max_steps:
            n = min(poll - steps % poll, max_steps - steps)
            rep = s.run(n)
            steps += rep.steps
            res = rep.residual
            if residual_drop > 0 and res < residual_drop * first:
                status = 0
                break
            if cl_tol > 0 and steps % poll == 0:
                cl_hist.append((steps, s.forces()[0]))
                old = [c for k, c in cl_hist if steps - k >= 100]
                if old and abs(cl_hist[-1][1] - old[-1]) < cl_tol:
                    status = 0
                    break
        cl, cd = s.forces()
    except NonPhysical:
        status = 8
    ni, nj = s.ni, s.nj
    s.close()
    t1 = time.perf_counter()
    return BatchResult(-1, status, steps, res, first, float("nan"), cl, cd, 0.0, 0.0, t1 - t0, ni, nj)


def percentile(xs, q):
    xs = [x for x in xs if math.isfinite(x)]
    return float(np.percentile(xs, q)) if xs else float("nan")
