#!/usr/bin/env python3
"""Benchmark of the explicit RANS residual / RK loop on B200.

Workload (default): NACA0012 O-mesh, 4097 x 1025 nodes with a closed ring
(4096 x 1024 = 4,194,304 cells), far field 30c, wall spacing 1e-6c, M 0.8,
alpha 1.25 deg, Re 1e7, FP32 fluxes with the FP64 state accumulator, fused
tiled stage kernels.  A step is one 5-stage RK step over the whole mesh;
throughput is Mcell-stage/s = cells * 5 * steps / seconds.  The mesh is
generated here (synthetic, seeded by construction); state + geometry
(~0.7 GB) exceed the 126 MB L2, so no flush is needed between steps.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

`--impl reference` times the CPU restatement of the reference's jst-rs loop
(oracle/libjst_oracle.so, FP64, OpenMP rows with all host threads) on the
same workload, a bounded number of steps.  Under torchrun (N > 1) every rank
solves its own independent instance (replicas, no data-path collective);
time is the max over ranks.
"""

from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

METRIC = "solves/s & p99 at CL/CD err<=1e-4, batched FP32 vs plain FP64; Mcell-stage/s"
UNIT = "Mcell-stage/s"

# Algorithmic (compulsory) HBM bytes per cell per stage of the stage kernels
# (U_n FP64 40 B; stage state and V/dt in the stage type T).
# Marching kernel (the autotuner's choice on large meshes): geometry is one
# record of 8 T per cell (tau and n normals, 1/V, 1/d^2, V, pad) plus the
# FP64 1/V of the updated cell (8 B).  In split precision stages 1-4 take
# their accumulator from the FP32 copy of U_n (stage 1 already reads it as
# its input); stage 5 adds to U_n in FP64:
#   split: stage 1: U_n copy 20 + write 20 + record 32 + 1/V 8 + ratio 4           = 84
#          stages 2-4: U 20 + U_n copy 20 + write 20 + record 32 + 1/V 8 + ratio 4 = 104
#          stage 5: U 20 + U_n 40 + write U_n 40 + FP32 copy 20 + record 32 + 1/V 8
#                   + V 4 + ratio 4+4                                               = 172
#          average 113.6 B
#   FP64:  stage 1: U_n 40 + write 40 + record 64 + 1/V 8 + ratio 8                 = 160
#          stages 2-4: U 40 + U_n 40 + write 40 + record 64 + 1/V 8 + ratio 8       = 200
#          stage 5: U 40 + U_n 40 + write U_n 40 + record 64 + 1/V 8 + V 8
#                   + ratio 8+8                                                     = 216
#          average 195.2 B
# Tile kernel: geometry = tau and n normals 32 B, V 8, 1/V 8, 1/d^2 8 = 56 B (FP64):
#   split: stages 1-4: U 20 + U_n 40 + write 20 + geom 56 + ratio 4  = 140;  stage 5: 184;  average 148.8 B
#   FP64:  stage 1: 144;  stages 2-4: 184;  stage 5: 192;  average 177.6 B
# Paired-column marching kernel (split only, strips 56 wide): the same bytes,
# except that the last stage takes V from the geometry record two rows back
# instead of reading it again:
#   split: 84, 104, 104, 104, last stage 172 - 4 = 168;  average 112.8 B
BYTES_PER_STAGE = {("march", "split"): [84, 104, 104, 104, 172], ("march", "fp64"): [160, 200, 200, 200, 216],
                   ("march2", "split"): [84, 104, 104, 104, 168],
                   ("tile", "split"): [140, 140, 140, 140, 184], ("tile", "fp64"): [144, 184, 184, 184, 192]}
# kernels of a single solve (the marching strips take the instance by value)
KERNEL_NAMES = {"march": "k_march_solo", "march2": "k_march2", "tile": "k_stage"}


def kernel_kind(kcfg) -> str:
    """(tile_i, tile_j, threads) -> which stage kernel runs (strips are 26
    wide, paired-column strips 56)."""
    return {26: "march", 56: "march2"}.get(kcfg[1], "tile")


def bytes_per_cell_stage(kind: str, prec: str) -> float:
    return sum(BYTES_PER_STAGE[(kind, prec)]) / 5.0


def measured_peaks():
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        d = json.loads(p.read_text())
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def ncu_traffic(kind: str, prec: str):
    """DRAM bytes per cell-stage of the stage kernel from the committed ncu
    summary (profiles/<kind>_kernel_*.md, line `traffic_bytes_per_cell_stage <prec> <value>`)."""
    for f in sorted((ROOT / "profiles").glob(f"{kind}_kernel_*.md")):
        for line in f.read_text().splitlines():
            parts = line.strip().strip("`").split()
            if len(parts) == 3 and parts[0] == "traffic_bytes_per_cell_stage" and parts[1] == prec:
                try:
                    return float(parts[2])
                except ValueError:
                    pass
    return None


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled during the timed region."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device: int):
        self.device = device
        self.proc = None
        self.lines = []

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.device}", f"--query-gpu={self.Q}",
                                          "--format=csv,noheader,nounits", "-lms", "100"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
            time.sleep(0.3)
        except (FileNotFoundError, OSError):
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *a):
        if self.proc:
            time.sleep(0.25)
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        sm, mx, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            f = [x.strip() for x in ln.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                mx.append(float(f[2]))
            except ValueError:
                continue
            for k, n in enumerate(names):
                if f[5 + k].lower().startswith("active"):
                    reasons.add(n)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": [], "samples": 0}
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": max(mx), "reasons": sorted(reasons),
                "samples": len(sm)}


def dist_setup(backend: str | None = None):
    """One process per GPU under torchrun: NCCL when CUDA is present (gloo
    otherwise, for the host-side tests).  The solves are independent replicas,
    so the only collectives are the timing barrier and the max over ranks."""
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import torch
        import torch.distributed as dist
        from datetime import timedelta
        if backend is None:
            backend = "nccl" if torch.cuda.is_available() else "gloo"
        if backend == "nccl":
            torch.cuda.set_device(local)
        dist.init_process_group(backend, timeout=timedelta(seconds=300))
    return world, rank, local


def _coll_device():
    import torch.distributed as dist
    return "cuda" if dist.get_backend() == "nccl" else "cpu"


def barrier(world):
    if world > 1:
        import torch
        import torch.distributed as dist
        dev = _coll_device()
        t = torch.zeros(1, device=dev)
        dist.all_reduce(t)
        if dev == "cuda":
            torch.cuda.synchronize()


def max_over_ranks(x: float, world: int) -> float:
    if world == 1:
        return x
    import torch
    import torch.distributed as dist
    t = torch.tensor([x], dtype=torch.float64, device=_coll_device())
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def replica_value(cells: int, steps: int, ms_max: float, world: int) -> float:
    """Whole-job Mcell-stage/s: every rank advances its own copy of the
    workload, the job takes as long as the slowest rank."""
    return world * cells * 5 * steps / (ms_max / 1e3) / 1e6


def cpu_model() -> str:
    try:
        for line in Path("/proc/cpuinfo").read_text().splitlines():
            if line.lower().startswith("model name"):
                return line.split(":", 1)[1].strip()
    except OSError:
        pass
    return "unknown"


def thread_counts(nproc: int) -> list[int]:
    """1, 2, 4, ... up to nproc, and nproc itself (the sweep of bin/jst.rs:43-48)."""
    out, t = [], 1
    while t < nproc:
        out.append(t)
        t *= 2
    return out + [nproc]


def cpu_reference(workload: str, timed_steps: int, warm_steps: int, sweep: list[int] | None = None):
    """Oracle (CPU restatement of jst-rs, FP64) on the host cores.  With a
    sweep, one RK step is timed at each thread count and the timed steps run
    at the fastest one; the result reports every point."""
    sys.path.insert(0, str(ROOT / "oracle"))
    import jst_oracle as jo
    from purinecfd_b200 import workloads
    cfg, xy, nr, nt = workloads.WORKLOADS[workload]()
    nproc = os.cpu_count() or 1
    jo.set_threads(nproc)
    t0 = time.perf_counter()
    o = jo.OracleSolver(cfg, xy, nr, nt)
    t_setup = time.perf_counter() - t0
    cells = o.n_cells
    if warm_steps:
        o.run(warm_steps)
    points = {}
    best = nproc
    if sweep:
        for t in sweep:
            jo.set_threads(t)
            t0 = time.perf_counter()
            o.run(1)
            points[t] = cells * 5 / (time.perf_counter() - t0) / 1e6
        best = max(points, key=points.get)
    jo.set_threads(best)
    t0 = time.perf_counter()
    o.run(timed_steps)
    dt = time.perf_counter() - t0
    o.close()
    return {"value": cells * 5 * timed_steps / dt / 1e6, "cores": best, "nproc": nproc, "seconds": dt,
            "setup_s": t_setup, "steps": timed_steps, "cells": cells, "cpu": cpu_model(),
            "sweep": {str(k): round(v, 3) for k, v in points.items()}}


def run_reference(args, world, rank):
    if rank != 0:
        return
    steps = max(1, min(args.steps, 3))
    warm = 1 if args.warmup > 0 else 0
    nproc = os.cpu_count() or 1
    r = cpu_reference(args.workload, steps, warm, sweep=sorted({max(1, nproc // 2), nproc}))
    sample = (f"{args.workload}: {r['cells']} cells, {warm} untimed + {steps} timed RK steps of the oracle "
              f"(CPU FP64 restatement of jst-rs; Rust toolchain absent), {r['cores']} OpenMP threads "
              f"(best of {sorted(int(k) for k in r['sweep'])} of {r['nproc']}), {r['cpu']}")
    line = {"metric": METRIC, "value": round(r["value"], 3), "unit": UNIT, "n_gpus": 0, "steps": steps,
            "warmup": warm, "ms_per_step": round(1e3 * r["seconds"] / steps, 3), "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "impl": "reference",
            "config": {"workload": args.workload, "precision": "fp64", "path": "cpu oracle"},
            "cpu_baseline": {"value": round(r["value"], 3), "unit": UNIT, "cores": r["cores"], "kind": "port",
                             "sample": sample, "cpu": r["cpu"], "nproc": r["nproc"], "sweep": r["sweep"]},
            "e2e": {"value": round(r["value"], 3), "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def run_ours(args, world, rank, local):
    from purinecfd_b200 import PATH_FUSED, PREC_FP32_SPLIT, PREC_FP64, Solver, workloads
    prec = PREC_FP32_SPLIT if args.precision == "split" else PREC_FP64
    cfg, xy, nr, nt = workloads.WORKLOADS[args.workload]()
    tile = {}
    if args.tile:
        parts = [int(x) for x in args.tile.lower().split("x")]
        tile = {"tile_i": parts[0], "tile_j": parts[1]}
        if len(parts) > 2:
            tile["block_threads"] = parts[2]
    s = Solver(cfg, xy, nr, nt, precision=prec, kernel_path=PATH_FUSED, device=local, staging=args.staging, **tile)
    cells = s.n_cells
    kcfg = s.kernel_config()
    kstg = s.kernel_staging()
    s.time_steps(args.warmup)
    barrier(world)
    with ClockSampler(local) as clk:
        ms, _ = s.time_steps(args.steps)
    barrier(world)
    ms_max = max_over_ranks(ms, world)
    _, stage_ms = s.time_steps(0, stages=True)
    residual = s.residual()
    s.close()
    value = replica_value(cells, args.steps, ms_max, world)

    line = {"metric": METRIC, "value": round(value, 3), "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": round(ms_max / args.steps, 5), "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None,
            "dtype": "f32+f64" if args.precision == "split" else "f64", "data": "synthetic",
            "config": {"workload": args.workload, "cells": cells, "precision": args.precision,
                       "path": {"march": "warp-marching strip", "march2": "paired-column warp-marching strip",
                                "tile": "tiled"}[kernel_kind(kcfg)] +
                               " stage kernel, one launch per RK stage, CUDA graph per RK step",
                       "tile": "x".join(map(str, kcfg)) + (" (autotuned)" if not args.tile else ""),
                       "staging": {0: None, 1: "per-lane cp.async", 2: "bulk cp.async.bulk (TMA)"}[kstg],
                       "parallelism": f"replicas x{world}" if world > 1 else "single GPU",
                       "l2": "inputs larger than L2 (state + geometry ~0.7 GB)"},
            "gpu_launches": 5 * args.steps, "residual_after": residual}

    if rank == 0:
        peak, peak_kind = measured_peaks()
        kind = kernel_kind(kcfg)
        bps = bytes_per_cell_stage(kind, args.precision)
        stage_avg = sum(stage_ms) / 5.0
        achieved = bps * cells / (stage_avg / 1e3) / 1e9
        trafc = ncu_traffic(kind, args.precision)
        line["roofline"] = {"bound": "hbm", "achieved": round(achieved, 1), "peak": peak, "unit": "GB/s",
                            "frac": round(achieved / peak, 4), "peak_kind": peak_kind,
                            "traffic": None if trafc is None else round(trafc * cells),
                            "kernel": KERNEL_NAMES[kind] +
                                      " (5 launches per step; mean stage times over 10 steps " +
                                      ", ".join(f"{x:.3f}" for x in stage_ms) + " ms)",
                            "bytes_per_cell_stage": round(bps, 1)}
        line["clocks"] = clk.summary()
        if world == 1 and not args.no_fp64:
            s64 = Solver(cfg, xy, nr, nt, precision=PREC_FP64, kernel_path=PATH_FUSED, device=local)
            s64.time_steps(3)
            k64 = max(5, min(args.steps, 100))
            ms64, st64 = s64.time_steps(k64, stages=True)
            v64 = cells * 5 * k64 / (ms64 / 1e3) / 1e6
            b64 = bytes_per_cell_stage(kernel_kind(s64.kernel_config()), "fp64")
            a64 = b64 * cells / (sum(st64) / 5.0 / 1e3) / 1e9
            line["fp64_plain"] = {"value": round(v64, 3), "unit": UNIT, "steps": k64,
                                  "ms_per_step": round(ms64 / k64, 5),
                                  "roofline": {"achieved": round(a64, 1), "peak": peak, "unit": "GB/s",
                                               "frac": round(a64 / peak, 4),
                                               "bytes_per_cell_stage": b64,
                                               "kernel": "x".join(map(str, s64.kernel_config()))}}
            s64.close()
            line["split_vs_fp64"] = split_vs_fp64(cfg, xy, nr, nt, local)
        # end to end through the public API from host buffers: create (mesh H2D,
        # geometry on the GPU), K steps with the per-step residual read back,
        # final fields D2H
        if not args.no_e2e:
            fields = ("rho", "u", "v", "p", "T", "nut")
            t0 = time.perf_counter()
            se = Solver(cfg, xy, nr, nt, precision=prec, kernel_path=PATH_FUSED, device=local)
            hist = []
            se.run(args.steps, lambda k, r: hist.append(r))
            out = [se.get(f) for f in fields]
            t_e2e = time.perf_counter() - t0
            se.close()
            h2d = xy.size * 8 + len(json.dumps(cfg))
            d2h = sum(a.nbytes for a in out) + 8 * args.steps
            line["e2e"] = {"value": round(cells * 5 * args.steps / t_e2e / 1e6, 3), "unit": UNIT,
                           "h2d_bytes_per_step": int(h2d / args.steps), "d2h_bytes_per_step": int(d2h / args.steps),
                           "seconds": round(t_e2e, 4),
                           "what": "jst_create from host nodes + jst_run with per-step residual callback + "
                                   "6 fields read back"}
    # every rank takes part in the batch and serving legs (instances are dealt over the ranks)
    if args.batch_instances > 0:
        batch = batched_leg(args, world, rank)
        if rank == 0:
            line["batch"] = batch
    if args.serve_requests > 0 and not args.no_serve:
        sv = serve_leg(args, world, rank, rates=[float(x) for x in args.serve_line_rates.split(",")])
        if rank == 0:
            line["serve"] = sv
    if rank == 0:
        if world == 1 and not args.no_cpu:
            r = cpu_reference(args.workload, 2, 1, sweep=thread_counts(os.cpu_count() or 1))
            line["cpu_baseline"] = {
                "value": round(r["value"], 3), "unit": UNIT, "cores": r["cores"], "kind": "port",
                "sample": f"{args.workload}: {r['cells']} cells, oracle (CPU FP64 restatement of jst-rs; Rust "
                          f"toolchain absent); 1 untimed step, then one step at each thread count of the sweep, "
                          f"then 2 timed RK steps at the fastest count ({r['cores']} of {r['nproc']})",
                "cpu": r["cpu"], "nproc": r["nproc"], "sweep_mcell_stage_per_s": r["sweep"],
                "ns_per_cell_step": round(1e9 * r["seconds"] / (r["cells"] * r["steps"]), 2)}
        print(json.dumps(line), flush=True)


def split_vs_fp64(cfg, xy, nr, nt, device, steps: int = 100) -> dict:
    """Error of the FP32/FP64 split path against the FP64 path (itself within
    1e-13 of the oracle on the parity workloads) on this workload: both run the
    same steps from the initial state; per field, the largest difference
    relative to the field's scale, and the CL/CD differences."""
    from purinecfd_b200 import PATH_FUSED, PREC_FP32_SPLIT, PREC_FP64, Solver
    runs = []
    for prec in (PREC_FP32_SPLIT, PREC_FP64):
        s = Solver(cfg, xy, nr, nt, precision=prec, kernel_path=PATH_FUSED, device=device)
        s.run(steps)
        runs.append(({f: s.get(f) for f in ("rho", "p", "T", "u", "v", "nut")}, s.forces()))
        s.close()
    (fa, (cla, cda)), (fb, (clb, cdb)) = runs
    err = {}
    for f in fa:
        scale = float(np.max(np.abs(fb[f]))) or 1.0
        err[f] = float(f"{float(np.max(np.abs(fa[f] - fb[f]))) / scale:.3g}")
    return {"steps": steps, "field_err_rel_scale": err, "cl_fp64": clb, "dcl": abs(cla - clb), "dcd": abs(cda - cdb)}


BATCH_SEED = 20261203


def stratified_sample(classes: list, m: int) -> list[int]:
    """Indices of about m instances with the mesh-class mix of the whole list
    (per class a share proportional to its count, at least one, the first
    ones drawn)."""
    by = {}
    for k, c in enumerate(classes):
        by.setdefault(c, []).append(k)
    out = []
    for c, ks in sorted(by.items()):
        take = max(1, round(m * len(ks) / len(classes)))
        out += ks[:take]
    return sorted(out)


def batched_leg(args, world: int = 1, rank: int = 0):
    """Config-4 distribution: NACA 4-digit instances on three mesh classes with
    seeded M, alpha, Re (local time stepping, CFL 1.0), solved (a) all at once
    in FP32-split batches, (b) all at once in FP64 batches as the CL/CD
    reference and (c) a sample with the same mesh-class mix one at a time on
    the plain FP64 path (a Solver per instance).  Every solve retires on a
    1e-6 residual drop, on |CL(n) - CL(n-100)| < cl_tol, or at the step cap.
    With several ranks the instances are dealt by purinecfd_b200.shard (least
    work first); the job time is the slowest rank's."""
    from purinecfd_b200 import DT_LOCAL, PREC_FP32_SPLIT, PREC_FP64, Solver, workloads
    from purinecfd_b200.serve import solve_alone
    from purinecfd_b200.shard import Group, solve_sharded
    g = Group()
    cases, classes = [], []
    for k in range(args.batch_instances):
        cfg, xy, nr, nt, _ = workloads.batch_instance(BATCH_SEED, k)
        cfg["simulation"]["CFL"] = 1.0
        cases.append((cfg, xy, nr, nt))
        classes.append(f"{nt + 1}x{nr}")
    rules = dict(max_steps=args.batch_steps, residual_drop=1e-6, cl_tol=args.batch_cl_tol)
    kinfo = {}
    barrier(world)
    split, wall, _ = solve_sharded(cases, PREC_FP32_SPLIT, group=g, info=kinfo, steps_per_poll=50, **rules)
    barrier(world)
    ref, wall_ref, _ = solve_sharded(cases, PREC_FP64, group=g, steps_per_poll=50, **rules)
    if rank != 0:
        return None
    n = len(cases)
    cells = [(c[2] - 1) * c[3] for c in cases]
    # plain FP64 one at a time on a sample with the batch's mesh-class mix;
    # per class the mean solve time, weighted by the class counts of the batch
    sample = stratified_sample(classes, args.plain_instances)
    # the autotuner's choice is cached per mesh class: one untimed solver per
    # class first, so that the sampled solves do not carry the one-off tuning
    # (the 256 instances would share it across 80-90 solves per class)
    warmed = set()
    for k in sample:
        if classes[k] not in warmed:
            warmed.add(classes[k])
            s = Solver(*cases[k], precision=PREC_FP64, dt_mode=DT_LOCAL, device=g.local_rank)
            s.run(1)
            s.close()
    t_cls, n_cls, plain_cell_steps, plain_wall = {}, {}, 0, 0.0
    for k in sample:
        r = solve_alone(cases[k], PREC_FP64, poll=50, device=g.local_rank, **rules)
        t_cls.setdefault(classes[k], []).append(r.t_done)
        plain_cell_steps += cells[k] * r.steps
        plain_wall += r.t_done
    for c in classes:
        n_cls[c] = n_cls.get(c, 0) + 1
    plain_time_all = sum(n_cls[c] * float(np.mean(t_cls[c])) for c in n_cls)
    plain_sps = n / plain_time_all
    ok = [(a, r) for a, r in zip(split, ref) if a.status != 8 and r.status != 8]
    dcl = [abs(a.cl - r.cl) for a, r in ok]
    dcd = [abs(a.cd - r.cd) for a, r in ok]
    conv = [k for k, a in enumerate(split) if a.status == 0]
    bad_split = {k for k, a in enumerate(split) if a.status == 8}
    bad_fp64 = {k for k, r in enumerate(ref) if r.status == 8}
    cell_steps = sum(c * a.steps for c, a in zip(cells, split))
    sps = n / wall
    return {"instances": n, "ranks": world, "cells": sum(cells), "step_cap": args.batch_steps,
            "rules": f"residual drop 1e-6, |dCL| < {args.batch_cl_tol:g} over 100 steps, cap {args.batch_steps}",
            "kernel": kinfo.get("kernel"), "classes": {c: n_cls[c] for c in sorted(n_cls)},
            "solves_per_s": round(sps, 3), "wall_s": round(wall, 3),
            "mcell_stage_per_s": round(cell_steps * 5 / wall / 1e6, 1),
            "converged": len(conv), "converged_solves_per_s": round(len(conv) / wall, 3),
            "nonphysical": len(bad_split), "nonphysical_fp64": len(bad_fp64),
            "nonphysical_in_both": len(bad_split & bad_fp64),
            "mean_steps": round(sum(a.steps for a in split) / max(1, n), 1),
            "fp64_batch_solves_per_s": round(n / wall_ref, 3) if wall_ref > 0 else None,
            "fp64_batch_converged": sum(1 for r in ref if r.status == 0),
            "plain_fp64_one_at_a_time": {
                "sample": len(sample), "sample_classes": {c: len(v) for c, v in sorted(t_cls.items())},
                "mean_s_per_class": {c: round(float(np.mean(v)), 4) for c, v in sorted(t_cls.items())},
                "solves_per_s_matched": round(plain_sps, 3),
                "mcell_stage_per_s": round(plain_cell_steps * 5 / plain_wall / 1e6, 1) if plain_wall else None,
                "what": "a Solver per instance (autotuned stage kernel, CUDA graph per step), FP64, the same "
                        "stopping rules checked every 50 steps, after one untimed solver per class (the autotuner "
                        "caches its choice per mesh class); solves/s for the batch's class mix = instances / "
                        "sum over classes of (count x mean solve time of the sampled instances of that class)"},
            "speedup_vs_plain": round(sps / (plain_sps * world), 2),
            "speedup_vs_plain_cell_steps": round((cell_steps * 5 / wall) / (plain_cell_steps * 5 / plain_wall), 2)
            if plain_wall else None,
            "cl_err_max": max(dcl) if dcl else None, "cd_err_max": max(dcd) if dcd else None,
            "within_1e-4": f"{sum(1 for x, y in zip(dcl, dcd) if x <= 1e-4 and y <= 1e-4)}/{n}",
            "what": f"seed {BATCH_SEED}, PCG64 stream per instance; local time step; CL/CD error of the split batch "
                    "vs the FP64 batch on the same instances (instances not NonPhysical in either); "
                    "instances dealt over the ranks by purinecfd_b200.shard, plain sample on rank 0 counted "
                    "once per GPU"}


def serve_leg(args, world: int = 1, rank: int = 0, rates=None, plain: bool = True):
    """Serving stream (config-5 draws: the batch distribution plus cylinders)
    with Poisson arrivals at each rate: the continuous-batching server
    (FP32-split) and, for comparison, the plain FP64 path serving the same
    stream one request at a time.  Requests are dealt over the ranks by
    purinecfd_b200.shard.  Returns the job figures (rank 0)."""
    from purinecfd_b200 import PREC_FP64
    from purinecfd_b200.serve import request_stream
    from purinecfd_b200.shard import Group, serve_sharded
    g = Group()
    out = []
    for rate in rates or [float(x) for x in args.serve_rates.split(",")]:
        reqs = request_stream(BATCH_SEED, args.serve_requests, max_steps=args.batch_steps)
        row = {"rate": rate}
        legs = [("batched_split", {})]
        if plain:
            legs.append(("plain_fp64", dict(precision=PREC_FP64, max_instances=1)))
        for name, kw in legs:
            barrier(world)
            st, _ = serve_sharded(reqs, rate, seed=int(rate), group=g, **kw)
            row[name] = {"completed": st.completed, "converged": st.converged, "nonphysical": st.nonphysical,
                         "wall_s": round(st.wall_s, 3), "solves_per_s": round(st.solves_per_s, 3),
                         "p50_s": round(st.p50_s, 4), "p99_s": round(st.p99_s, 4),
                         "mean_steps": round(st.mean_steps, 1)}
        if plain and row["plain_fp64"]["solves_per_s"]:
            row["speedup_solves_per_s"] = round(row["batched_split"]["solves_per_s"] /
                                                row["plain_fp64"]["solves_per_s"], 2)
        out.append(row)
        if rank == 0 and args.serve:
            print(json.dumps({"serve": row}), flush=True)
    return {"requests": args.serve_requests, "ranks": world, "step_cap": args.batch_steps,
            "rules": "residual drop 1e-6 or |dCL| < 1e-5 over 100 steps", "rates": out} if rank == 0 else None


def main():
    ap = argparse.ArgumentParser(description=__doc__, formatter_class=argparse.RawDescriptionHelpFormatter)
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=500)
    ap.add_argument("--warmup", type=int, default=10)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--workload", default="naca0012_4097x1025")
    ap.add_argument("--precision", choices=["split", "fp64"], default="split")
    ap.add_argument("--tile", default="", help="fused tile TIxTJ (default: the library's choice)")
    ap.add_argument("--staging", type=int, default=0, help="marching-strip row staging: 0 auto, 1 per-lane, 2 bulk")
    ap.add_argument("--no-fp64", action="store_true", help="skip the FP64 plain-path line")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-cpu", action="store_true", help="skip the CPU baseline sample")
    ap.add_argument("--batch-instances", type=int, default=256, help="config-4 batch size (0 = skip)")
    ap.add_argument("--batch-steps", type=int, default=2000, help="step cap per batched instance")
    ap.add_argument("--batch-cl-tol", type=float, default=1e-5, help="CL window tolerance of the batch leg")
    ap.add_argument("--plain-instances", type=int, default=24, help="FP64 one-at-a-time sample (class mix kept)")
    ap.add_argument("--serve", action="store_true", help="run the serving sweep instead of the benchmark")
    ap.add_argument("--serve-rates", default="1,10,50,200", help="rates of the --serve sweep")
    ap.add_argument("--serve-line-rates", default="10,200", help="rates of the serving summary in the line")
    ap.add_argument("--serve-requests", type=int, default=48)
    ap.add_argument("--no-serve", action="store_true", help="skip the serving summary")
    args = ap.parse_args()
    if args.warmup < 3 and args.impl == "ours":
        args.warmup = 3
    world, rank, local = dist_setup() if args.impl == "ours" else (int(os.environ.get("WORLD_SIZE", "1")),
                                                                   int(os.environ.get("RANK", "0")), 0)
    try:
        if args.serve:
            serve_leg(args, world, rank)
            return
        if args.impl == "reference":
            run_reference(args, world, rank)
        else:
            run_ours(args, world, rank, local)
    finally:
        if world > 1 and args.impl == "ours":
            import torch.distributed as dist
            dist.destroy_process_group()


if __name__ == "__main__":
    main()
