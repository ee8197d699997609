"""The benchmark meshes against the oracle (CPU FP64 restatement of jst-rs).

* The single large solve: NACA0012 O-mesh 4097 x 1025 nodes (4,194,304
  cells, wall spacing 1e-6 chord, far field 30 chords), M 0.8, alpha 1.25 deg,
  Re 1e7 — the mesh every throughput figure is measured on — for 5 RK steps
  from the free stream, with the strip heights the autotuner picks there and
  forced ones.  FP64: every state field within 1e-10 of its scale, the
  residual history within 1e-9 relative, and the per-cell residual of the
  final state within 1e-10 of each component's scale.  FP32/FP64 split:
  fields within 1e-4.
* The batch distribution: one instance of each mesh class (129 x 65,
  257 x 129, 513 x 257 nodes; NACA 4-digit sections, wall spacing 1e-6
  chord) from the seeded batch draws, solved together in one batch with local
  time steps (the batch mode) and compared with the oracle instance by
  instance: conserved state within 1e-10 (FP64) or 1e-4 (split) of each
  field's scale, CL and CD within 1e-8 (FP64) or 1e-4 (split).
"""

from __future__ import annotations

import numpy as np
import pytest

from gpu_common import STATE_FIELDS, rel_field_err
from test_gpu_residual import comp_errors, oracle_residual

import jst_oracle as jo

pytestmark = pytest.mark.gpu

STEPS = 5
BATCH_SEED = 20261203
BATCH_STEPS = 20


def _clcd(o, cfg, xy, nt):
    """Oracle CL/CD of its current state (wall force after residual_terms)."""
    o.residual_terms()
    fx, fy = o.wall_force()
    a = np.deg2rad(cfg["simulation"]["AOA"])
    d = o.derived()
    n = nt - 1 if np.allclose(xy[0], xy[nt - 1]) else nt
    q = 0.5 * d["rho_inf"] * (d["u_inf"] ** 2 + d["v_inf"] ** 2) * (xy[:n, 0].max() - xy[:n, 0].min())
    return (-fx * np.sin(a) + fy * np.cos(a)) / q, (fx * np.cos(a) + fy * np.sin(a)) / q


@pytest.fixture(scope="module")
def naca_4097():
    from purinecfd_b200 import workloads
    cfg, xy, nr, nt = workloads.naca0012_4097x1025()
    o = jo.OracleSolver(cfg, xy, nr, nt)
    _, _, _, _, hist = o.run(STEPS, history=True)
    fields = {f: o.get(f) for f in STATE_FIELDS}
    resid = oracle_residual(o)
    o.close()
    return cfg, xy, nr, nt, hist, fields, resid


def _kernel_opts(kernel: str) -> dict:
    """Solver options of a kernel label: autotuned, strips_HxWxT (per-lane
    staging), bulk_HxWxT (bulk row staging), pairs_HxWxT."""
    if kernel == "autotuned":
        return {}
    h, w, t = map(int, kernel.split("_")[1].split("x"))
    kw = dict(tile_i=h, tile_j=w, block_threads=t)
    if kernel.startswith("bulk"):
        kw["staging"] = 2
    return kw


@pytest.mark.parametrize("kernel", ["autotuned", "strips_47x26x64", "strips_94x26x128", "bulk_47x26x64"])
def test_benchmark_mesh_fp64_matches_oracle(naca_4097, kernel):
    from purinecfd_b200 import PREC_FP64, Solver
    cfg, xy, nr, nt, hist_o, fields_o, resid_o = naca_4097
    kw = _kernel_opts(kernel)
    s = Solver(cfg, xy, nr, nt, precision=PREC_FP64, **kw)
    hist = []
    rep = s.run(STEPS, lambda k, r: hist.append(r))
    assert rep.steps == STEPS
    np.testing.assert_allclose(hist, hist_o, rtol=1e-9)
    errs = {f: rel_field_err(s.get(f), fields_o[f]) for f in STATE_FIELDS}
    assert max(errs.values()) < 1e-10, errs
    r_errs = comp_errors(s.stage_residual(), resid_o)
    assert max(r_errs) < 1e-10, r_errs
    print(f"4097x1025 fp64 {kernel} {s.kernel_config()}: fields {max(errs.values()):.1e}, "
          f"per-cell residual {max(r_errs):.1e}")
    s.close()


@pytest.mark.parametrize("kernel", ["autotuned", "strips_94x26x128", "bulk_94x26x128", "pairs_64x56x64"])
def test_benchmark_mesh_split_within_tolerance(naca_4097, kernel):
    from purinecfd_b200 import PREC_FP32_SPLIT, Solver
    cfg, xy, nr, nt, hist_o, fields_o, _ = naca_4097
    kw = _kernel_opts(kernel)
    s = Solver(cfg, xy, nr, nt, precision=PREC_FP32_SPLIT, **kw)
    rep = s.run(STEPS)
    assert rep.steps == STEPS
    errs = {f: rel_field_err(s.get(f), fields_o[f]) for f in STATE_FIELDS}
    print(f"4097x1025 split {kernel} {s.kernel_config()}: " + ", ".join(f"{k} {v:.1e}" for k, v in errs.items()))
    assert max(errs.values()) < 1e-4, errs
    assert abs(rep.residual - hist_o[-1]) < 1e-3 * hist_o[-1]
    s.close()


def _one_per_mesh_class():
    """The first instance of each mesh class in the seeded batch draws."""
    from purinecfd_b200 import workloads
    found = {}
    k = 0
    while len(found) < len(workloads.MESH_CLASSES):
        cfg, xy, nr, nt, meta = workloads.batch_instance(BATCH_SEED, k)
        found.setdefault((nr, nt), (k, cfg, xy, nr, nt))
        k += 1
    return [found[c] for c in workloads.MESH_CLASSES]


@pytest.fixture(scope="module")
def class_oracles():
    out = []
    for k, cfg, xy, nr, nt in _one_per_mesh_class():
        o = jo.OracleSolver(cfg, xy, nr, nt, local_dt=True)
        o.run(BATCH_STEPS)
        u = np.stack([o.get(f"U{c}") for c in range(5)])
        cl, cd = _clcd(o, cfg, xy, nt)
        out.append(dict(k=k, cfg=cfg, xy=xy, nr=nr, nt=nt, u=u, cl=cl, cd=cd))
        o.close()
    return out


@pytest.mark.parametrize("kernel", ["autotuned", "strips_64x26x64", "pairs_64x56x64"])
@pytest.mark.parametrize("prec", ["fp64", "split"])
def test_batch_mesh_classes_match_oracle(class_oracles, prec, kernel):
    from purinecfd_b200 import DT_LOCAL, PREC_FP32_SPLIT, PREC_FP64
    from purinecfd_b200.batch import Batch
    if kernel.startswith("pairs") and prec == "fp64":
        pytest.skip("the paired-column kernel is the split precision's")
    kw = {} if kernel == "autotuned" else dict(tile_i=64, tile_j=int(kernel.split("x")[1]), block_threads=64)
    b = Batch(precision=PREC_FP64 if prec == "fp64" else PREC_FP32_SPLIT, dt_mode=DT_LOCAL, steps_per_poll=10,
              keep_fields=True, hbm_budget_gb=4.0, **kw)
    ids = [b.submit(c["cfg"], c["xy"], c["nr"], c["nt"], max_steps=BATCH_STEPS) for c in class_oracles]
    res = {r.id: r for r in b.run_all(chunk=BATCH_STEPS)}
    field_tol, force_tol = (1e-10, 1e-8) if prec == "fp64" else (1e-4, 1e-4)
    for i, c in zip(ids, class_oracles):
        r = res[i]
        assert r.steps == BATCH_STEPS and r.status in (0, 10), (c["k"], r.status)
        errs = [rel_field_err(r.fields[q], c["u"][q]) for q in range(5)]
        print(f"batch {prec} {kernel} {b.kernel_config()} instance {c['k']} ({c['nr']}x{c['nt']}): "
              f"U {max(errs):.1e}, CL {abs(r.cl - c['cl']):.1e}, CD {abs(r.cd - c['cd']):.1e}")
        assert max(errs) < field_tol, (c["k"], errs)
        assert abs(r.cl - c["cl"]) < force_tol and abs(r.cd - c["cd"]) < force_tol, (r.cl, c["cl"], r.cd, c["cd"])
    b.close()
