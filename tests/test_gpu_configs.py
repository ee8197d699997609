"""The two single-mesh parity workloads at their full iteration counts, each
path against the oracle (CPU FP64 restatement of jst-rs) on the same mesh and
inputs:

* cylinder O-mesh 40 x 17 nodes (D = 1, far field 20, first spacing 1e-3),
  M 0.3, Re 1e5, nu-tilde = 3 nu, CFL 2.5, 2000 iterations;
* NACA0012 O-mesh 257 x 129 nodes (far field 30c, wall spacing 1e-6c),
  M 0.75, alpha 2 deg, Re 6e6, 5000 iterations.

Tolerances: FP64 paths within 1e-10 of each field's scale and 1e-8 on CL and
CD (measured: 3e-15 / 6e-14 on the fields, 2e-15 on CL and CD; the strict
passes path agrees with the oracle to the last bit on most fields of the NACA
case); FP32/FP64 split within 1e-4 on the fields, CL and CD (measured: 7e-7 and
4e-6 on the fields, 7e-7 and 4e-9 on CL/CD)."""

from __future__ import annotations

import numpy as np
import pytest

import jst_oracle as jo
from gpu_common import STATE_FIELDS, rel_field_err

pytestmark = pytest.mark.gpu

CASES = {"cylinder_40x17": 2000, "naca0012_257x129": 5000}


def _closed_ring(xy, nt):
    return nt - 1 if np.allclose(xy[0], xy[nt - 1]) else nt


@pytest.fixture(scope="module", params=list(CASES))
def reference(request):
    """(name, steps, cfg, mesh, oracle results) with the oracle run once per case."""
    from purinecfd_b200 import workloads
    name, steps = request.param, CASES[request.param]
    cfg, xy, nr, nt = workloads.WORKLOADS[name]()
    o = jo.OracleSolver(cfg, xy, nr, nt)
    done, res, _, _ = o.run(steps)
    assert done == steps
    fields = {f: o.get(f) for f in STATE_FIELDS}
    o.residual_terms()
    fx, fy = o.wall_force()
    a = np.deg2rad(cfg["simulation"]["AOA"])
    d = o.derived()
    n = _closed_ring(xy, nt)
    q = 0.5 * d["rho_inf"] * (d["u_inf"] ** 2 + d["v_inf"] ** 2) * (xy[:n, 0].max() - xy[:n, 0].min())
    cl, cd = (-fx * np.sin(a) + fy * np.cos(a)) / q, (fx * np.cos(a) + fy * np.sin(a)) / q
    o.close()
    return name, steps, cfg, (xy, nr, nt), {"residual": res, "fields": fields, "cl": cl, "cd": cd}


# the *_strips paths force the marching strips, whose single-solve kernel takes
# the instance descriptor as a launch parameter: the 5000-step run outgrows the
# residual history (4096 steps), and the step graph is captured again after it
STRIPS = dict(tile_i=16, tile_j=26, block_threads=64)


@pytest.mark.parametrize("path", ["fused_fp64", "passes", "fused_split", "fused_fp64_strips", "fused_split_strips"])
def test_full_run_matches_oracle(reference, path):
    from purinecfd_b200 import PATH_FUSED, PATH_PASSES, PREC_FP32_SPLIT, PREC_FP64, Solver
    name, steps, cfg, (xy, nr, nt), ref = reference
    kw = {"fused_fp64": dict(kernel_path=PATH_FUSED, precision=PREC_FP64),
          "passes": dict(kernel_path=PATH_PASSES, precision=PREC_FP64),
          "fused_split": dict(kernel_path=PATH_FUSED, precision=PREC_FP32_SPLIT),
          "fused_fp64_strips": dict(kernel_path=PATH_FUSED, precision=PREC_FP64, **STRIPS),
          "fused_split_strips": dict(kernel_path=PATH_FUSED, precision=PREC_FP32_SPLIT, **STRIPS)}[path]
    split = path.startswith("fused_split")
    field_tol, force_tol = (1e-4, 1e-4) if split else (1e-10, 1e-8)
    s = Solver(cfg, xy, nr, nt, **kw)
    rep = s.run(steps)
    assert rep.steps == steps
    for f in STATE_FIELDS:
        assert rel_field_err(s.get(f), ref["fields"][f]) < field_tol, (name, f)
    cl, cd = s.forces()
    assert abs(cl - ref["cl"]) < force_tol and abs(cd - ref["cd"]) < force_tol, (cl, ref["cl"], cd, ref["cd"])
    if not split:
        assert abs(rep.residual - ref["residual"]) < 1e-10 * ref["residual"]
    if "strips" in path:
        assert s.kernel_config() == (16, 26, 64)
        hist = []
        s.run(3, lambda k, r: hist.append(r))  # after the history grew: the graph runs on
        assert len(hist) == 3 and all(np.isfinite(hist))
    s.close()
