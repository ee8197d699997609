"""Per-cell residual of the production stage kernels against the reference.

jst_stage_residual returns R = Fc - Fv - Fd (R[4] -= S), the residual the RK
update applies (solver.rs:128-133), computed by the stage kernel a solver runs
its RK stages with: the marching-strip kernel or a tile kernel of the fused
path (stage 0 run without its update), or the strict passes.  It is checked

* against the reference's golden single-stage terms (after the golden's 3
  warm-up steps, jst-rs/tests/golden.rs:221-275 checks the same terms one by
  one), within 1e-10 of each component's field scale;
* against the oracle at the start of each of the first 100 iterations
  (the north-star criterion: 1e-10 relative per-cell residual over the first
  100 iterations), field-scaled, on the cylinder 40 x 17 case and on a
  NACA 4-digit mesh with a 1e-6 chord wall spacing;
* for the FP32/FP64 split kernels, against the FP64 oracle on the same
  (FP64) state: within 2e-3 of each component's field scale (measured 6.3e-4
  on a NACA mesh with a 1e-6 chord wall spacing; the residual is a small
  difference of FP32 face fluxes, so its error is set by the size of the
  terms it is made of, which the test prints beside it).
"""

from __future__ import annotations

import numpy as np
import pytest

from conftest import golden_cases, load_config, load_golden
from gpu_common import cylinder_case

import jst_oracle as jo

pytestmark = pytest.mark.gpu

# Stage kernels, as (name, solver options).  Strips: (max height, 26 columns,
# threads per block); tiles: (rows, columns, threads per block).
KERNELS = {
    "fused_autotuned": dict(kernel_path=0),
    "strips_8x26x64": dict(kernel_path=0, tile_i=8, tile_j=26, block_threads=64),
    "strips_32x26x128": dict(kernel_path=0, tile_i=32, tile_j=26, block_threads=128),
    "strips_64x26x256": dict(kernel_path=0, tile_i=64, tile_j=26, block_threads=256),
    "tiles_4x32x256": dict(kernel_path=0, tile_i=4, tile_j=32, block_threads=256),
    "tiles_16x32x384": dict(kernel_path=0, tile_i=16, tile_j=32, block_threads=384),
    "passes": dict(kernel_path=1),
}


def oracle_residual(o) -> np.ndarray:
    """R of the oracle's current state, after timestep::compute as in the
    first stage of a step (solver.rs:109-133)."""
    o.timestep()
    o.residual_terms()
    r = np.stack([o.get(f"Fc{k}") - o.get(f"Fv{k}") - o.get(f"Fd{k}") for k in range(5)])
    r[4] -= o.get("S")
    return r


def golden_residual(doc) -> np.ndarray:
    """R from the golden's separate terms (flat, i-major / j-minor)."""
    t = doc["terms"]
    r = np.stack([np.ravel(t[f"Fc{k + 1}"]) - np.ravel(t[f"Fv{k + 1}"]) - np.ravel(t[f"Fd{k + 1}"])
                  for k in range(5)])
    r[4] -= np.ravel(t["S5"])
    return r


def comp_errors(got: np.ndarray, want: np.ndarray) -> list[float]:
    """Per component: max |got - want| / max |want| over the cells."""
    out = []
    for k in range(5):
        w = np.asarray(want[k], float).ravel()
        g = np.asarray(got[k], float).ravel()
        scale = float(np.max(np.abs(w))) or 1.0
        out.append(float(np.max(np.abs(g - w)) / scale))
    return out


@pytest.mark.parametrize("kernel", list(KERNELS))
@pytest.mark.parametrize("case", golden_cases(), ids=lambda p: p.stem)
def test_stage_residual_matches_golden_terms(case, kernel):
    from purinecfd_b200 import Solver
    doc, cfg, mesh_text = load_golden(case)
    nr, nt, xy = jo.parse_mesh(mesh_text)
    s = Solver(cfg, xy, nr, nt, **KERNELS[kernel])
    s.run(doc["meta"]["warmup"])
    got = s.stage_residual()
    want = golden_residual(doc).reshape(5, s.ni, s.nj)
    errs = comp_errors(got, want)
    assert max(errs) < 1e-10, (kernel, errs)
    # and the same state's residual from the oracle, which follows the
    # reference's arithmetic: only contraction and CUDA's libm differ
    o = jo.OracleSolver(cfg, xy, nr, nt)
    o.run(doc["meta"]["warmup"])
    assert max(comp_errors(got, oracle_residual(o))) < 1e-11, kernel
    s.close()
    o.close()


def _naca_case():
    from purinecfd_b200 import meshgen
    xy = meshgen.naca4_o_mesh(33, 128, 0.02, 0.4, 0.12, r_far=30.0, first_spacing=1e-6)
    cfg = load_config({"simulation": {"Ma": 0.6, "AOA": 2.0, "CFL": 0.8}})
    return cfg, xy, 33, 128


@pytest.mark.parametrize("kernel", ["fused_autotuned", "strips_8x26x64", "strips_32x26x128", "tiles_4x32x256"])
@pytest.mark.parametrize("case", ["cylinder_40x17", "naca_33x128_wall1e-6"])
def test_stage_residual_first_100_iterations_within_1e10(case, kernel):
    """The north-star criterion, literally: at the start of each of the first
    100 iterations the GPU's per-cell residual agrees with the oracle's (each
    side on its own trajectory) within 1e-10 of the component's field scale."""
    from purinecfd_b200 import Solver
    cfg, xy, nr, nt = cylinder_case() if case == "cylinder_40x17" else _naca_case()
    s = Solver(cfg, xy, nr, nt, **KERNELS[kernel])
    o = jo.OracleSolver(cfg, xy, nr, nt)
    worst = 0.0
    for it in range(100):
        e = max(comp_errors(s.stage_residual(), oracle_residual(o)))
        worst = max(worst, e)
        assert e < 1e-10, (it, e)
        s.advance()
        o.advance()
    print(f"{case} {kernel}: worst field-scaled per-cell residual error over 100 iterations {worst:.2e}")
    s.close()
    o.close()


@pytest.mark.parametrize("kernel", ["fused_autotuned", "strips_8x26x64", "tiles_4x32x256"])
def test_split_stage_residual_within_fp32_tolerance(kernel):
    from purinecfd_b200 import PREC_FP32_SPLIT, Solver
    cfg, xy, nr, nt = _naca_case()
    s = Solver(cfg, xy, nr, nt, precision=PREC_FP32_SPLIT, **KERNELS[kernel])
    o = jo.OracleSolver(cfg, xy, nr, nt)
    for it in range(20):
        s.advance()
        o.advance()
    # the split state differs from the FP64 one by FP32 roundings; compare the
    # split kernel's residual of the FP64 state, so that only the stage
    # arithmetic differs
    u = np.stack([o.get(f"U{k}") for k in range(5)])
    s.set_conserved(u)
    got, want = s.stage_residual(), oracle_residual(o)
    errs = comp_errors(got, want)
    # the same error against the size of the terms R is the sum of
    terms = [np.abs(o.get(f"Fc{k}")) + np.abs(o.get(f"Fv{k}")) + np.abs(o.get(f"Fd{k}")) for k in range(5)]
    terms[4] = terms[4] + np.abs(o.get("S"))
    t_errs = [float(np.max(np.abs(got[k] - want[k])) / np.max(terms[k])) for k in range(5)]
    k_worst = int(np.argmax(errs))
    i, j = np.unravel_index(int(np.argmax(np.abs(got[k_worst] - want[k_worst]))), want[k_worst].shape)
    print(f"split {kernel}: residual error per component, field-scaled {['%.1e' % e for e in errs]}, "
          f"term-scaled {['%.1e' % e for e in t_errs]}; worst component {k_worst} at cell ({i}, {j})")
    assert max(errs) < 2e-3, errs
    s.close()
    o.close()
