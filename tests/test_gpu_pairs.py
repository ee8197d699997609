"""The paired-column marching kernel of the FP32/FP64 split precision
(k_march2: two columns per lane in the sm_100 paired FP32 instructions,
strips of 56 columns, selected by tile_j = 56) against the oracle and against
the one-column marching kernel (tile_j = 26) of the same precision.

Tolerances are the split path's: fields within 1e-5 of their scale after
100 steps (the FP32 stage arithmetic against the FP64 oracle), the per-cell
residual of the FP64 state within 2e-3 of each component's scale.  Between
the two FP32 kernels the differences are FP32 roundings of the same formulas
(contracted differently), so they are held to the same tolerances."""

from __future__ import annotations

import numpy as np
import pytest

from conftest import load_config
from gpu_common import STATE_FIELDS, cylinder_case, rel_field_err
from test_gpu_residual import comp_errors, oracle_residual

import jst_oracle as jo

pytestmark = pytest.mark.gpu

PAIRS = [(16, 56, 64), (64, 56, 64), (32, 56, 128), (8, 56, 64), (5, 56, 128)]


def _split(cfg, xy, nr, nt, cfgt=None, **kw):
    from purinecfd_b200 import PATH_FUSED, PREC_FP32_SPLIT, Solver
    if cfgt:
        kw.update(tile_i=cfgt[0], tile_j=cfgt[1], block_threads=cfgt[2])
    return Solver(cfg, xy, nr, nt, kernel_path=PATH_FUSED, precision=PREC_FP32_SPLIT, **kw)


def _naca(nr=33, nt=128, spacing=1e-6, mach=0.6, aoa=2.0):
    from purinecfd_b200 import meshgen
    xy = meshgen.naca4_o_mesh(nr, nt, 0.02, 0.4, 0.12, r_far=30.0, first_spacing=spacing)
    return load_config({"simulation": {"Ma": mach, "AOA": aoa, "CFL": 0.8}}), xy, nr, nt


@pytest.mark.parametrize("cfgt", PAIRS, ids=lambda t: "x".join(map(str, t)))
@pytest.mark.parametrize("case", ["cylinder_33x64", "cylinder_29x63_odd", "naca_33x128_wall1e-6"])
def test_pairs_track_oracle_and_single_column_kernel(case, cfgt):
    """100 steps: fields within 1e-5 of the FP64 oracle and of the one-column
    split kernel; residual histories within 1e-4 of each other.  The odd ring
    (63 columns) takes the element-wise copies and stores."""
    if case == "cylinder_33x64":
        cfg, xy, nr, nt = cylinder_case(33, 64)
    elif case == "cylinder_29x63_odd":
        cfg, xy, nr, nt = cylinder_case(29, 63)
    else:
        cfg, xy, nr, nt = _naca()
    p = _split(cfg, xy, nr, nt, cfgt)
    assert p.kernel_config() == cfgt
    one = _split(cfg, xy, nr, nt, (16, 26, 64))
    o = jo.OracleSolver(cfg, xy, nr, nt)
    hp, h1 = [], []
    p.run(100, lambda k, r: hp.append(r))
    one.run(100, lambda k, r: h1.append(r))
    o.run(100)
    np.testing.assert_allclose(hp, h1, rtol=1e-4)
    for name in STATE_FIELDS:
        e_o = rel_field_err(p.get(name), o.get(name))
        e_1 = rel_field_err(p.get(name), one.get(name))
        assert e_o < 1e-5 and e_1 < 1e-5, (name, e_o, e_1)
    p.close()
    one.close()


@pytest.mark.parametrize("cfgt", [(16, 56, 64), (64, 56, 128)], ids=lambda t: "x".join(map(str, t)))
def test_pairs_stage_residual_of_the_fp64_state(cfgt):
    cfg, xy, nr, nt = _naca()
    o = jo.OracleSolver(cfg, xy, nr, nt)
    o.run(20)
    s = _split(cfg, xy, nr, nt, cfgt)
    s.set_conserved(np.stack([o.get(f"U{k}") for k in range(5)]))
    errs = comp_errors(s.stage_residual(), oracle_residual(o))
    one = _split(cfg, xy, nr, nt, (16, 26, 64))
    one.set_conserved(np.stack([o.get(f"U{k}") for k in range(5)]))
    errs1 = comp_errors(one.stage_residual(), oracle_residual(o))
    print(f"pairs {cfgt}: field-scaled residual error {['%.1e' % e for e in errs]} "
          f"(one-column kernel {['%.1e' % e for e in errs1]})")
    assert max(errs) < 2e-3, errs
    s.close()
    one.close()
    o.close()


def test_pairs_report_the_first_failed_cell_like_the_single_column_kernel():
    from purinecfd_b200 import NonPhysical
    from gpu_common import mesh_case
    xy, nr, nt = mesh_case("fangdata.txt")
    cfg = load_config({"simulation": {"CFL": 20.0}})
    got = []
    for cfgt in [(8, 56, 64), (8, 26, 64)]:
        s = _split(cfg, xy, nr, nt, cfgt)
        with pytest.raises(NonPhysical) as ei:
            s.advance()
        got.append((ei.value.i, ei.value.j))
        s.close()
    assert got[0] == got[1], got


def test_pairs_run_to_run_bitwise():
    cfg, xy, nr, nt = _naca()
    runs = []
    for _ in range(2):
        s = _split(cfg, xy, nr, nt, (16, 56, 64))
        rep = s.run(30)
        runs.append((rep.residual, [s.get(f"U{k}") for k in range(5)]))
        s.close()
    assert runs[0][0] == runs[1][0]
    for k in range(5):
        assert np.array_equal(runs[0][1][k], runs[1][1][k])


def test_pairs_batch_equals_alone_bitwise():
    """Instances of different sizes (even and odd rings) in one batch on the
    paired kernel give bitwise the state each gives alone."""
    from purinecfd_b200 import DT_LOCAL, PREC_FP32_SPLIT
    from purinecfd_b200.batch import Batch
    cases = [_naca(33, 128), _naca(17, 64, 1e-4, 0.4, -1.0), cylinder_case(29, 63)]
    steps = 40
    kw = dict(precision=PREC_FP32_SPLIT, dt_mode=DT_LOCAL, steps_per_poll=20, keep_fields=True, tile_i=16,
              tile_j=56, block_threads=64)
    mixed = Batch(hbm_budget_gb=2.0, **kw)
    ids = [mixed.submit(cfg, xy, nr, nt, max_steps=steps) for cfg, xy, nr, nt in cases]
    res = {r.id: r for r in mixed.run_all(chunk=20)}
    assert mixed.kernel_config() == (16, 56, 64)
    for i, (cfg, xy, nr, nt) in zip(ids, cases):
        s = _split(cfg, xy, nr, nt, (16, 56, 64), dt_mode=DT_LOCAL)
        s.run(steps)
        for c in range(5):
            assert np.array_equal(s.get(f"U{c}"), res[i].fields[c]), (i, c)
        s.close()
    mixed.close()
