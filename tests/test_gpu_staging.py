"""Bulk (TMA) row staging of the marching-strip kernels (JST_STAGING_BULK):
each field's row segment is one cp.async.bulk copy issued by one lane and
completed on the row buffer's mbarrier, instead of one cp.async per lane.

Staging changes only how the inputs reach shared memory, so on rings where
bulk copies apply (width a multiple of 16 bytes of the stage type and at
least 36 columns; the strips that cross the periodic seam copy their segments
in two pieces) the results are bitwise those of the per-lane staging, in FP64
and in the split precision.  On other rings the bulk kernel falls back to
per-lane copies; that fallback is a separately compiled code path, whose
FP32 contractions may differ in the last bit, so there the results agree
within the split precision's rounding (1e-6 of the field scale) and, in FP64,
within 1e-13.  The FP64 path also stays within 1e-10 of the oracle.

The failure path: a test hook makes every row barrier expect more bytes than
its copies deliver, the kernels' bounded waits run out, and the step returns
JST_ERR_TIMEOUT without faulting; a solver made afterwards runs normally."""

from __future__ import annotations

import numpy as np
import pytest

from conftest import load_config
from gpu_common import STATE_FIELDS, cylinder_case, rel_field_err

import jst_oracle as jo

pytestmark = pytest.mark.gpu

STRIPS = [(8, 26, 64), (32, 26, 128), (47, 26, 64)]


def _naca(nr, nt, spacing=1e-6):
    from purinecfd_b200 import meshgen
    xy = meshgen.naca4_o_mesh(nr, nt, 0.02, 0.4, 0.12, r_far=30.0, first_spacing=spacing)
    return load_config({"simulation": {"Ma": 0.6, "AOA": 2.0, "CFL": 0.8}}), xy, nr, nt


def _case(name):
    if name == "naca_33x128":
        return _naca(33, 128)
    nr, nt = map(int, name.split("_")[1].split("x"))
    return cylinder_case(nr, nt)


def _run(cfg, xy, nr, nt, prec, cfgt, staging, steps=30):
    from purinecfd_b200 import PATH_FUSED, Solver
    s = Solver(cfg, xy, nr, nt, kernel_path=PATH_FUSED, precision=prec, tile_i=cfgt[0], tile_j=cfgt[1],
               block_threads=cfgt[2], staging=staging)
    hist = []
    s.run(steps, lambda k, r: hist.append(r))
    out = (hist, [s.get(f"U{k}") for k in range(5)], s.kernel_staging())
    s.close()
    return out


@pytest.mark.parametrize("cfgt", STRIPS, ids=lambda t: "x".join(map(str, t)))
@pytest.mark.parametrize("prec", [0, 1], ids=["fp64", "split"])
@pytest.mark.parametrize("case", ["naca_33x128", "cylinder_33x64", "cylinder_29x38", "cylinder_29x63"])
def test_bulk_staging_is_bitwise_the_per_lane_staging(case, prec, cfgt):
    from purinecfd_b200.solver import STAGING_BULK, STAGING_PER_LANE
    cfg, xy, nr, nt = _case(case)
    h1, u1, st1 = _run(cfg, xy, nr, nt, prec, cfgt, STAGING_PER_LANE)
    h2, u2, st2 = _run(cfg, xy, nr, nt, prec, cfgt, STAGING_BULK)
    assert (st1, st2) == (STAGING_PER_LANE, STAGING_BULK)
    bulk_applies = nt % (4 if prec else 2) == 0 and nt >= 36
    if bulk_applies:
        assert h1 == h2
        for k in range(5):
            assert np.array_equal(u1[k], u2[k]), k
    else:
        tol = 1e-6 if prec else 1e-13
        np.testing.assert_allclose(h1, h2, rtol=tol)
        for k in range(5):
            assert rel_field_err(u2[k], u1[k]) < tol, k


@pytest.mark.parametrize("cfgt", STRIPS, ids=lambda t: "x".join(map(str, t)))
def test_bulk_staging_fp64_matches_oracle(cfgt):
    from purinecfd_b200 import PATH_FUSED, PREC_FP64, Solver
    from purinecfd_b200.solver import STAGING_BULK
    cfg, xy, nr, nt = _naca(33, 128)
    s = Solver(cfg, xy, nr, nt, kernel_path=PATH_FUSED, precision=PREC_FP64, tile_i=cfgt[0], tile_j=cfgt[1],
               block_threads=cfgt[2], staging=STAGING_BULK)
    o = jo.OracleSolver(cfg, xy, nr, nt)
    hist = []
    s.run(50, lambda k, r: hist.append(r))
    _, _, _, _, hist_o = o.run(50, history=True)
    np.testing.assert_allclose(hist, hist_o, rtol=1e-10)
    for name in STATE_FIELDS:
        assert rel_field_err(s.get(name), o.get(name)) < 1e-10, name
    s.close()
    o.close()


def test_bulk_staging_batch_equals_alone_bitwise():
    """A mixed batch on bulk staging (two rings where bulk copies apply, one
    odd ring that falls back) gives bitwise the state each instance gives
    alone on bulk staging, and the per-lane staging's state bitwise where bulk
    applies, within FP32 rounding on the fallback ring."""
    from purinecfd_b200 import DT_LOCAL, PREC_FP32_SPLIT
    from purinecfd_b200.batch import Batch
    from purinecfd_b200.solver import STAGING_BULK, STAGING_PER_LANE
    cases = [_naca(33, 128), _naca(17, 64, 1e-4), cylinder_case(29, 63)]
    kw = dict(precision=PREC_FP32_SPLIT, dt_mode=DT_LOCAL, steps_per_poll=20, keep_fields=True, tile_i=16, tile_j=26,
              block_threads=64, staging=STAGING_BULK)
    mixed = Batch(hbm_budget_gb=2.0, **kw)
    ids = [mixed.submit(cfg, xy, nr, nt, max_steps=40) for cfg, xy, nr, nt in cases]
    res = {r.id: r for r in mixed.run_all(chunk=20)}
    assert mixed.kernel_staging() == STAGING_BULK
    for i, (cfg, xy, nr, nt) in zip(ids, cases):
        for stg in (STAGING_BULK, STAGING_PER_LANE):
            alone = Batch(hbm_budget_gb=1.0, **dict(kw, staging=stg))
            alone.submit(cfg, xy, nr, nt, max_steps=40)
            ra = alone.run_all(chunk=20)[0]
            for c in range(5):
                if stg == STAGING_BULK or nt % 4 == 0:
                    assert np.array_equal(ra.fields[c], res[i].fields[c]), (i, stg, c)
                else:
                    assert rel_field_err(res[i].fields[c], ra.fields[c]) < 1e-6, (i, stg, c)
            alone.close()
    mixed.close()


def test_bounded_wait_running_out_is_reported_not_fatal():
    from purinecfd_b200 import PATH_FUSED, PREC_FP32_SPLIT, JstError, Solver
    from purinecfd_b200.solver import ERR_TIMEOUT, STAGING_BULK
    cfg, xy, nr, nt = _naca(33, 128)
    kw = dict(kernel_path=PATH_FUSED, precision=PREC_FP32_SPLIT, tile_i=16, tile_j=26, block_threads=64,
              staging=STAGING_BULK)
    s = Solver(cfg, xy, nr, nt, **kw)
    s.debug_staging_extra_tx(16)  # every row barrier waits for 16 bytes that never come
    with pytest.raises(JstError) as ei:
        s.advance()
    assert ei.value.status == ERR_TIMEOUT
    assert "bounded wait" in str(ei.value)
    s.close()
    # the context is still usable: a new solver runs and matches the per-lane staging
    h2, u2, _ = _run(cfg, xy, nr, nt, PREC_FP32_SPLIT, (16, 26, 64), STAGING_BULK, steps=10)
    h1, u1, _ = _run(cfg, xy, nr, nt, PREC_FP32_SPLIT, (16, 26, 64), 1, steps=10)
    assert h1 == h2 and all(np.array_equal(a, b) for a, b in zip(u1, u2))
