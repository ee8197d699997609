"""Batched solving: every instance of a mixed batch gives the same result as
when solved alone (bitwise: no arithmetic crosses instances, reductions are
per instance and deterministic), instances retire on their own criteria, and
a non-physical instance retires without disturbing the others."""

from __future__ import annotations

import numpy as np
import pytest

from conftest import load_config

pytestmark = pytest.mark.gpu


def _cases():
    from purinecfd_b200 import meshgen
    out = []
    for k, (nr, nt, m, t, mach, aoa) in enumerate([(33, 64, 0.0, 0.12, 0.5, 2.0), (17, 128, 0.02, 0.10, 0.7, -1.0),
                                                   (65, 96, 0.04, 0.15, 0.3, 6.0)]):
        xy = meshgen.naca4_o_mesh(nr, nt, m, 0.4, t, first_spacing=1e-3)
        cfg = load_config({"simulation": {"Ma": mach, "AOA": aoa, "CFL": 1.5}})
        out.append((cfg, xy, nr, nt))
    return out


@pytest.mark.parametrize("prec", [0, 1], ids=["fp64", "split"])
def test_batch_results_equal_alone_results(prec):
    from purinecfd_b200 import DT_LOCAL, Solver
    from purinecfd_b200.batch import Batch
    cases = _cases()
    steps = 60
    mixed = Batch(precision=prec, dt_mode=DT_LOCAL, steps_per_poll=20, keep_fields=True, hbm_budget_gb=2.0)
    ids = [mixed.submit(cfg, xy, nr, nt, max_steps=steps) for cfg, xy, nr, nt in cases]
    res = {r.id: r for r in mixed.run_all(chunk=20)}
    assert set(res) == set(ids)
    for k, (cfg, xy, nr, nt) in enumerate(cases):
        alone = Batch(precision=prec, dt_mode=DT_LOCAL, steps_per_poll=20, keep_fields=True, hbm_budget_gb=1.0)
        a_id = alone.submit(cfg, xy, nr, nt, max_steps=steps)
        ra = alone.run_all(chunk=20)[0]
        rm = res[ids[k]]
        assert ra.steps == rm.steps == steps
        assert np.array_equal(ra.fields, rm.fields)
        assert ra.residual == rm.residual and ra.cl == rm.cl and ra.cd == rm.cd
        # and the single-solver path gives the same state
        s = Solver(cfg, xy, nr, nt, precision=prec, dt_mode=DT_LOCAL)
        s.run(steps)
        for c in range(5):
            assert np.array_equal(s.get(f"U{c}"), rm.fields[c]), c
        alone.close()
        s.close()
    mixed.close()


def test_batch_retires_on_residual_drop_and_step_limit():
    from purinecfd_b200.batch import Batch
    cases = _cases()
    b = Batch(steps_per_poll=10, hbm_budget_gb=1.0)
    i_drop = b.submit(*cases[0], max_steps=5000, residual_drop=0.3)
    i_lim = b.submit(*cases[1], max_steps=40, residual_drop=1e-12)
    res = {r.id: r for r in b.run_all(chunk=50)}
    assert res[i_drop].status == 0 and res[i_drop].residual < 0.3 * res[i_drop].residual_first
    assert res[i_drop].steps < 5000
    assert res[i_lim].status == 10 and res[i_lim].steps == 40  # JST_ERR_TIMEOUT: step limit
    for r in res.values():
        assert np.isfinite(r.cl) and np.isfinite(r.cd)
        assert r.t_submit <= r.t_admit <= r.t_done


def test_nonphysical_instance_retires_alone():
    from purinecfd_b200 import meshgen
    from purinecfd_b200.batch import Batch
    cases = _cases()
    b = Batch(steps_per_poll=10, hbm_budget_gb=1.0, keep_fields=True)
    good = b.submit(*cases[0], max_steps=50)
    xy = meshgen.ellipse_o_mesh(13, 40)
    bad = b.submit(load_config({"simulation": {"CFL": 200.0}}), xy, 13, 40, max_steps=400)
    res = {r.id: r for r in b.run_all(chunk=50)}
    assert res[bad].status == 8  # JST_ERR_NONPHYSICAL
    assert res[good].status == 10 and res[good].steps == 50
    assert np.all(np.isfinite(res[good].fields))


def test_admission_is_limited_by_slots_and_continues():
    from purinecfd_b200.batch import Batch
    cases = _cases()
    b = Batch(max_instances=2, steps_per_poll=10, hbm_budget_gb=1.0)
    ids = [b.submit(*cases[k % 3], max_steps=30) for k in range(5)]
    b.step(0)
    a, q, _ = b.stats()
    assert a <= 2 and a + q == 5
    res = {r.id: r for r in b.run_all(chunk=30)}
    assert set(res) == set(ids) and all(r.steps == 30 for r in res.values())


def test_kernel_configuration_is_reported():
    """Given options are kept; otherwise the autotuner's choice at the first
    step is one of the compiled configurations."""
    from purinecfd_b200.batch import Batch
    cases = _cases()
    fixed = Batch(tile_i=32, tile_j=26, block_threads=64, steps_per_poll=10, hbm_budget_gb=1.0)
    fixed.submit(*cases[0], max_steps=10)
    fixed.run_all(chunk=10)
    assert fixed.kernel_config() == (32, 26, 64)
    tuned = Batch(steps_per_poll=10, hbm_budget_gb=1.0)
    tuned.submit(*cases[1], max_steps=10)
    tuned.run_all(chunk=10)
    ti, tj, nt = tuned.kernel_config()
    assert tj in (26, 32, 64) and ti > 0 and nt in (64, 128, 256)


@pytest.mark.parametrize("prec", [0, 1], ids=["fp64", "split"])
def test_single_instance_kernel_equals_batch_kernel(prec):
    """A single solve on marching strips runs the kernel that takes the
    instance descriptor as a parameter (k_march_solo); a batch runs the one
    that reads it from the instance table.  Same strips, same arithmetic: the
    states agree bit for bit."""
    from purinecfd_b200 import DT_LOCAL, Solver
    from purinecfd_b200.batch import Batch
    cfg, xy, nr, nt = _cases()[2]
    steps = 40
    s = Solver(cfg, xy, nr, nt, precision=prec, dt_mode=DT_LOCAL, tile_i=16, tile_j=26, block_threads=64)
    s.run(steps)
    b = Batch(precision=prec, dt_mode=DT_LOCAL, steps_per_poll=20, keep_fields=True, hbm_budget_gb=1.0, tile_i=16,
              tile_j=26, block_threads=64)
    b.submit(cfg, xy, nr, nt, max_steps=steps)
    r = b.run_all(chunk=20)[0]
    assert s.kernel_config() == b.kernel_config() == (16, 26, 64)
    for c in range(5):
        assert np.array_equal(s.get(f"U{c}"), r.fields[c]), c
    s.close()
    b.close()
