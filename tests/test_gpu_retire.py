"""Batch monitoring rules that decide when an instance leaves the GPU.

* CL window: an instance submitted with cl_tol > 0 retires, converged, at the
  first poll where its lift coefficient has moved by less than cl_tol over
  the last 100 or more steps.  CL is sampled at polls at least 50 steps apart
  (every poll here: 50 steps per graph replay), and each sample is compared
  with the latest sample at least 100 steps older.  The expected step is
  computed independently from a single solver's CL history at the same steps
  (batch and single solves give bitwise identical states).
* HBM budget: instances are admitted while their footprint fits the batch's
  device-memory budget, even with free slots; the rest wait in the queue and
  are admitted as earlier instances retire.
"""

from __future__ import annotations

import numpy as np
import pytest

from conftest import load_config

pytestmark = pytest.mark.gpu


def _case(mach=0.5, aoa=3.0):
    from purinecfd_b200 import meshgen
    xy = meshgen.naca4_o_mesh(33, 96, 0.02, 0.4, 0.12, first_spacing=1e-3)
    cfg = load_config({"simulation": {"Ma": mach, "AOA": aoa, "CFL": 1.5}})
    return cfg, xy, 33, 96


def test_cl_window_retires_at_the_step_the_rule_gives():
    from purinecfd_b200 import DT_LOCAL, PREC_FP64, Solver
    from purinecfd_b200.batch import Batch
    cfg, xy, nr, nt = _case()
    poll, cap = 50, 2000
    # CL history of the same solve at the poll steps
    strips = dict(tile_i=16, tile_j=26, block_threads=64)  # the same stage kernel on both sides
    s = Solver(cfg, xy, nr, nt, precision=PREC_FP64, dt_mode=DT_LOCAL, **strips)
    steps, cls = [], []
    for k in range(1, cap // poll + 1):
        s.run(poll)
        steps.append(k * poll)
        cls.append(s.forces()[0])
    s.close()
    cls = np.asarray(cls)
    d = np.abs(cls[2:] - cls[:-2])  # |CL(s) - CL(s - 100)| for s = 150, 200, ...
    # a tolerance the window meets for the first time in the middle of the run
    k_mid = len(d) // 2
    tol = float(np.min(d[: k_mid + 1])) * (1.0 + 1e-9)
    first = int(np.argmax(d < tol))
    expected = steps[first + 2]
    assert 150 <= expected < cap
    b = Batch(precision=PREC_FP64, dt_mode=DT_LOCAL, steps_per_poll=poll, keep_fields=False, hbm_budget_gb=1.0,
              **strips)
    i_win = b.submit(cfg, xy, nr, nt, max_steps=cap, cl_tol=tol)
    i_cap = b.submit(cfg, xy, nr, nt, max_steps=expected + 2 * poll)  # no window: runs to its cap
    res = {r.id: r for r in b.run_all(chunk=poll)}
    assert res[i_win].status == 0 and res[i_win].steps == expected, (res[i_win].status, res[i_win].steps, expected)
    assert res[i_cap].status == 10 and res[i_cap].steps == expected + 2 * poll
    # the retired instance's CL is the solver's at that step
    assert abs(res[i_win].cl - cls[first + 2]) <= 1e-12 * abs(cls[first + 2])
    b.close()


def test_admission_is_limited_by_the_hbm_budget():
    from purinecfd_b200 import DT_LOCAL, PREC_FP64
    from purinecfd_b200.batch import Batch
    cfg, xy, nr, nt = _case()
    steps, poll = 40, 20
    # footprint of one instance, from a batch that admits it
    probe = Batch(precision=PREC_FP64, dt_mode=DT_LOCAL, steps_per_poll=poll, hbm_budget_gb=1.0)
    probe.submit(cfg, xy, nr, nt, max_steps=steps)
    probe.step(poll)
    _, _, one = probe.stats()
    probe.close()
    assert one > 0
    budget = 2.5 * one  # room for two instances, not three
    b = Batch(precision=PREC_FP64, dt_mode=DT_LOCAL, steps_per_poll=poll, keep_fields=True,
              hbm_budget_gb=budget / 1e9, max_instances=64)
    ids = [b.submit(cfg, xy, nr, nt, max_steps=steps) for _ in range(5)]
    b.step(poll)
    active, queued, used = b.stats()
    assert (active, queued) == (2, 3), (active, queued)
    assert used <= budget
    res = {r.id: r for r in b.run_all(chunk=poll)}
    assert set(res) == set(ids)
    first = res[ids[0]]
    for i in ids:
        r = res[i]
        assert r.steps == steps and r.status == 10
        assert np.array_equal(r.fields, first.fields)  # the same solve, whenever it was admitted
    # the queued instances were admitted only after earlier ones retired
    assert min(res[i].t_admit for i in ids[2:]) >= min(res[ids[0]].t_done, res[ids[1]].t_done)
    b.close()
