"""Continuous batching: requests arriving while others run are admitted as
slots free up, every request completes, and each result equals the result of
the same request solved alone."""

from __future__ import annotations

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def test_serving_completes_every_request_and_matches_alone():
    from purinecfd_b200 import PREC_FP32_SPLIT
    from purinecfd_b200.batch import Batch
    from purinecfd_b200.serve import request_stream, serve
    reqs = request_stream(7, 6, max_steps=60)
    for r in reqs:  # keep the test small
        r.residual_drop, r.cl_tol = 0.0, 0.0
    st, results = serve(reqs, rate=50.0, max_instances=3, hbm_budget_gb=4.0, chunk=20, steps_per_poll=20)
    assert st.completed == 6 and st.p99_s >= st.p50_s > 0.0
    assert all(res.steps == 60 for _, res, _ in results)
    for k, res, _ in results[:2]:
        r = reqs[k]
        b = Batch(precision=PREC_FP32_SPLIT, steps_per_poll=20, hbm_budget_gb=1.0)
        b.submit(r.config, r.xy, r.n_rings, r.n_theta, max_steps=60)
        alone = b.run_all(chunk=20)[0]
        # the same state bitwise; the residual is a sum over tiles in an order set by the tile shape
        assert alone.cl == res.cl and alone.cd == res.cd
        assert abs(alone.residual - res.residual) <= 1e-12 * res.residual
        assert abs(alone.residual_first - res.residual_first) <= 1e-12 * res.residual_first
        b.close()
