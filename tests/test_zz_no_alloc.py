"""jst_residual_noalloc: the density residual for callers that cannot allocate
device memory (plugin hosts that own every device allocation, monitoring loops
that must not call cudaMalloc).  The caller owns the two density fields and the
result slot; the entry point only launches kernels, using a fixed file-scope
device array as scratch.

Checked through the C ABI against the solver's own residual (jst_residual,
the existing entry point) on two calls in a row.  This file is named so that
pytest collects it last.
"""

from __future__ import annotations

import ctypes

import numpy as np
import pytest

from conftest import load_config

pytestmark = pytest.mark.gpu

MAX_CELLS = 8192 * 2048


def _residual_noalloc(lib, rho, prev, ni, nj, out, stream):
    return lib.jst_residual_noalloc(ctypes.c_void_p(rho), ctypes.c_void_p(prev), ni, nj, ctypes.c_void_p(out),
                                    ctypes.c_void_p(stream))


def test_residual_noalloc_matches_solver_residual_on_two_calls():
    import torch

    from purinecfd_b200 import Solver, meshgen
    from purinecfd_b200.solver import lib

    L = lib()
    xy = meshgen.naca4_o_mesh(65, 128, 0.02, 0.4, 0.12, first_spacing=1e-4)
    cfg = load_config({"simulation": {"AOA": 2.0, "Ma": 0.5}})
    s = Solver(cfg, xy, 65, 128)
    out = torch.full((1,), float("nan"), dtype=torch.float64, device="cuda")
    stream = torch.cuda.current_stream().cuda_stream
    for _ in range(2):  # two calls in a row; the second sees the first call's leftover scratch
        prev = s.get("U0")
        s.advance()
        cur = s.get("U0")
        want = s.residual()
        d_prev = torch.tensor(prev, dtype=torch.float64, device="cuda")
        d_cur = torch.tensor(cur, dtype=torch.float64, device="cuda")
        rc = _residual_noalloc(L, d_cur.data_ptr(), d_prev.data_ptr(), s.ni, s.nj, out.data_ptr(), stream)
        assert rc == 0, L.jst_last_error(None)
        torch.cuda.synchronize()
        got = float(out.item())
        assert want > 0.0
        assert abs(got - want) <= 1e-12 * want, (got, want)
        # same value as the serial sum of the reference's formula (solver.rs:190-200)
        ref = float(np.sqrt(np.sum((cur - prev) ** 2) / s.ni / s.nj))
        assert abs(got - ref) <= 1e-12 * ref
    s.close()


def test_residual_noalloc_rejects_sizes_beyond_its_scratch():
    import torch

    from purinecfd_b200.solver import ERR_ARG, lib

    L = lib()
    d = torch.zeros(4, dtype=torch.float64, device="cuda")
    out = torch.zeros(1, dtype=torch.float64, device="cuda")
    rc = _residual_noalloc(L, d.data_ptr(), d.data_ptr(), 4097, 4097, out.data_ptr(), 0)
    assert rc == ERR_ARG
    assert b"exceed the maximum" in L.jst_last_error(None)
    assert 4097 * 4097 > MAX_CELLS
