"""The marching kernels' FP64 quotient, square root, exponential and inverse
sixth root (hardware approximations refined by Newton-Raphson steps; Cody-Waite
reduction and a Taylor polynomial) against CUDA's: the quotient and root at
most one unit in the last place from the correctly rounded ones over operands
spanning sixty decades, the exponential within two units of CUDA's exp, the
inverse sixth root within four units of 1 / cbrt(sqrt(d)), and NaN in, NaN
out."""

from __future__ import annotations

import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _run(a: np.ndarray, b: np.ndarray) -> np.ndarray:
    from purinecfd_b200.solver import OK, lib
    a = np.ascontiguousarray(a, dtype=np.float64)
    b = np.ascontiguousarray(b, dtype=np.float64)
    out = np.empty(8 * a.size)
    pd = C.POINTER(C.c_double)
    rc = lib().jst_debug_quick_arith(a.ctypes.data_as(pd), b.ctypes.data_as(pd), out.ctypes.data_as(pd), a.size)
    assert rc == OK
    return out.reshape(-1, 8)


def _ulps(x: np.ndarray, y: np.ndarray) -> np.ndarray:
    """Distance in units in the last place between same-signed finite doubles."""
    assert np.all(np.signbit(x) == np.signbit(y))
    return np.abs(x.view(np.int64) - y.view(np.int64))


def test_quotient_and_root_within_one_ulp():
    rng = np.random.default_rng(20261204)
    n = 1 << 20
    a = rng.choice([-1.0, 1.0], n) * 10.0 ** rng.uniform(-30, 30, n)
    b = 10.0 ** rng.uniform(-30, 30, n)
    # mantissas at the ends of the binade, exact quotients and roots
    a[:8] = [1.0, 3.0, 2.0, 1.0 - 2 ** -53, 7.0, 1e300, -5.0, 0.0]
    b[:8] = [3.0, 3.0, 4.0, 1.0 + 2 ** -52, 1.0 - 2 ** -53, 1e-7, 2.0, 9.0]
    r = _run(a, b)
    nz = a != 0.0
    assert _ulps(r[nz, 0], r[nz, 1]).max() <= 1
    assert np.all(r[~nz, 0] == 0.0)
    assert _ulps(r[:, 2], r[:, 3]).max() <= 1
    # the exact cases come out exact
    assert r[1, 0] == 1.0 and r[2, 0] == 0.5 and r[6, 0] == -2.5 and r[7, 2] == 3.0 and r[2, 2] == 2.0


def test_solver_value_ranges_within_one_ulp():
    """Operands of the sizes the stage arithmetic divides: densities, pressures,
    viscosities, sensor sums, volumes."""
    rng = np.random.default_rng(7)
    n = 1 << 18
    a = 10.0 ** rng.uniform(-12, 8, n)
    b = 10.0 ** rng.uniform(-12, 8, n)
    r = _run(a, b)
    assert _ulps(r[:, 0], r[:, 1]).max() <= 1
    assert _ulps(r[:, 2], r[:, 3]).max() <= 1


def test_nan_propagates():
    a = np.array([np.nan, 1.0, np.nan])
    b = np.array([2.0, np.nan, np.nan])
    r = _run(a, b)
    assert np.all(np.isnan(r[:, 0]))
    assert np.isnan(r[1, 2]) and np.isnan(r[2, 2])
    assert np.isnan(r[0, 4]) and np.isnan(r[1, 6]) and np.isnan(r[2, 6])


def test_exp_within_two_ulps():
    rng = np.random.default_rng(11)
    n = 1 << 20
    a = np.concatenate([rng.uniform(-745.0, 709.0, n // 2), rng.uniform(-40.0, 40.0, n // 2)])
    a[:6] = [0.0, 1.0, -1.0, -2e8, -0.5 * np.log(2.0), 700.0]
    r = _run(a, np.ones_like(a))
    assert r[0, 4] == 1.0
    assert r[3, 4] == 0.0 and r[3, 5] == 0.0
    assert _ulps(r[:, 4], r[:, 5]).max() <= 2


def test_inverse_sixth_root_within_four_ulps():
    rng = np.random.default_rng(13)
    n = 1 << 20
    b = 10.0 ** rng.uniform(-300.0, 300.0, n)
    b[:4] = [64.0, 1.0, 2.0 ** 60, 4096.0]
    r = _run(np.ones_like(b), b)
    assert r[0, 6] == 0.5 and r[1, 6] == 1.0 and r[2, 6] == 2.0 ** -10 and r[3, 6] == 0.25
    assert _ulps(r[:, 6], r[:, 7]).max() <= 4
    special = _run(np.ones(2), np.array([np.inf, np.nan]))
    assert special[0, 6] == 0.0 and np.isnan(special[1, 6])
