"""Shared pytest setup.

Markers: ``gpu`` — needs a CUDA device (B200); everything else runs on CPU.
"""

from __future__ import annotations

import json
import sys
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parent.parent
GOLDEN = Path(__file__).resolve().parent / "golden"
sys.path.insert(0, str(ROOT))
sys.path.insert(0, str(ROOT / "oracle"))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (sm_100a)")


def load_config(overrides: dict | None = None) -> dict:
    cfg = json.loads((GOLDEN / "config.json").read_text())
    for sec, kv in (overrides or {}).items():
        cfg.setdefault(sec, {}).update(kv)
    return cfg


def golden_files():
    return sorted(GOLDEN.glob("*.json"))


def golden_cases():
    return [p for p in golden_files() if p.name != "config.json"]


def load_golden(path: Path):
    doc = json.loads(path.read_text())
    mesh_text = (GOLDEN / doc["meta"]["mesh"]).read_text()
    cfg = load_config(doc["meta"].get("config_overrides"))
    return doc, cfg, mesh_text


def cmp_field(got, want, label, rtol, atol=0.0):
    """Field-scaled comparison of the reference's golden tests
    (jst-rs/tests/golden.rs:53-79): |got - want| <= atol + rtol * max|want|."""
    got = np.asarray(got, dtype=np.float64).ravel()
    want = np.asarray(want, dtype=np.float64).ravel()
    assert got.shape == want.shape, f"{label}: shape {got.shape} != {want.shape}"
    scale = float(np.max(np.abs(want))) if want.size else 0.0
    tol = atol + rtol * scale
    err = np.abs(got - want)
    k = int(np.argmax(err)) if err.size else 0
    assert err.size == 0 or err[k] <= tol, (
        f"{label}: mismatch at flat index {k}: got {got[k]!r}, want {want[k]!r} "
        f"(abs err {err[k]:e} > tol {tol:e}; field scale {scale:e}, rtol {rtol:e})")
    return float(err.max() / scale) if err.size and scale > 0 else 0.0


@pytest.fixture(scope="session")
def base_config():
    return load_config()


@pytest.fixture(scope="session")
def fangdata_text():
    return (GOLDEN / "fangdata.txt").read_text()
