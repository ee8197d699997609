"""Pin the oracle (CPU restatement of jst-rs) to the reference's golden data.

Graded cascade and tolerances of the reference's jst-rs/tests/golden.rs:11-21
(geometry 1e-14/1e-13, initial state 1e-14, single-stage terms 1e-10, state
after N steps 1e-8); ``tests/golden/*.json`` are the reference's own golden files
plus one live export of its jst-py (see tests/golden/make_golden.py).
"""

from __future__ import annotations

import numpy as np
import pytest

from conftest import cmp_field, golden_cases, load_golden

import jst_oracle as jo

CASES = golden_cases()


@pytest.fixture(params=CASES, ids=lambda p: p.stem)
def golden(request):
    doc, cfg, mesh_text = load_golden(request.param)
    s = jo.OracleSolver.from_mesh_text(cfg, mesh_text)
    yield doc, cfg, s
    s.close()


def test_golden_files_present():
    assert len(CASES) >= 3


def test_meta_agrees(golden):
    doc, cfg, s = golden
    m = doc["meta"]
    assert s.ni + 1 == m["i_total"]
    assert s.nj == m["j_total"]
    assert s.n_cells == m["n_cells"]
    for key, val in (("gamma", cfg["physics"]["gamma"]), ("R", cfg["physics"]["R"]),
                     ("CFL", cfg["simulation"]["CFL"]), ("Ma", cfg["simulation"]["Ma"]),
                     ("k2", cfg["dissipation"]["k2"]), ("k4", cfg["dissipation"]["k4"])):
        assert abs(m[key] - val) < 1e-15, key


def test_geometry_agrees(golden):
    doc, _, s = golden
    g = doc["geometry"]
    cmp_field(s.get("vol"), g["cell_vol"], "vol", 1e-14)
    cmp_field(s.get("cx"), g["cell_x"], "cx", 1e-13, 1e-15)
    cmp_field(s.get("cy"), g["cell_y"], "cy", 1e-13, 1e-15)
    cmp_field(s.get("wall_dist"), g["cell_sad"], "wall_dist", 1e-14)
    tau = s.faces(0).reshape(-1, 4)
    nrm = s.faces(1).reshape(-1, 4)
    for k, key in enumerate(("tau_nx", "tau_ny", "tau_mx", "tau_my")):
        cmp_field(tau[:, k], g[key], key, 1e-13, 1e-15)
    for k, key in enumerate(("n_nx", "n_ny", "n_mx", "n_my")):
        cmp_field(nrm[:, k], g[key], key, 1e-13, 1e-15)


def test_initial_state_agrees(golden):
    doc, _, s = golden
    ini = doc["init"]
    for key, name in (("rho", "rho"), ("p", "p"), ("T", "T"), ("u", "u"), ("v", "v"), ("E", "E"),
                      ("H", "H"), ("c", "c"), ("miubl", "nut")):
        cmp_field(s.get(name), ini[key], f"init.{key}", 1e-14, 1e-300)
    for k in range(5):
        cmp_field(s.get(f"U{k}"), ini[f"U{k + 1}"], f"init.U{k + 1}", 1e-14, 1e-300)


def test_single_stage_residual_terms_agree(golden):
    doc, _, s = golden
    t = doc["terms"]
    s.run(doc["meta"]["warmup"])
    dt = s.timestep()
    s.residual_terms()
    assert abs(dt - t["dt"]) < 1e-12 * t["dt"]
    for key, name in (("ugrad_x", "dudx"), ("ugrad_y", "dudy"), ("vgrad_x", "dvdx"), ("vgrad_y", "dvdy"),
                      ("Tgrad_x", "dtdx"), ("Tgrad_y", "dtdy"), ("miublgrad_x", "dnutdx"),
                      ("miublgrad_y", "dnutdy"), ("chi", "chi"), ("fv1", "fv1")):
        cmp_field(s.get(name), t[key], f"terms.{key}", 1e-10, 1e-280)
    for k in range(5):
        for term in ("Fc", "Fv", "Fd"):
            cmp_field(s.get(f"{term}{k}"), t[f"{term}{k + 1}"], f"terms.{term}{k + 1}", 1e-10, 1e-280)
    cmp_field(s.get("S"), t["S5"], "terms.S5", 1e-10, 1e-280)


def test_final_state_agrees(golden):
    doc, _, s = golden
    f = doc["final"]
    steps, res, total, _ = s.run(doc["meta"]["steps"])
    assert steps == f["steps"]
    assert abs(res - f["residual"]) < 1e-8 * f["residual"]
    assert abs(total - f["totaltime"]) < 1e-10 * f["totaltime"]
    for key, name in (("rho", "rho"), ("p", "p"), ("T", "T"), ("u", "u"), ("v", "v"), ("miubl", "nut")):
        cmp_field(s.get(name), f[key], f"final.{key}", 1e-8, 1e-300)


def test_final_state_tighter_than_reference_tolerance(golden):
    """The restatement tracks the golden trajectories far inside 1e-8."""
    doc, _, s = golden
    f = doc["final"]
    s.run(doc["meta"]["steps"])
    worst = max(cmp_field(s.get(n), f[k], k, 1e-8, 1e-300)
                for k, n in (("rho", "rho"), ("p", "p"), ("u", "u"), ("v", "v"), ("miubl", "nut")))
    assert worst < 1e-11, worst
