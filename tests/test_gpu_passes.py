"""Parity of the strict FP64 passes path (one kernel per reference pass) with
the oracle and with the reference's golden data, through the C ABI."""

from __future__ import annotations

import numpy as np
import pytest

from conftest import cmp_field, golden_cases, load_config, load_golden
from gpu_common import STATE_FIELDS, cylinder_case, mesh_case, rel_field_err

import jst_oracle as jo

pytestmark = pytest.mark.gpu


def _solver(cfg, xy, nr, nt, **kw):
    from purinecfd_b200 import PATH_PASSES, Solver
    return Solver(cfg, xy, nr, nt, kernel_path=PATH_PASSES, **kw)


@pytest.fixture(params=golden_cases(), ids=lambda p: p.stem)
def golden(request):
    doc, cfg, mesh_text = load_golden(request.param)
    nr, nt, xy = jo.parse_mesh(mesh_text)
    s = _solver(cfg, xy, nr, nt)
    o = jo.OracleSolver(cfg, xy, nr, nt)
    yield doc, s, o
    s.close()
    o.close()


def test_geometry_bit_exact(golden):
    _, s, o = golden
    for name in ("vol", "cx", "cy", "wall_dist"):
        assert np.array_equal(s.get(name), o.get(name)), name
    for which in (0, 1):
        assert np.array_equal(s.faces(which).ravel(), o.faces(which)), which


@pytest.mark.parametrize("mesh", ["naca_129x256", "naca_257x512", "ellipse_29x70", "cylinder_65x300"])
def test_wall_distance_bit_exact_on_larger_meshes(mesh):
    """The GPU wall distance (a shared-memory window per block, one square
    root per cell) equals the reference's per-face search bit for bit, on
    rings wider and narrower than a block and with windows up to nj/5."""
    from purinecfd_b200 import Solver, meshgen
    kind, size = mesh.split("_")
    nr, nt = map(int, size.split("x"))
    if kind == "naca":
        xy = meshgen.naca4_o_mesh(nr, nt, 0.02, 0.4, 0.12, first_spacing=1e-6)
    elif kind == "ellipse":
        xy = meshgen.ellipse_o_mesh(nr, nt, stretch=1.1)
    else:
        xy = meshgen.cylinder_o_mesh(nr, nt, radius=0.5, r_far=20.0, first_spacing=1e-3)
    cfg = load_config()
    s = Solver(cfg, xy, nr, nt)
    o = jo.OracleSolver(cfg, xy, nr, nt)
    assert np.array_equal(s.get("wall_dist"), o.get("wall_dist"))


def test_initial_state_bit_exact(golden):
    _, s, o = golden
    for name in ("rho", "p", "T", "u", "v", "E", "H", "c", "nut", "U0", "U1", "U2", "U3", "U4"):
        assert np.array_equal(s.get(name), o.get(name)), name


def test_single_stage_terms_match_golden_and_oracle(golden):
    doc, s, o = golden
    t = doc["terms"]
    s.run(doc["meta"]["warmup"])
    o.run(doc["meta"]["warmup"])
    dt = s.residual_terms(with_timestep=True)
    dto = o.timestep()
    o.residual_terms()
    assert abs(dt - t["dt"]) < 1e-12 * t["dt"]
    assert abs(dt - dto) <= 1e-15 * dto
    names = {"ugrad_x": "dudx", "ugrad_y": "dudy", "vgrad_x": "dvdx", "vgrad_y": "dvdy", "Tgrad_x": "dtdx",
             "Tgrad_y": "dtdy", "miublgrad_x": "dnutdx", "miublgrad_y": "dnutdy", "chi": "chi", "fv1": "fv1",
             "S5": "S"}
    for k in range(5):
        for term in ("Fc", "Fv", "Fd"):
            names[f"{term}{k + 1}"] = f"{term}{k}"
    worst = 0.0
    for gkey, name in names.items():
        got = s.get(name)
        cmp_field(got, t[gkey], gkey, 1e-10, 1e-280)
        worst = max(worst, rel_field_err(got, o.get(name)))
    # Same arithmetic as the oracle; only libm vs CUDA exp/cbrt/pow/hypot differ.
    assert worst < 1e-12, worst


def test_final_state_matches_golden(golden):
    doc, s, o = golden
    f = doc["final"]
    rep = s.run(doc["meta"]["steps"])
    assert rep.steps == f["steps"]
    assert abs(rep.residual - f["residual"]) < 1e-8 * f["residual"]
    assert abs(rep.totaltime - f["totaltime"]) < 1e-10 * f["totaltime"]
    for key, name in (("rho", "rho"), ("p", "p"), ("T", "T"), ("u", "u"), ("v", "v"), ("miubl", "nut")):
        cmp_field(s.get(name), f[key], key, 1e-8, 1e-300)


def test_trajectory_100_steps_matches_oracle():
    """Cylinder O-mesh 40 x 17 (diameter 1, far field 20, first spacing 1e-3),
    M = 0.3, CFL 2.5: the strict path follows the oracle within 1e-10 per
    field (north-star criterion) over the first 100 iterations."""
    cfg, xy, nr, nt = cylinder_case()
    s = _solver(cfg, xy, nr, nt)
    o = jo.OracleSolver(cfg, xy, nr, nt)
    hist_s = []
    rep = s.run(100, lambda k, r: hist_s.append(r))
    _, _, _, _, hist_o = o.run(100, history=True)
    assert rep.steps == 100
    np.testing.assert_allclose(hist_s, hist_o, rtol=1e-8)
    for name in STATE_FIELDS:
        assert rel_field_err(s.get(name), o.get(name)) < 1e-10, name
    assert abs(s.totaltime - o.totaltime) <= 1e-12 * o.totaltime


def test_nonphysical_is_reported_not_fatal():
    """solver.rs:358-365: a negative density is reported as NonPhysical."""
    from purinecfd_b200 import NonPhysical
    xy, nr, nt = mesh_case("fangdata.txt")
    from conftest import load_config
    s = _solver(load_config(), xy, nr, nt)
    u = np.stack([s.get(f"U{k}") for k in range(5)])
    u[0, 2, 5] = -1.0
    with pytest.raises(NonPhysical) as ei:
        s.set_conserved(u)
    assert (ei.value.i, ei.value.j) == (2, 5)
    assert ei.value.rho == -1.0


def test_blowup_reports_nonphysical_like_oracle():
    """properties.rs:204-221: CFL 200 must end in NonPhysical, not NaN (the
    oracle blows up too; the exact cell is chaotic and not compared)."""
    from purinecfd_b200 import NonPhysical
    from purinecfd_b200 import meshgen
    from conftest import load_config
    xy = meshgen.ellipse_o_mesh(13, 40)
    cfg = load_config({"simulation": {"CFL": 200.0}})
    s = _solver(cfg, xy, 13, 40)
    o = jo.OracleSolver(cfg, xy, 13, 40)
    with pytest.raises(NonPhysical) as ei:
        s.run(400)
    with pytest.raises(FloatingPointError):
        o.run(400)
    e = ei.value
    assert 0 <= e.i < s.ni and 0 <= e.j < s.nj
    assert np.isnan(e.rho) or e.rho <= 1e-15 or np.isnan(e.p) or e.p <= 1e-15
