"""Parity of the fused tiled path (one kernel per RK stage) with the oracle,
through the C ABI: FP64 within 1e-10 over 100 iterations (the north-star
criterion), FP32-split within its stated tolerance, bitwise tile-shape
invariance and run-to-run determinism."""

from __future__ import annotations

import numpy as np
import pytest

from conftest import cmp_field, golden_cases, load_config, load_golden
from gpu_common import STATE_FIELDS, cylinder_case, mesh_case, rel_field_err

import jst_oracle as jo

pytestmark = pytest.mark.gpu


def _solver(cfg, xy, nr, nt, **kw):
    from purinecfd_b200 import PATH_FUSED, Solver
    return Solver(cfg, xy, nr, nt, kernel_path=PATH_FUSED, **kw)


@pytest.mark.parametrize("case", golden_cases(), ids=lambda p: p.stem)
def test_fused_fp64_final_state_matches_golden(case):
    doc, cfg, mesh_text = load_golden(case)
    nr, nt, xy = jo.parse_mesh(mesh_text)
    s = _solver(cfg, xy, nr, nt)
    f = doc["final"]
    rep = s.run(doc["meta"]["steps"])
    assert rep.steps == f["steps"]
    assert abs(rep.residual - f["residual"]) < 1e-8 * f["residual"]
    assert abs(rep.totaltime - f["totaltime"]) < 1e-10 * f["totaltime"]
    for key, name in (("rho", "rho"), ("p", "p"), ("T", "T"), ("u", "u"), ("v", "v"), ("miubl", "nut")):
        cmp_field(s.get(name), f[key], key, 1e-8, 1e-300)


def test_fused_fp64_trajectory_100_steps_within_1e10():
    """Config-1 geometry: cylinder 40 x 17 nodes, D = 1, far field 20, first
    spacing 1e-3, M = 0.3, CFL 2.5."""
    cfg, xy, nr, nt = cylinder_case()
    s = _solver(cfg, xy, nr, nt)
    o = jo.OracleSolver(cfg, xy, nr, nt)
    hist = []
    rep = s.run(100, lambda k, r: hist.append(r))
    _, _, _, _, hist_o = o.run(100, history=True)
    assert rep.steps == 100 and len(hist) == 100
    np.testing.assert_allclose(hist, hist_o, rtol=1e-9)
    for name in STATE_FIELDS:
        assert rel_field_err(s.get(name), o.get(name)) < 1e-10, name
    assert abs(s.totaltime - o.totaltime) <= 1e-12 * o.totaltime


def test_fused_fp64_local_timestep_matches_oracle():
    from purinecfd_b200 import DT_LOCAL
    xy, nr, nt = mesh_case("ell_13x40.txt")
    cfg = load_config({"simulation": {"AOA": 3.0, "Ma": 0.4}})
    s = _solver(cfg, xy, nr, nt, dt_mode=DT_LOCAL)
    o = jo.OracleSolver(cfg, xy, nr, nt, local_dt=True)
    s.run(50)
    o.run(50)
    for name in STATE_FIELDS:
        assert rel_field_err(s.get(name), o.get(name)) < 1e-10, name


@pytest.mark.parametrize("tile", [(16, 32), (8, 64), (4, 64)])
def test_fused_tile_shape_invariance_bitwise(tile):
    """Every face flux and cell update is computed from the same inputs with
    the same operations whatever the tiling, so U is bitwise identical."""
    from purinecfd_b200 import meshgen
    xy = meshgen.ellipse_o_mesh(29, 70, stretch=1.1)
    cfg = load_config({"simulation": {"AOA": 5.0, "Ma": 0.5}})
    a = _solver(cfg, xy, 29, 70, tile_i=8, tile_j=32)
    b = _solver(cfg, xy, 29, 70, tile_i=tile[0], tile_j=tile[1])
    a.run(20)
    b.run(20)
    for k in range(5):
        assert np.array_equal(a.get(f"U{k}"), b.get(f"U{k}")), k


@pytest.mark.parametrize("cfgt", [(4, 32, 256), (8, 32, 128), (8, 32, 192), (16, 32, 384), (8, 64, 256),
                                  (16, 26, 128), (32, 26, 128), (64, 26, 128), (32, 26, 256), (32, 26, 64),
                                  (11, 26, 64), (48, 26, 64)],
                         ids=lambda t: "x".join(map(str, t)))
def test_fused_every_compiled_configuration_matches_oracle(cfgt):
    """Every tile shape and block size the autotuner may pick (block sizes
    that are not powers of two included, and the marching strips of 26
    columns) reproduces the oracle's residual history, global time step and
    fields."""
    cfg, xy, nr, nt = cylinder_case(33, 64)
    s = _solver(cfg, xy, nr, nt, tile_i=cfgt[0], tile_j=cfgt[1], block_threads=cfgt[2])
    o = jo.OracleSolver(cfg, xy, nr, nt)
    hist = []
    s.run(30, lambda k, r: hist.append(r))
    _, _, _, _, hist_o = o.run(30, history=True)
    np.testing.assert_allclose(hist, hist_o, rtol=1e-10)
    assert abs(s.totaltime - o.totaltime) <= 1e-12 * o.totaltime
    for name in STATE_FIELDS:
        assert rel_field_err(s.get(name), o.get(name)) < 1e-10, name


def test_fused_run_to_run_bitwise():
    cfg, xy, nr, nt = cylinder_case(33, 64)
    runs = []
    for _ in range(2):
        s = _solver(cfg, xy, nr, nt)
        rep = s.run(30)
        runs.append((rep.residual, s.totaltime, [s.get(f"U{k}") for k in range(5)]))
    assert runs[0][0] == runs[1][0] and runs[0][1] == runs[1][1]
    for k in range(5):
        assert np.array_equal(runs[0][2][k], runs[1][2][k])


def test_fused_fp32_split_tracks_oracle():
    """FP32 fluxes/gradients/SA with the FP64 accumulator: after 100 steps the
    fields stay within 1e-5 of the FP64 oracle (field-scaled)."""
    from purinecfd_b200 import PREC_FP32_SPLIT
    cfg, xy, nr, nt = cylinder_case()
    s = _solver(cfg, xy, nr, nt, precision=PREC_FP32_SPLIT)
    o = jo.OracleSolver(cfg, xy, nr, nt)
    s.run(100)
    o.run(100)
    for name in STATE_FIELDS:
        assert rel_field_err(s.get(name), o.get(name)) < 1e-5, name


def test_fused_nonphysical_reported():
    from purinecfd_b200 import NonPhysical, meshgen
    xy = meshgen.ellipse_o_mesh(13, 40)
    cfg = load_config({"simulation": {"CFL": 200.0}})
    s = _solver(cfg, xy, 13, 40)
    with pytest.raises(NonPhysical) as ei:
        s.run(400)
    e = ei.value
    assert 0 <= e.i < s.ni and 0 <= e.j < s.nj
    assert np.isnan(e.rho) or e.rho <= 1e-15 or np.isnan(e.p) or e.p <= 1e-15


def test_fused_set_conserved_nonphysical():
    from purinecfd_b200 import NonPhysical
    xy, nr, nt = mesh_case("fangdata.txt")
    s = _solver(load_config(), xy, nr, nt)
    u = np.stack([s.get(f"U{k}") for k in range(5)])
    u[0, 3, 7] = -2.0
    with pytest.raises(NonPhysical) as ei:
        s.set_conserved(u)
    assert (ei.value.i, ei.value.j, ei.value.rho) == (3, 7, -2.0)


@pytest.mark.parametrize("path", ["strips", "tiles", "passes"])
@pytest.mark.parametrize("case", [("fangdata", 20.0), ("ellipse", 50.0)], ids=lambda c: f"{c[0]}-cfl{c[1]:g}")
def test_first_failed_cell_matches_oracle(path, case):
    """At a CFL where the first step already fails, the reported cell is the
    oracle's: the first failing cell in row-major order of the first stage with
    one (solver.rs:160-171) — (0, 5) on fangdata at CFL 20, not (0, 0) — with
    its density and pressure."""
    from purinecfd_b200 import PATH_PASSES, NonPhysical, Solver, meshgen
    name, cfl = case
    if name == "fangdata":
        xy, nr, nt = mesh_case("fangdata.txt")
    else:
        nr, nt = 13, 40
        xy = meshgen.ellipse_o_mesh(nr, nt)
    cfg = load_config({"simulation": {"CFL": cfl}})
    o = jo.OracleSolver(cfg, xy, nr, nt)
    with pytest.raises(FloatingPointError):
        o.advance()
    oi, oj, orho, op = o.nonphysical()
    kw = {"strips": dict(tile_i=8, tile_j=26, block_threads=64), "tiles": dict(tile_i=8, tile_j=32, block_threads=256)}
    s = Solver(cfg, xy, nr, nt, kernel_path=PATH_PASSES) if path == "passes" else _solver(cfg, xy, nr, nt, **kw[path])
    with pytest.raises(NonPhysical) as ei:
        s.advance()
    e = ei.value
    assert (e.i, e.j) == (oi, oj)
    assert abs(e.rho - orho) <= 1e-8 * abs(orho)
    assert (np.isnan(e.p) and np.isnan(op)) or abs(e.p - op) <= 1e-6 * abs(op)


def test_forces_agree_across_paths_and_oracle():
    """CL/CD (no counterpart in the reference) from the fused path, the passes
    path and the oracle's wall-force integrator agree on the same state."""
    from purinecfd_b200 import PATH_PASSES, Solver, meshgen
    xy = meshgen.naca4_o_mesh(33, 64, first_spacing=1e-3)
    cfg = load_config({"simulation": {"AOA": 4.0, "Ma": 0.4}})
    f = _solver(cfg, xy, 33, 64)
    p = Solver(cfg, xy, 33, 64, kernel_path=PATH_PASSES)
    o = jo.OracleSolver(cfg, xy, 33, 64)
    f.run(40)
    p.run(40)
    o.run(40)
    o.residual_terms()
    fx, fy = o.wall_force()
    a = np.deg2rad(4.0)
    d = o.derived()
    q = 0.5 * d["rho_inf"] * (d["u_inf"] ** 2 + d["v_inf"] ** 2) * (xy[:64, 0].max() - xy[:64, 0].min())
    cd_o = (fx * np.cos(a) + fy * np.sin(a)) / q
    cl_o = (-fx * np.sin(a) + fy * np.cos(a)) / q
    cl_f, cd_f = f.forces()
    cl_p, cd_p = p.forces()
    assert abs(cl_p - cl_o) < 1e-10 * max(1.0, abs(cl_o)) and abs(cd_p - cd_o) < 1e-10 * max(1.0, abs(cd_o))
    assert abs(cl_f - cl_o) < 1e-9 * max(1.0, abs(cl_o)) and abs(cd_f - cd_o) < 1e-9 * max(1.0, abs(cd_o))
