"""Cross-module properties of the scheme (jst-rs/tests/properties.rs:82-157),
checked on the oracle: discrete mass conservation, no mass through the wall,
free-stream preservation of the whole residual chain.  The same properties
are checked on the CUDA paths in test_gpu_properties.py."""

from __future__ import annotations

import numpy as np

from conftest import load_config

import jst_oracle as jo


def _mesh(rings, nj, stretch):
    from purinecfd_b200 import meshgen
    return meshgen.ellipse_o_mesh(rings, nj, stretch=stretch)  # properties.rs:14-38 family


def test_discrete_mass_conservation_and_no_wall_flux():
    """properties.rs:82-122: interior face fluxes cancel pairwise, so the sum
    of the cells' convective mass residuals equals the far-field minus the
    wall face fluxes, and the wall mirror makes the wall flux vanish."""
    o = jo.OracleSolver(load_config(), _mesh(17, 48, 1.1), 17, 48)
    o.run(30)
    o.timestep()
    o.residual_terms()
    ni, nj = o.ni, o.nj
    tflux = o.faces(2).reshape(ni + 1, nj, 5)
    fc = o.get("Fc0")
    cells_total = fc.sum()
    boundary = (tflux[ni, :, 0] - tflux[0, :, 0]).sum()
    scale = max(np.abs(fc).max(), 1.0)
    assert abs(cells_total - boundary) < 1e-10 * scale
    wall_scale = max(np.abs(tflux[1, :, 0]).max(), 1.0)
    assert np.all(np.abs(tflux[0, :, 0]) < 1e-10 * wall_scale)


def test_free_stream_preserved_end_to_end():
    """properties.rs:126-157: a uniform state (ghosts included) gives a zero
    mean-flow residual Fc - Fv - Fd to machine precision."""
    o = jo.OracleSolver(load_config(), _mesh(13, 40, 1.0), 13, 40)
    o.set_uniform(1.176, 69.4, 17.3, 101_325.0, 1.5e-4)
    o.timestep()
    for k in ("convection", "gradient", "viscous", "dissipation"):
        o.kernel(k)
    scale = np.abs(o.faces(2)).max()
    for k in range(4):
        r = o.get(f"Fc{k}") - o.get(f"Fv{k}") - o.get(f"Fd{k}")
        assert np.abs(r).max() < 1e-13 * scale, k


def test_timestep_shrinks_with_mesh_refinement():
    """properties.rs:224-233."""
    coarse = jo.OracleSolver(load_config(), _mesh(9, 32, 1.0), 9, 32).timestep()
    fine = jo.OracleSolver(load_config(), _mesh(17, 64, 1.0), 17, 64).timestep()
    assert 0.2 * coarse < fine < coarse
