"""Helpers shared by the GPU parity tests."""

from __future__ import annotations

import numpy as np

from conftest import GOLDEN, load_config

import jst_oracle as jo


def cylinder_case(n_rings=17, n_theta=40, mach=0.3, aoa=0.0, cfl=2.5, nut_ratio=None):
    """A cylinder O-mesh (diameter 1, far field 20, first spacing 1e-3) in the
    reference's config with the given flow conditions."""
    from purinecfd_b200 import meshgen
    xy = meshgen.cylinder_o_mesh(n_rings, n_theta, radius=0.5, r_far=20.0, first_spacing=1e-3)
    cfg = load_config({"simulation": {"Ma": mach, "AOA": aoa, "CFL": cfl}})
    if nut_ratio is not None:
        cfg["simulation"]["nut_inf_ratio"] = nut_ratio
    return cfg, xy, n_rings, n_theta


def mesh_case(name: str):
    text = (GOLDEN / name).read_text()
    nr, nt, xy = jo.parse_mesh(text)
    return xy, nr, nt


def rel_field_err(got, want) -> float:
    got = np.asarray(got, float).ravel()
    want = np.asarray(want, float).ravel()
    scale = float(np.max(np.abs(want))) or 1.0
    return float(np.max(np.abs(got - want)) / scale)


STATE_FIELDS = ["rho", "p", "T", "u", "v", "nut", "U0", "U1", "U2", "U3", "U4"]
