"""Synthetic inputs with the shapes, sizes and flow conditions of the
benchmark configurations (all generated here; no dataset is involved).

Each workload returns (config dict, nodes[n_rings*n_theta, 2], n_rings,
n_theta).  The configuration starts from the reference's sample config.json
values; Reynolds numbers are reached by scaling `physics.mu0` (the reference
has no Re field, Re follows from mu0, T, P, Ma and the chord), and the
free-stream nu-tilde ratio is the optional `simulation.nut_inf_ratio` key.
"""

from __future__ import annotations

import copy
import math

import numpy as np

from . import meshgen

# The reference's sample configuration (config.json of PurineCFD).
BASE_CONFIG = {
    "physics": {"gamma": 1.4, "R": 287.06, "T0": 288.16, "Ts": 110, "mu0": 1.7894e-05, "P0": 101325.0,
                "c0": 340.28},
    "simulation": {"AOA": 0, "Ma": 0.2, "CFL": 0.8, "IM": 3, "T": 300, "P": 101325.0},
    "solver": {"iteration": 10000, "targetres": 1e-10},
    "spalart_allmaras": {"Cv1": 7.1, "Pr": 0.71, "Prt": 0.9, "sigma": 1.5, "Cb1": 0.1355, "Cb2": 0.622,
                         "Ct3": 1.2, "Ct4": 0.5, "Cw2": 0.3, "Cw3": 2.0, "fv3": 1.0, "kappa": 0.41, "rmax": 10},
    "dissipation": {"k2": 0.5, "k4": 0.0078125},
}


def sutherland(mu0, t, t_ref, t_suth):
    r = t / t_ref
    return mu0 * (r * math.sqrt(r)) * (t_ref + t_suth) / (t + t_suth)


def flow_config(mach: float, aoa: float, reynolds: float | None = None, chord: float = 1.0, cfl: float | None = None,
                nut_ratio: float | None = None, pr: float | None = None, k4: float | None = None,
                iterations: int | None = None, base: dict | None = None) -> dict:
    """A config.json dict for the given free stream.  Re is per `chord`."""
    cfg = copy.deepcopy(base or BASE_CONFIG)
    s, p = cfg["simulation"], cfg["physics"]
    s["Ma"], s["AOA"] = float(mach), float(aoa)
    if cfl is not None:
        s["CFL"] = float(cfl)
    if nut_ratio is not None:
        s["nut_inf_ratio"] = float(nut_ratio)
    if chord != 1.0:
        s["chord"] = float(chord)
    if pr is not None:
        cfg["spalart_allmaras"]["Pr"] = float(pr)
    if k4 is not None:
        cfg["dissipation"]["k4"] = float(k4)
    if iterations is not None:
        cfg["solver"]["iteration"] = int(iterations)
    if reynolds is not None:
        gamma, r_gas, t_inf, p_inf = p["gamma"], p["R"], s["T"], s["P"]
        rho = p_inf / (r_gas * t_inf)
        v = mach * math.sqrt(gamma * r_gas * t_inf)
        mu_target = rho * v * chord / reynolds
        mu_now = sutherland(p["mu0"], t_inf, p["T0"], p["Ts"])
        p["mu0"] = p["mu0"] * mu_target / mu_now
    return cfg


def reynolds_of(cfg: dict, chord: float = 1.0) -> float:
    p, s = cfg["physics"], cfg["simulation"]
    rho = s["P"] / (p["R"] * s["T"])
    v = s["Ma"] * math.sqrt(p["gamma"] * p["R"] * s["T"])
    return rho * v * chord / sutherland(p["mu0"], s["T"], p["T0"], p["Ts"])


def cylinder_40x17():
    """Circular cylinder O-mesh, 40 circumferential x 17 radial nodes, D = 1,
    far field 20, first spacing 1e-3; M 0.3, alpha 0, Re 1e5 per diameter,
    nu-tilde = 3 nu, Pr 0.72, CFL 2.5, k4 = 1/64."""
    cfg = flow_config(0.3, 0.0, 1e5, cfl=2.5, nut_ratio=3.0, pr=0.72, k4=1.0 / 64.0, iterations=2000)
    return cfg, meshgen.cylinder_o_mesh(17, 40, radius=0.5, r_far=20.0, first_spacing=1e-3), 17, 40


def naca0012_257x129():
    """NACA0012, 257 x 129 nodes closed ring (256 x 128 cells), far field 30c,
    wall spacing 1e-6c; M 0.75, alpha 2 deg, Re 6e6."""
    cfg = flow_config(0.75, 2.0, 6e6, iterations=5000)
    return cfg, meshgen.naca4_o_mesh(129, 256, 0.0, 0.4, 0.12, r_far=30.0, first_spacing=1e-6), 129, 256


def naca0012_4097x1025():
    """NACA0012, 4097 x 1025 nodes closed ring (4096 x 1024 = 4,194,304
    cells), far field 30c, wall spacing 1e-6c; M 0.8, alpha 1.25 deg, Re 1e7."""
    cfg = flow_config(0.8, 1.25, 1e7, iterations=500)
    return cfg, meshgen.naca4_o_mesh(1025, 4096, 0.0, 0.4, 0.12, r_far=30.0, first_spacing=1e-6), 1025, 4096


WORKLOADS = {
    "cylinder_40x17": cylinder_40x17,
    "naca0012_257x129": naca0012_257x129,
    "naca0012_4097x1025": naca0012_4097x1025,
}


# Batch/serving draws (config 4): mesh class, NACA 4-digit shape and flow
# conditions per instance from PCG64(seed, stream k).
MESH_CLASSES = [(65, 128), (129, 256), (257, 512)]  # (n_rings, n_theta): 129x65, 257x129, 513x257 nodes closed


def batch_instance(seed: int, k: int):
    rng = np.random.Generator(np.random.PCG64([seed, k]))
    cls = MESH_CLASSES[int(rng.integers(0, 3))]
    t = rng.uniform(0.08, 0.18)
    m = rng.uniform(0.0, 0.04)
    p = rng.uniform(0.3, 0.5)
    mach = rng.uniform(0.3, 0.8)
    aoa = rng.uniform(-4.0, 8.0)
    re = 10.0 ** rng.uniform(6.0, 7.0)
    nr, nt = cls
    cfg = flow_config(mach, aoa, re)
    xy = meshgen.naca4_o_mesh(nr, nt, m, p, t, r_far=30.0, first_spacing=1e-6)
    return cfg, xy, nr, nt, dict(thickness=t, camber=m, camber_pos=p, mach=mach, aoa=aoa, re=re)
