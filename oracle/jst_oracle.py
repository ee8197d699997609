"""ORACLE — test infrastructure only, never the product.

ctypes wrapper around ``oracle/libjst_oracle.so``, the CPU FP64 restatement of
the reference's jst-rs solver loop (see ``jst_oracle.cpp``).  Only ``tests/``,
``__graft_entry__.smoke()`` and ``bench.py``'s CPU-baseline leg import this
module; the product path never does.
"""

from __future__ import annotations

import ctypes as C
import os
import subprocess
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
LIB_PATH = HERE / "libjst_oracle.so"

# Parameter vector order (matches jst_oracle.cpp's C API comment).
PARAM_KEYS = [
    ("physics", "gamma"), ("physics", "R"), ("physics", "T0"), ("physics", "Ts"), ("physics", "mu0"),
    ("simulation", "AOA"), ("simulation", "Ma"), ("simulation", "CFL"), ("simulation", "IM"),
    ("simulation", "T"), ("simulation", "P"),
    ("solver", "iteration"), ("solver", "targetres"),
    ("spalart_allmaras", "Cv1"), ("spalart_allmaras", "Pr"), ("spalart_allmaras", "Prt"),
    ("spalart_allmaras", "sigma"), ("spalart_allmaras", "Cb1"), ("spalart_allmaras", "Cb2"),
    ("spalart_allmaras", "Ct3"), ("spalart_allmaras", "Ct4"), ("spalart_allmaras", "Cw2"),
    ("spalart_allmaras", "Cw3"), ("spalart_allmaras", "fv3"), ("spalart_allmaras", "kappa"),
    ("spalart_allmaras", "rmax"),
    ("dissipation", "k2"), ("dissipation", "k4"),
]
# solver section defaults (config.rs:130-135)
SOLVER_DEFAULTS = {"iteration": 10000, "targetres": 1e-10}

DERIVED_KEYS = ["cv", "cp", "cw1", "cv1_cubed", "c_inf", "u_inf", "v_inf", "rho_inf", "mu_inf", "nut_inf",
                "supersonic", "suth_num", "inv_t_ref", "inv_pr", "inv_prt", "inv_kappa2", "cw3_6",
                "one_plus_cw3_6"]

MESH_ERRORS = {1: "BadHeader", 2: "Empty", 3: "CountMismatch", 4: "BadPoint", 5: "TooSmall"}


def build() -> Path:
    """Compile the oracle library with its Makefile (idempotent)."""
    subprocess.run(["make", "-s", "-C", str(HERE)], check=True)
    return LIB_PATH


_lib = None


def lib():
    global _lib
    if _lib is None:
        if not LIB_PATH.exists():
            build()
        L = C.CDLL(str(LIB_PATH))
        d, i, l, vp, cp = C.c_double, C.c_int, C.c_long, C.c_void_p, C.c_char_p
        pd = C.POINTER(C.c_double)
        L.jo_new.restype = vp
        L.jo_new.argtypes = [pd, pd, i, i]
        L.jo_free.argtypes = [vp]
        L.jo_ni.argtypes = [vp]
        L.jo_nj.argtypes = [vp]
        L.jo_derived.argtypes = [vp, pd]
        L.jo_advance.argtypes = [vp]
        L.jo_nonphysical.argtypes = [vp, C.POINTER(l), C.POINTER(l), pd, pd]
        L.jo_run.argtypes = [vp, l, pd, C.POINTER(l), pd]
        L.jo_timestep.restype = d
        L.jo_timestep.argtypes = [vp]
        L.jo_residual_terms.argtypes = [vp]
        L.jo_residual.restype = d
        L.jo_residual.argtypes = [vp]
        L.jo_totaltime.restype = d
        L.jo_totaltime.argtypes = [vp]
        L.jo_step.restype = l
        L.jo_step.argtypes = [vp]
        L.jo_unpack.argtypes = [vp]
        L.jo_boundary.argtypes = [vp]
        L.jo_set_uniform.argtypes = [vp, d, d, d, d, d]
        L.jo_kernel.argtypes = [vp, cp]
        L.jo_get.argtypes = [vp, cp, pd]
        L.jo_get_halo.argtypes = [vp, cp, pd]
        L.jo_set_u.argtypes = [vp, i, pd]
        L.jo_faces.restype = l
        L.jo_faces.argtypes = [vp, i, pd]
        L.jo_wall_force.argtypes = [vp, pd, pd]
        L.jo_mesh_parse.argtypes = [cp, pd, l, C.POINTER(i), C.POINTER(i), C.POINTER(l), C.POINTER(l)]
        L.jo_set_threads.argtypes = [i]
        L.jo_max_threads.restype = i
        _lib = L
    return _lib


def _ptr(a: np.ndarray):
    return a.ctypes.data_as(C.POINTER(C.c_double))


def params_from_config(cfg: dict, *, nut_inf_ratio: float | None = None, local_dt: bool = False) -> np.ndarray:
    """Flatten a parsed config.json into the oracle's parameter vector."""
    out = []
    for sec, key in PARAM_KEYS:
        if sec == "solver":
            out.append(float(cfg.get("solver", {}).get(key, SOLVER_DEFAULTS[key])))
        else:
            out.append(float(cfg[sec][key]))
    ratio = nut_inf_ratio
    if ratio is None:
        ratio = float(cfg.get("simulation", {}).get("nut_inf_ratio", 0.1))
    out.append(ratio)
    out.append(1.0 if local_dt else 0.0)
    return np.asarray(out, dtype=np.float64)


def parse_mesh(text: str):
    """Restatement of mesh.rs:109-189.  Returns (n_rings, n_theta, xy[n_rings*n_theta, 2]).

    Raises ValueError("<MeshError variant>: ...") on malformed input."""
    L = lib()
    cap = 2 * (text.count("\n") + 2)
    xy = np.zeros(cap, dtype=np.float64)
    nr, nt = C.c_int(0), C.c_int(0)
    ea, eb = C.c_long(0), C.c_long(0)
    rc = L.jo_mesh_parse(text.encode(), _ptr(xy), cap, C.byref(nr), C.byref(nt), C.byref(ea), C.byref(eb))
    if rc != 0:
        raise ValueError(f"{MESH_ERRORS.get(rc, rc)}: {ea.value} {eb.value}")
    n = nr.value * nt.value
    return nr.value, nt.value, xy[: 2 * n].reshape(n, 2).copy()


class OracleSolver:
    """The reference's ``Solver`` (solver.rs:25-256) restated on the CPU."""

    def __init__(self, cfg: dict, xy: np.ndarray, n_rings: int, n_theta: int, *, nut_inf_ratio=None,
                 local_dt=False):
        self._L = lib()
        self.params = params_from_config(cfg, nut_inf_ratio=nut_inf_ratio, local_dt=local_dt)
        xy = np.ascontiguousarray(xy, dtype=np.float64).reshape(-1)
        assert xy.size == 2 * n_rings * n_theta
        self._h = self._L.jo_new(_ptr(self.params), _ptr(xy), n_rings, n_theta)
        self.ni = self._L.jo_ni(self._h)
        self.nj = self._L.jo_nj(self._h)
        self.halo = int(self.params[8])

    @classmethod
    def from_mesh_text(cls, cfg: dict, text: str, **kw):
        nr, nt, xy = parse_mesh(text)
        return cls(cfg, xy, nr, nt, **kw)

    def close(self):
        if getattr(self, "_h", None):
            self._L.jo_free(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @property
    def n_cells(self):
        return self.ni * self.nj

    def derived(self) -> dict:
        out = np.zeros(len(DERIVED_KEYS))
        self._L.jo_derived(self._h, _ptr(out))
        return dict(zip(DERIVED_KEYS, out.tolist()))

    def advance(self):
        if self._L.jo_advance(self._h) != 0:
            raise FloatingPointError(self._nonphysical_msg())

    def _nonphysical_msg(self):
        i, j, r, p = C.c_long(), C.c_long(), C.c_double(), C.c_double()
        self._L.jo_nonphysical(self._h, C.byref(i), C.byref(j), C.byref(r), C.byref(p))
        return f"non-physical state at cell ({i.value}, {j.value}): rho = {r.value:e}, p = {p.value:e}"

    def nonphysical(self):
        i, j, r, p = C.c_long(), C.c_long(), C.c_double(), C.c_double()
        self._L.jo_nonphysical(self._h, C.byref(i), C.byref(j), C.byref(r), C.byref(p))
        return i.value, j.value, r.value, p.value

    def run(self, max_steps: int | None = None, history: bool = False):
        """Returns (steps, residual, totaltime, converged[, history])."""
        n = -1 if max_steps is None else int(max_steps)
        cap = n if n >= 0 else int(self.params[11])
        hist = np.zeros(max(cap, 1))
        done, res = C.c_long(0), C.c_double(0)
        rc = self._L.jo_run(self._h, n, _ptr(hist), C.byref(done), C.byref(res))
        if rc != 0:
            raise FloatingPointError(self._nonphysical_msg())
        out = (done.value, res.value, self.totaltime, res.value < self.params[12])
        return out + (hist[: done.value].copy(),) if history else out

    def timestep(self) -> float:
        return self._L.jo_timestep(self._h)

    def residual_terms(self):
        self._L.jo_residual_terms(self._h)

    def residual(self) -> float:
        return self._L.jo_residual(self._h)

    def unpack(self) -> bool:
        return self._L.jo_unpack(self._h) == 0

    def boundary(self):
        self._L.jo_boundary(self._h)

    def kernel(self, name: str):
        self._L.jo_kernel(self._h, name.encode())

    def set_uniform(self, rho, vx, vy, p, nut):
        self._L.jo_set_uniform(self._h, rho, vx, vy, p, nut)

    @property
    def totaltime(self) -> float:
        return self._L.jo_totaltime(self._h)

    @property
    def step(self) -> int:
        return self._L.jo_step(self._h)

    def get(self, name: str) -> np.ndarray:
        out = np.zeros(self.ni * self.nj)
        if self._L.jo_get(self._h, name.encode(), _ptr(out)) != 0:
            raise KeyError(name)
        return out.reshape(self.ni, self.nj)

    def get_halo(self, name: str) -> np.ndarray:
        h = self.halo
        out = np.zeros((self.ni + 2 * h) * (self.nj + 2 * h))
        if self._L.jo_get_halo(self._h, name.encode(), _ptr(out)) != 0:
            raise KeyError(name)
        return out.reshape(self.ni + 2 * h, self.nj + 2 * h)

    def set_u(self, k: int, arr: np.ndarray):
        a = np.ascontiguousarray(arr, dtype=np.float64).reshape(-1)
        self._L.jo_set_u(self._h, k, _ptr(a))

    def faces(self, which: int) -> np.ndarray:
        n_t = (self.ni + 1) * self.nj
        out = np.zeros(max(n_t, self.ni * self.nj) * 5)
        n = self._L.jo_faces(self._h, which, _ptr(out))
        return out[:n].copy()

    def wall_force(self):
        fx, fy = C.c_double(), C.c_double()
        self._L.jo_wall_force(self._h, C.byref(fx), C.byref(fy))
        return fx.value, fy.value


def set_threads(n: int):
    lib().jo_set_threads(int(n))


def max_threads() -> int:
    return lib().jo_max_threads()


def default_threads() -> int:
    return os.cpu_count() or 1
