"""Python binding of the C ABI (include/jst_gpu.h) — the reference's ``Solver``
(jst-rs/src/solver.rs:25-256) on a B200.

    from purinecfd_b200 import Solver
    s = Solver.from_paths("config.json", "fangdata.txt")
    report = s.run(1000, lambda step, res: None)

The CUDA library is required: importing works without it, but constructing a
solver raises ``RuntimeError`` when ``libjst_gpu.so`` is missing or no CUDA
device is present.  There is no CPU fallback.
"""

from __future__ import annotations

import ctypes as C
import json
from dataclasses import dataclass
from pathlib import Path

import numpy as np

PKG = Path(__file__).resolve().parent
LIB_PATH = PKG / "libjst_gpu.so"

# jst_status
OK, ERR_MESH_IO, ERR_MESH_BAD_HEADER, ERR_MESH_EMPTY, ERR_MESH_COUNT_MISMATCH, ERR_MESH_BAD_POINT, \
    ERR_MESH_TOO_SMALL, ERR_CONFIG, ERR_NONPHYSICAL, ERR_CUDA, ERR_TIMEOUT, ERR_OOM, ERR_ARG = range(13)
STATUS_NAMES = ["OK", "MESH_IO", "MESH_BAD_HEADER", "MESH_EMPTY", "MESH_COUNT_MISMATCH", "MESH_BAD_POINT",
                "MESH_TOO_SMALL", "CONFIG", "NONPHYSICAL", "CUDA", "TIMEOUT", "OOM", "ARG"]

PREC_FP64, PREC_FP32_SPLIT = 0, 1
DT_GLOBAL, DT_LOCAL = 0, 1
PATH_FUSED, PATH_PASSES = 0, 1
STAGING_AUTO, STAGING_PER_LANE, STAGING_BULK = 0, 1, 2

FIELDS = (["rho", "p", "T", "u", "v", "E", "H", "c", "nut"] + [f"U{k}" for k in range(5)] +
          [f"Fc{k}" for k in range(5)] + [f"Fv{k}" for k in range(5)] + [f"Fd{k}" for k in range(5)] +
          ["S", "dudx", "dudy", "dvdx", "dvdy", "dtdx", "dtdy", "dnutdx", "dnutdy", "chi", "fv1", "localdt",
           "vol", "cx", "cy", "wall_dist"])
FIELD_ID = {n: k for k, n in enumerate(FIELDS)}

# C ABI symbols declared in include/jst_gpu.h (checked by the CPU test suite).
EXPORTS = ["jst_default_opts", "jst_create_from_paths", "jst_create", "jst_destroy", "jst_last_error", "jst_ni",
           "jst_nj", "jst_advance", "jst_run", "jst_residual_terms", "jst_timestep", "jst_residual",
           "jst_totaltime", "jst_step_count", "jst_get_field", "jst_get_faces", "jst_set_conserved",
           "jst_forces", "jst_write_csv", "jst_version", "jst_time_steps", "jst_residual_noalloc", "jst_kernel_config",
           "jst_checkpoint_save", "jst_checkpoint_load", "jst_stage_residual", "jst_kernel_staging"]
# test hooks declared in include/jst_gpu_debug.h
DEBUG_EXPORTS = ["jst_debug_set_uniform", "jst_debug_kernel", "jst_debug_quick_arith", "jst_debug_staging_extra_tx"]


class Opts(C.Structure):
    _fields_ = [("precision", C.c_int), ("dt_mode", C.c_int), ("kernel_path", C.c_int), ("device", C.c_int),
                ("tile_i", C.c_int), ("tile_j", C.c_int), ("use_graph", C.c_int), ("nut_inf_ratio", C.c_double),
                ("block_threads", C.c_int), ("staging", C.c_int)]


class NonPhysicalC(C.Structure):
    _fields_ = [("i", C.c_int64), ("j", C.c_int64), ("rho", C.c_double), ("p", C.c_double)]


class RunReportC(C.Structure):
    _fields_ = [("steps", C.c_int64), ("residual", C.c_double), ("totaltime", C.c_double), ("converged", C.c_int)]


STEP_CB = C.CFUNCTYPE(None, C.c_void_p, C.c_uint64, C.c_double)


class JstError(RuntimeError):
    def __init__(self, status: int, msg: str):
        self.status = status
        name = STATUS_NAMES[status] if 0 <= status < len(STATUS_NAMES) else str(status)
        super().__init__(f"{name}: {msg}")


class NonPhysical(JstError):
    """state.rs:242-257: raised instead of producing NaNs."""

    def __init__(self, i, j, rho, p):
        self.i, self.j, self.rho, self.p = i, j, rho, p
        super().__init__(ERR_NONPHYSICAL, f"non-physical state at cell ({i}, {j}): rho = {rho:e}, p = {p:e}")


@dataclass
class RunReport:
    steps: int
    residual: float
    totaltime: float
    converged: bool


_lib = None


def lib() -> C.CDLL:
    """Load libjst_gpu.so (raises if it has not been built)."""
    global _lib
    if _lib is None:
        if not LIB_PATH.exists():
            raise RuntimeError(f"{LIB_PATH} is missing: build it with `python -m purinecfd_b200.build`")
        L = C.CDLL(str(LIB_PATH))
        vp, i, d, sz = C.c_void_p, C.c_int, C.c_double, C.c_size_t
        pd = C.POINTER(C.c_double)
        L.jst_default_opts.argtypes = [C.POINTER(Opts)]
        L.jst_create.argtypes = [C.c_char_p, pd, i, i, C.POINTER(Opts), C.POINTER(vp)]
        L.jst_create_from_paths.argtypes = [C.c_char_p, C.c_char_p, C.POINTER(Opts), C.POINTER(vp)]
        L.jst_destroy.argtypes = [vp]
        L.jst_last_error.argtypes = [vp]
        L.jst_last_error.restype = C.c_char_p
        L.jst_ni.argtypes = [vp]
        L.jst_nj.argtypes = [vp]
        L.jst_advance.argtypes = [vp, C.POINTER(NonPhysicalC)]
        L.jst_run.argtypes = [vp, C.c_int64, STEP_CB, vp, C.POINTER(RunReportC), C.POINTER(NonPhysicalC)]
        L.jst_residual_terms.argtypes = [vp, pd]
        L.jst_stage_residual.argtypes = [vp, pd, sz]
        L.jst_timestep.argtypes = [vp, pd]
        L.jst_residual.argtypes = [vp, pd]
        L.jst_totaltime.argtypes = [vp, pd]
        L.jst_step_count.argtypes = [vp, C.POINTER(C.c_int64)]
        L.jst_get_field.argtypes = [vp, i, pd, sz]
        L.jst_get_faces.argtypes = [vp, i, pd, sz]
        L.jst_set_conserved.argtypes = [vp, pd, sz, C.POINTER(NonPhysicalC)]
        L.jst_forces.argtypes = [vp, pd, pd]
        L.jst_write_csv.argtypes = [vp, C.c_char_p]
        L.jst_checkpoint_save.argtypes = [vp, C.c_char_p]
        L.jst_checkpoint_load.argtypes = [vp, C.c_char_p, C.POINTER(NonPhysicalC)]
        L.jst_version.restype = C.c_char_p
        L.jst_time_steps.argtypes = [vp, i, pd, pd]
        L.jst_residual_noalloc.argtypes = [vp, vp, i, i, vp, vp]
        L.jst_kernel_config.argtypes = [vp, C.POINTER(i), C.POINTER(i), C.POINTER(i)]
        L.jst_kernel_staging.argtypes = [vp, C.POINTER(i)]
        L.jst_debug_staging_extra_tx.argtypes = [vp, i]
        L.jst_debug_set_uniform.argtypes = [vp, d, d, d, d, d]
        L.jst_debug_kernel.argtypes = [vp, C.c_char_p]
        L.jst_debug_quick_arith.argtypes = [pd, pd, pd, sz]
        _lib = L
    return _lib


def _ptr(a: np.ndarray):
    return a.ctypes.data_as(C.POINTER(C.c_double))


def make_opts(precision=PREC_FP64, dt_mode=DT_GLOBAL, kernel_path=PATH_FUSED, device=0, tile_i=0, tile_j=0,
              use_graph=1, nut_inf_ratio=0.0, block_threads=0, staging=0) -> Opts:
    o = Opts()
    lib().jst_default_opts(C.byref(o))
    o.precision, o.dt_mode, o.kernel_path, o.device = precision, dt_mode, kernel_path, device
    o.tile_i, o.tile_j, o.use_graph, o.nut_inf_ratio = tile_i, tile_j, use_graph, nut_inf_ratio
    o.block_threads = block_threads
    o.staging = staging
    return o


class Solver:
    """Solver handle (jst-rs/src/solver.rs:25-34) backed by libjst_gpu.so."""

    def __init__(self, config: dict | str, xy: np.ndarray, n_rings: int, n_theta: int, **opts):
        L = lib()
        text = config if isinstance(config, str) else json.dumps(config)
        xy = np.ascontiguousarray(xy, dtype=np.float64).reshape(-1)
        if xy.size != 2 * n_rings * n_theta:
            raise ValueError("xy must hold n_rings*n_theta (x, y) pairs")
        self._o = make_opts(**opts)
        h = C.c_void_p()
        rc = L.jst_create(text.encode(), _ptr(xy), n_rings, n_theta, C.byref(self._o), C.byref(h))
        if rc != OK:
            raise JstError(rc, L.jst_last_error(None).decode())
        self._h = h
        self.ni = L.jst_ni(h)
        self.nj = L.jst_nj(h)

    @classmethod
    def from_paths(cls, config_path, mesh_path, **opts) -> "Solver":
        """Solver::from_paths (solver.rs:64-68)."""
        L = lib()
        self = cls.__new__(cls)
        self._o = make_opts(**opts)
        h = C.c_void_p()
        rc = L.jst_create_from_paths(str(config_path).encode(), str(mesh_path).encode(), C.byref(self._o),
                                     C.byref(h))
        if rc != OK:
            raise JstError(rc, L.jst_last_error(None).decode())
        self._h = h
        self.ni = L.jst_ni(h)
        self.nj = L.jst_nj(h)
        return self

    def close(self):
        if getattr(self, "_h", None):
            lib().jst_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    @property
    def n_cells(self) -> int:
        return self.ni * self.nj

    def _check(self, rc, bad: NonPhysicalC | None = None):
        if rc == OK:
            return
        if rc == ERR_NONPHYSICAL and bad is not None:
            raise NonPhysical(bad.i, bad.j, bad.rho, bad.p)
        raise JstError(rc, lib().jst_last_error(self._h).decode())

    def advance(self):
        """Solver::advance (solver.rs:97-120)."""
        bad = NonPhysicalC()
        self._check(lib().jst_advance(self._h, C.byref(bad)), bad)

    def run(self, max_steps: int | None = None, on_step=None) -> RunReport:
        """Solver::run (solver.rs:203-226)."""
        bad = NonPhysicalC()
        rep = RunReportC()
        cb = STEP_CB(lambda _u, k, r: on_step(int(k), float(r))) if on_step else STEP_CB()
        rc = lib().jst_run(self._h, -1 if max_steps is None else int(max_steps), cb, None, C.byref(rep),
                           C.byref(bad))
        self._check(rc, bad)
        return RunReport(int(rep.steps), float(rep.residual), float(rep.totaltime), bool(rep.converged))

    def residual_terms(self, with_timestep: bool = False):
        """Solver::residual_terms (solver.rs:86-94); optionally timestep first."""
        dt = C.c_double(0.0)
        self._check(lib().jst_residual_terms(self._h, C.byref(dt) if with_timestep else None))
        return dt.value if with_timestep else None

    def stage_residual(self) -> np.ndarray:
        """R = Fc - Fv - Fd (R[4] -= S) of every cell of the current state, as
        the RK update applies it (solver.rs:128-133), from the stage kernel this
        solver runs with; shape (5, NI, NJ)."""
        n = self.ni * self.nj
        out = np.empty(5 * n)
        self._check(lib().jst_stage_residual(self._h, _ptr(out), out.size))
        return out.reshape(5, self.ni, self.nj)

    def timestep(self) -> float:
        """timestep::compute (timestep.rs:24-57)."""
        dt = C.c_double(0.0)
        self._check(lib().jst_timestep(self._h, C.byref(dt)))
        return dt.value

    def residual(self) -> float:
        r = C.c_double(0.0)
        self._check(lib().jst_residual(self._h, C.byref(r)))
        return r.value

    @property
    def totaltime(self) -> float:
        r = C.c_double(0.0)
        self._check(lib().jst_totaltime(self._h, C.byref(r)))
        return r.value

    @property
    def step(self) -> int:
        r = C.c_int64(0)
        self._check(lib().jst_step_count(self._h, C.byref(r)))
        return r.value

    def get(self, name: str) -> np.ndarray:
        out = np.empty(self.ni * self.nj)
        self._check(lib().jst_get_field(self._h, FIELD_ID[name], _ptr(out), out.size))
        return out.reshape(self.ni, self.nj)

    def faces(self, which: int) -> np.ndarray:
        n = (self.ni + 1 if which == 0 else self.ni) * self.nj
        out = np.empty(4 * n)
        self._check(lib().jst_get_faces(self._h, which, _ptr(out), out.size))
        return out.reshape(n, 4)

    def set_conserved(self, u5: np.ndarray):
        a = np.ascontiguousarray(u5, dtype=np.float64).reshape(-1)
        bad = NonPhysicalC()
        self._check(lib().jst_set_conserved(self._h, _ptr(a), a.size, C.byref(bad)), bad)

    def forces(self):
        """(CL, CD) of the current state (no counterpart in the reference)."""
        cl, cd = C.c_double(), C.c_double()
        self._check(lib().jst_forces(self._h, C.byref(cl), C.byref(cd)))
        return cl.value, cd.value

    def write_csv(self, path):
        """Solver::write_csv (solver.rs:229-255)."""
        self._check(lib().jst_write_csv(self._h, str(path).encode()))

    def save_checkpoint(self, path):
        """Writes U, the step count and the physical time (no counterpart in the reference)."""
        self._check(lib().jst_checkpoint_save(self._h, str(path).encode()))

    def load_checkpoint(self, path):
        """Continues from a checkpoint of a solver on the same mesh."""
        bad = NonPhysicalC()
        self._check(lib().jst_checkpoint_load(self._h, str(path).encode(), C.byref(bad)), bad)

    def time_steps(self, nsteps: int, stages: bool = False):
        """Device time (ms) of `nsteps` RK steps with the convergence test off,
        measured with CUDA events on the solver's stream; with stages=True ten
        more steps run back to back with events between the stage launches
        and the five stage kernels' mean times are returned."""
        ms = C.c_double(0.0)
        st = np.zeros(5)
        self._check(lib().jst_time_steps(self._h, int(nsteps), C.byref(ms), _ptr(st) if stages else None))
        return ms.value, (st.tolist() if stages else None)

    def kernel_config(self):
        """(tile_i, tile_j, block_threads) of the fused path (autotuned when not given)."""
        a, b, c = C.c_int(), C.c_int(), C.c_int()
        self._check(lib().jst_kernel_config(self._h, C.byref(a), C.byref(b), C.byref(c)))
        return a.value, b.value, c.value

    def kernel_staging(self) -> int:
        """STAGING_PER_LANE or STAGING_BULK for marching strips, 0 otherwise."""
        v = C.c_int()
        self._check(lib().jst_kernel_staging(self._h, C.byref(v)))
        return v.value

    # test hooks
    def debug_staging_extra_tx(self, nbytes: int):
        """Make every bulk row-copy barrier expect nbytes more than its copies
        deliver (0 restores it): the bounded waits run out."""
        self._check(lib().jst_debug_staging_extra_tx(self._h, int(nbytes)))

    def set_uniform(self, rho, vx, vy, p, nut):
        self._check(lib().jst_debug_set_uniform(self._h, rho, vx, vy, p, nut))

    def kernel(self, name: str):
        self._check(lib().jst_debug_kernel(self._h, name.encode()))
