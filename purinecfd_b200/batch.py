"""Python binding of the batched solver (jst_batch_* in include/jst_gpu.h).

Many independent solves of different meshes and flow conditions share one
persistent stage kernel over a device tile table; each RK step is replayed
from a CUDA graph; instances are admitted as memory and slots allow and retire
individually.
"""

from __future__ import annotations

import ctypes as C
import json
from dataclasses import dataclass

import numpy as np

from .solver import (DT_LOCAL, OK, PREC_FP32_SPLIT, JstError, NonPhysicalC, lib)


class BatchOptsC(C.Structure):
    _fields_ = [("precision", C.c_int), ("dt_mode", C.c_int), ("device", C.c_int), ("tile_i", C.c_int),
                ("tile_j", C.c_int), ("max_instances", C.c_int), ("steps_per_poll", C.c_int),
                ("hbm_budget_gb", C.c_double), ("keep_fields", C.c_int), ("block_threads", C.c_int),
                ("staging", C.c_int)]


class BatchResultC(C.Structure):
    _fields_ = [("id", C.c_int64), ("status", C.c_int), ("steps", C.c_int64), ("residual", C.c_double),
                ("residual_first", C.c_double), ("totaltime", C.c_double), ("cl", C.c_double), ("cd", C.c_double),
                ("t_submit", C.c_double), ("t_admit", C.c_double), ("t_done", C.c_double), ("ni", C.c_int),
                ("nj", C.c_int), ("bad", NonPhysicalC)]


@dataclass
class BatchResult:
    id: int
    status: int
    steps: int
    residual: float
    residual_first: float
    totaltime: float
    cl: float
    cd: float
    t_submit: float
    t_admit: float
    t_done: float
    ni: int
    nj: int
    fields: np.ndarray | None = None

    @property
    def latency(self) -> float:
        return self.t_done - self.t_submit


# The batch entry points of include/jst_gpu.h this module binds.
BATCH_EXPORTS = ["jst_batch_default_opts", "jst_batch_create", "jst_batch_destroy", "jst_batch_submit",
                 "jst_batch_step", "jst_batch_stats", "jst_batch_poll", "jst_batch_result_get",
                 "jst_batch_kernel_config", "jst_batch_kernel_staging"]


def _bind():
    L = lib()
    if getattr(L, "_batch_bound", False):
        return L
    vp, i, d = C.c_void_p, C.c_int, C.c_double
    pd = C.POINTER(C.c_double)
    L.jst_batch_default_opts.argtypes = [C.POINTER(BatchOptsC)]
    L.jst_batch_create.argtypes = [C.POINTER(BatchOptsC), C.POINTER(vp)]
    L.jst_batch_destroy.argtypes = [vp]
    L.jst_batch_submit.argtypes = [vp, C.c_char_p, pd, i, i, C.c_int64, d, d, C.POINTER(C.c_int64)]
    L.jst_batch_step.argtypes = [vp, i]
    L.jst_batch_stats.argtypes = [vp, C.POINTER(i), C.POINTER(i), pd]
    L.jst_batch_kernel_config.argtypes = [vp, C.POINTER(i), C.POINTER(i), C.POINTER(i)]
    L.jst_batch_kernel_staging.argtypes = [vp, C.POINTER(i)]
    L.jst_batch_poll.argtypes = [vp, C.POINTER(C.c_int64), i, C.POINTER(i)]
    L.jst_batch_result_get.argtypes = [vp, C.c_int64, C.POINTER(BatchResultC), pd, C.c_size_t]
    L._batch_bound = True
    return L


class Batch:
    def __init__(self, precision=PREC_FP32_SPLIT, dt_mode=DT_LOCAL, device=0, tile_i=0, tile_j=0,
                 max_instances=256, steps_per_poll=20, hbm_budget_gb=0.0, keep_fields=False, block_threads=0,
                 staging=0):
        L = _bind()
        o = BatchOptsC()
        L.jst_batch_default_opts(C.byref(o))
        o.precision, o.dt_mode, o.device, o.tile_i, o.tile_j = precision, dt_mode, device, tile_i, tile_j
        o.max_instances, o.steps_per_poll, o.hbm_budget_gb = max_instances, steps_per_poll, hbm_budget_gb
        o.keep_fields = 1 if keep_fields else 0
        o.block_threads = block_threads
        o.staging = staging
        h = C.c_void_p()
        rc = L.jst_batch_create(C.byref(o), C.byref(h))
        if rc != OK:
            raise JstError(rc, L.jst_last_error(None).decode())
        self._h = h
        self._keep = keep_fields
        self._sizes = {}

    def close(self):
        if getattr(self, "_h", None):
            lib().jst_batch_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def submit(self, config: dict | str, xy: np.ndarray, n_rings: int, n_theta: int, max_steps: int = -1,
               residual_drop: float = 0.0, cl_tol: float = 0.0) -> int:
        L = lib()
        text = config if isinstance(config, str) else json.dumps(config)
        a = np.ascontiguousarray(xy, dtype=np.float64).reshape(-1)
        ident = C.c_int64()
        rc = L.jst_batch_submit(self._h, text.encode(), a.ctypes.data_as(C.POINTER(C.c_double)), n_rings, n_theta,
                                int(max_steps), float(residual_drop), float(cl_tol), C.byref(ident))
        if rc != OK:
            raise JstError(rc, L.jst_last_error(None).decode())
        return ident.value

    def step(self, nsteps: int):
        rc = lib().jst_batch_step(self._h, int(nsteps))
        if rc != OK:
            raise JstError(rc, lib().jst_last_error(None).decode())

    def stats(self):
        a, q, b = C.c_int(), C.c_int(), C.c_double()
        lib().jst_batch_stats(self._h, C.byref(a), C.byref(q), C.byref(b))
        return a.value, q.value, b.value

    def kernel_config(self):
        """(tile_i, tile_j, block_threads) of the batch's stage kernel."""
        a, b, c = C.c_int(), C.c_int(), C.c_int()
        lib().jst_batch_kernel_config(self._h, C.byref(a), C.byref(b), C.byref(c))
        return a.value, b.value, c.value

    def kernel_staging(self) -> int:
        """jst_staging of the batch's stage kernel (0 when not marching strips)."""
        v = C.c_int()
        lib().jst_batch_kernel_staging(self._h, C.byref(v))
        return v.value

    def poll(self, cap: int = 4096) -> list[int]:
        ids = (C.c_int64 * cap)()
        n = C.c_int()
        lib().jst_batch_poll(self._h, ids, cap, C.byref(n))
        return [ids[k] for k in range(n.value)]

    def result(self, ident: int) -> BatchResult:
        L = lib()
        r = BatchResultC()
        rc = L.jst_batch_result_get(self._h, int(ident), C.byref(r), None, 0)
        if rc != OK:
            raise KeyError(ident)
        fields = None
        if self._keep:
            n = r.ni * r.nj
            fields = np.empty(5 * n)
            L.jst_batch_result_get(self._h, int(ident), C.byref(r), fields.ctypes.data_as(C.POINTER(C.c_double)),
                                   fields.size)
            fields = fields.reshape(5, r.ni, r.nj)
        return BatchResult(r.id, r.status, r.steps, r.residual, r.residual_first, r.totaltime, r.cl, r.cd,
                           r.t_submit, r.t_admit, r.t_done, r.ni, r.nj, fields)

    def run_all(self, chunk: int = 200, max_rounds: int = 10**9) -> list[BatchResult]:
        """Step until nothing is active or queued; return every result."""
        out = []
        for _ in range(max_rounds):
            a, q, _ = self.stats()
            if a == 0 and q == 0:
                break
            self.step(chunk)
            out += [self.result(i) for i in self.poll()]
        out += [self.result(i) for i in self.poll()]
        return out
