"""Batched ensembles of independent hydrodynamics runs (``amrvac_ens_*``).

An ``Ensemble`` holds many standalone runs — 1-D and 2-D instances of uneven
sizes, each with its own flux scheme, limiter and end time — and advances all
of them with one persistent kernel launch per RK stage.  Each instance follows
the reference's time loop (src/amrvac.t:241-343) with its own CFL time step
(setdt, src/mod_dt.t:10-99).  The shared settings come from one ``amrvac_cfg``
built with ``make_cfg(physics="hd", ...)``.

Block arrays are numpy ``float64`` of shape (nblocks, nw, 1, ny, nx) with
nw = ndim + 2 (ny = 1 in 1-D), the Fortran ``w(ixG^S,1:nw)`` of each block, ghosts included;
blocks are ordered x-fastest within an instance.
"""
from __future__ import annotations

import ctypes
from dataclasses import dataclass

import numpy as np

from . import _lib


@dataclass
class Instance:
    ndim: int
    domain_nx: tuple
    xprobmin: tuple = (0.0, 0.0)
    xprobmax: tuple = (1.0, 1.0)
    flux_scheme: str = "hll"
    limiter: str = "minmod"
    time_max: float = 0.2


def _dp(a):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))


class Ensemble:
    def __init__(self, cfg: _lib.AmrvacCfg, instances):
        self.L = _lib.load()
        self.cfg = cfg
        self.instances = list(instances)
        arr = (_lib.AmrvacEnsInstance * len(self.instances))()
        for k, q in enumerate(self.instances):
            a = arr[k]
            a.ndim = q.ndim
            for d in range(2):
                a.domain_nx[d] = int(q.domain_nx[d]) if d < q.ndim else 16
                a.xprobmin[d] = float(q.xprobmin[d]) if d < q.ndim else 0.0
                a.xprobmax[d] = float(q.xprobmax[d]) if d < q.ndim else 1.0
            a.flux_scheme = _lib.FS[q.flux_scheme]
            a.limiter = _lib.LIMITER[q.limiter]
            a.time_max = float(q.time_max)
        h = ctypes.c_void_p()
        _lib.check(self.L.amrvac_ens_create(ctypes.byref(cfg), len(arr), arr, ctypes.byref(h)),
                   "amrvac_ens_create")
        self.h = h
        self.ninst = len(self.instances)
        ng = cfg.nghostcells
        self.nblocks = [self.L.amrvac_ens_nblocks(h, i) for i in range(self.ninst)]
        self.block_shape = [(q.ndim + 2, 1, 16 + 2 * ng if q.ndim == 2 else 1, 16 + 2 * ng)
                            for q in self.instances]

    def close(self):
        if getattr(self, "h", None) is not None and self.h.value:
            self.L.amrvac_ens_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def cells(self, i: int) -> int:
        q = self.instances[i]
        return int(np.prod(q.domain_nx[: q.ndim]))

    def upload(self, i: int, blocks: np.ndarray):
        """blocks: (nblocks, nw, 1, ny, nx) — ny = 1 for a 1-D instance."""
        w = np.ascontiguousarray(blocks, dtype=np.float64)
        need = self.nblocks[i] * int(np.prod(self.block_shape[i]))
        if w.size != need:
            raise ValueError(f"instance {i}: expected {need} values, got {w.size}")
        _lib.check(self.L.amrvac_ens_upload(self.h, i, _dp(w)), "amrvac_ens_upload")

    def download(self, i: int) -> np.ndarray:
        out = np.empty((self.nblocks[i],) + self.block_shape[i], np.float64)
        _lib.check(self.L.amrvac_ens_download(self.h, i, _dp(out)), "amrvac_ens_download")
        return out

    def reset_time(self):
        _lib.check(self.L.amrvac_ens_reset_time(self.h), "amrvac_ens_reset_time")

    def step(self):
        _lib.check(self.L.amrvac_ens_step(self.h), "amrvac_ens_step")

    def run(self, max_steps: int = 1 << 30, chunk: int = 16):
        taken = ctypes.c_int()
        act = ctypes.c_int()
        _lib.check(self.L.amrvac_ens_run(self.h, max_steps, chunk, ctypes.byref(taken), ctypes.byref(act)),
                   "amrvac_ens_run")
        return taken.value, act.value

    def state(self):
        t = np.zeros(self.ninst)
        dt = np.zeros(self.ninst)
        steps = np.zeros(self.ninst, np.int32)
        done = np.zeros(self.ninst, np.int32)
        ip = ctypes.POINTER(ctypes.c_int)
        _lib.check(self.L.amrvac_ens_state(self.h, _dp(t), _dp(dt), steps.ctypes.data_as(ip),
                                           done.ctypes.data_as(ip)), "amrvac_ens_state")
        return t, dt, steps, done

    def status(self):
        f = ctypes.c_uint32()
        per = np.zeros(self.ninst, np.uint32)
        _lib.check(self.L.amrvac_ens_status(self.h, ctypes.byref(f),
                                            per.ctypes.data_as(ctypes.POINTER(ctypes.c_uint32))),
                   "amrvac_ens_status")
        return f.value, per

    def set_grid(self, ctas: int):
        _lib.check(self.L.amrvac_ens_set_grid(self.h, ctas), "amrvac_ens_set_grid")

    def grid(self):
        c = ctypes.c_int()
        w = ctypes.c_int()
        _lib.check(self.L.amrvac_ens_grid(self.h, ctypes.byref(c), ctypes.byref(w)), "amrvac_ens_grid")
        return c.value, w.value

    def set_variant(self, var: int):
        _lib.check(self.L.amrvac_ens_set_variant(self.h, var), "amrvac_ens_set_variant")

    def variant(self):
        """{"variant", "nvariants", "ctas_per_sm"} of the stage kernel."""
        v, n, c = ctypes.c_int(), ctypes.c_int(), ctypes.c_int()
        _lib.check(self.L.amrvac_ens_variant(self.h, ctypes.byref(v), ctypes.byref(n), ctypes.byref(c)),
                   "amrvac_ens_variant")
        return {"variant": v.value, "nvariants": n.value, "ctas_per_sm": c.value}

    def autotune(self, reps: int = 5):
        c = ctypes.c_int()
        ms = ctypes.c_double()
        _lib.check(self.L.amrvac_ens_autotune(self.h, reps, ctypes.byref(c), ctypes.byref(ms)),
                   "amrvac_ens_autotune")
        return c.value, ms.value

    def stream_ptr(self) -> int:
        p = ctypes.c_void_p()
        _lib.check(self.L.amrvac_ens_stream(self.h, ctypes.byref(p)), "amrvac_ens_stream")
        return p.value or 0

    def launch_count(self) -> int:
        return int(self.L.amrvac_ens_launch_count(self.h))
