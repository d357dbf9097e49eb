"""Host-side API mirroring the reference's driver of the finite-volume path.

``Context`` owns one ``amrvac_ctx`` (one CUDA stream, one set of resident
block registers ps/ps1/ps2).  Its methods follow the reference routines they
replace:

  ``getdt()``     -> setdt / getdt_courant   (src/mod_dt.t:10-287)
  ``advect1()``   -> advect1 / finite_volume (src/mod_advance.t:611-734,
                     src/mod_finite_volume.t:116-339)
  ``advance()``   -> advance/advect with the configured time stepper
                     (src/mod_advance.t:17-567), setdt included
  ``download()``  -> the ghosted block arrays after getbc
                     (src/mod_ghostcells_update.t:350-615)

Block arrays are numpy ``float64`` with shape (nblocks, nw, nz, ny, nx) in C
order, i.e. the Fortran ``w(ixG^S,1:nw)`` of each block, ghosts included.
"""
from __future__ import annotations

import ctypes

import numpy as np

from . import _lib
from .config import make_cfg  # noqa: F401  (re-export)

REG = {"ps": 0, "ps1": 1, "ps2": 2}


def _dp(a):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))


class Context:
    def __init__(self, cfg: _lib.AmrvacCfg):
        self.L = _lib.load()
        self.cfg = cfg
        self.nw = self.L.amrvac_gpu_nw(cfg)
        h = ctypes.c_void_p()
        _lib.check(self.L.amrvac_gpu_create(ctypes.byref(cfg), ctypes.byref(h)), "amrvac_gpu_create")
        self.h = h
        self.nblocks = 0
        ng = cfg.nghostcells
        self.bn = int(cfg.block_nx[0])  # cells per block edge
        self.ghosted = tuple([self.bn + 2 * ng if d < cfg.ndim else 1 for d in (2, 1, 0)])
        self.block_shape = (self.nw,) + self.ghosted

    def close(self):
        if getattr(self, "h", None) is not None and self.h.value:
            self.L.amrvac_gpu_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    # ---------------------------------------------------------------- blocks
    def set_uniform_grid(self, domain_nx, xprobmin, xprobmax):
        d = np.ascontiguousarray(domain_nx, dtype=np.int32)
        a = np.ascontiguousarray(xprobmin, dtype=np.float64)
        b = np.ascontiguousarray(xprobmax, dtype=np.float64)
        _lib.check(self.L.amrvac_gpu_set_uniform_grid(
            self.h, d.ctypes.data_as(ctypes.POINTER(ctypes.c_int)), _dp(a), _dp(b)), "set_uniform_grid")
        self.nblocks = self.L.amrvac_gpu_nblocks(self.h)

    def set_amr_grid(self, leaves, nbase, xprobmin, xprobmax):
        """Static multi-level grid: leaves [(level, ig0, ig1[, ig2])] of a 2:1
        balanced tree over nbase root blocks per direction (periodic)."""
        nd = self.cfg.ndim
        lv = np.zeros((len(leaves), 4), np.int32)
        for b, t in enumerate(leaves):
            lv[b, :len(t)] = t
        nb = np.ascontiguousarray(list(nbase)[:nd] + [1] * (3 - nd), dtype=np.int32)
        a = np.ascontiguousarray(list(xprobmin)[:nd] + [0.0] * (3 - nd), dtype=np.float64)
        b = np.ascontiguousarray(list(xprobmax)[:nd] + [1.0] * (3 - nd), dtype=np.float64)
        ip = ctypes.POINTER(ctypes.c_int)
        _lib.check(self.L.amrvac_gpu_set_amr_grid(self.h, len(leaves), lv.ctypes.data_as(ip), nb.ctypes.data_as(ip),
                                                  _dp(a), _dp(b)), "set_amr_grid")
        self.nblocks = self.L.amrvac_gpu_nblocks(self.h)

    def amr_regrid(self, leaves, ops):
        """Regrid in place: new leaves and per new leaf the op row (9 ints)
        saying how its state comes from the old tree (amrvac_b200.amr.ops)."""
        lv = np.zeros((len(leaves), 4), np.int32)
        for b, t in enumerate(leaves):
            lv[b, :len(t)] = t
        op = np.ascontiguousarray(ops, dtype=np.int32).reshape(len(leaves), 9)
        ip = ctypes.POINTER(ctypes.c_int)
        _lib.check(self.L.amrvac_gpu_amr_regrid(self.h, len(leaves), lv.ctypes.data_as(ip), op.ctypes.data_as(ip)),
                   "amr_regrid")
        self.nblocks = self.L.amrvac_gpu_nblocks(self.h)

    def amr_resettree(self, weight, logflag=None, refine_max_level=2, refine_threshold=0.1, derefine_ratio=0.125,
                      amr_wavefilter=1e-2):
        """resettree on the resident state (Löhner, tree decision, remap) in
        one library call; returns True if the tree changed."""
        nl = refine_max_level
        per = lambda x: np.ascontiguousarray(np.broadcast_to(np.asarray(x, np.float64), (nl,)))  # noqa: E731
        w = np.ascontiguousarray(weight, np.float64)
        lf = None if logflag is None else np.ascontiguousarray(logflag, np.int32)
        ip = ctypes.POINTER(ctypes.c_int)
        ch = ctypes.c_int(0)
        _lib.check(self.L.amrvac_gpu_amr_resettree(self.h, _dp(w), lf.ctypes.data_as(ip) if lf is not None else None,
                                                   nl, _dp(per(refine_threshold)), _dp(per(derefine_ratio)),
                                                   _dp(per(amr_wavefilter)), ctypes.byref(ch)), "amr_resettree")
        self.nblocks = self.L.amrvac_gpu_nblocks(self.h)
        return bool(ch.value)

    def amr_leaves(self):
        """The current leaves as (level, ig0, ig1, ig2) tuples in block order."""
        n = self.L.amrvac_gpu_amr_leaves(self.h, None)
        if n < 0:
            raise RuntimeError("amr_leaves: no multi-level grid")
        out = np.zeros((n, 4), np.int32)
        self.L.amrvac_gpu_amr_leaves(self.h, out.ctypes.data_as(ctypes.POINTER(ctypes.c_int)))
        return [tuple(int(x) for x in r) for r in out]

    @property
    def amr_slots(self):
        return self.L.amrvac_gpu_amr_slots(self.h)

    def amr_kernel_ms(self, reps=10):
        """(ghost pass ms, flux fix ms) per launch; the fix changes register ps2."""
        g, f = ctypes.c_double(), ctypes.c_double()
        _lib.check(self.L.amrvac_gpu_amr_kernel_ms(self.h, reps, ctypes.byref(g), ctypes.byref(f)), "amr_kernel_ms")
        return g.value, f.value

    def set_blocks(self, dx, neighbor):
        dx = np.ascontiguousarray(dx, dtype=np.float64)
        nb = np.ascontiguousarray(neighbor, dtype=np.int32)
        _lib.check(self.L.amrvac_gpu_set_blocks(self.h, dx.shape[0], _dp(dx),
                                                 nb.ctypes.data_as(ctypes.POINTER(ctypes.c_int))),
                   "set_blocks")
        self.nblocks = dx.shape[0]

    def upload(self, w: np.ndarray, reg="ps", first=0):
        w = np.ascontiguousarray(w, dtype=np.float64)
        if w.ndim != 1 + len(self.block_shape) or tuple(w.shape[1:]) != tuple(self.block_shape):
            raise ValueError(f"upload: blocks of shape {tuple(self.block_shape)} expected, got {w.shape[1:]}")
        n = w.shape[0]
        if first < 0 or first + n > self.nblocks:
            raise ValueError(f"upload: blocks {first}..{first + n - 1} outside 0..{self.nblocks - 1}")
        _lib.check(self.L.amrvac_gpu_upload(self.h, REG.get(reg, reg), first, n, _dp(w)), "upload")

    def download(self, reg="ps", first=0, n=None) -> np.ndarray:
        n = self.nblocks - first if n is None else n
        out = np.empty((n,) + self.block_shape, np.float64)
        _lib.check(self.L.amrvac_gpu_download(self.h, REG.get(reg, reg), first, n, _dp(out)), "download")
        return out

    # ---------------------------------------------------------------- path
    def getdt(self, reg="ps"):
        dt = ctypes.c_double()
        cm = ctypes.c_double()
        st = _lib.check(self.L.amrvac_gpu_getdt(self.h, REG.get(reg, reg), ctypes.byref(dt), ctypes.byref(cm)),
                        "getdt")
        return dt.value, cm.value, st

    def set_cmax_global(self, cmax_global: float):
        _lib.check(self.L.amrvac_gpu_set_cmax_global(self.h, cmax_global), "set_cmax_global")

    def advect1(self, reg_ct, reg_new, dtfactor, dt, reg_base="ps", a_base=0.0, b_in=1.0, idim=0):
        """One stage; idim 1..ndim restricts it to that direction (a
        dimensionally split sweep), 0 advances all directions."""
        if idim:
            return _lib.check(self.L.amrvac_gpu_advect1_dim(self.h, REG.get(reg_ct, reg_ct), REG.get(reg_new, reg_new),
                                                            REG.get(reg_base, reg_base), a_base, b_in, dtfactor, dt,
                                                            idim), "advect1_dim")
        return _lib.check(self.L.amrvac_gpu_advect1(self.h, REG.get(reg_ct, reg_ct), REG.get(reg_new, reg_new),
                                                    REG.get(reg_base, reg_base), a_base, b_in, dtfactor, dt),
                          "advect1")

    def set_time(self, t=0.0, time_max=1.0e99, dtsave=0.0):
        _lib.check(self.L.amrvac_gpu_set_time(self.h, t, time_max, dtsave), "set_time")

    def step(self):
        _lib.check(self.L.amrvac_gpu_step(self.h), "step")

    def run(self, nsteps: int):
        _lib.check(self.L.amrvac_gpu_run(self.h, nsteps), "run")

    def run_timed(self, nsteps: int):
        """(total_ms, stage_kernels_ms, getdt_kernels_ms) over nsteps steps."""
        a, b, c = ctypes.c_double(), ctypes.c_double(), ctypes.c_double()
        _lib.check(self.L.amrvac_gpu_run_timed(self.h, nsteps, ctypes.byref(a), ctypes.byref(b), ctypes.byref(c)),
                   "run_timed")
        return a.value, b.value, c.value

    def autotune(self, reps: int = 3, cache: bool = True):
        """Pick the z-chunk of the 3-D stage kernel by timing (see tuning.py)."""
        from . import tuning
        return tuning.autotune(self, reps=reps, cache=cache)

    def set_zchunk(self, zchunk: int):
        _lib.check(self.L.amrvac_gpu_set_zchunk(self.h, zchunk), "set_zchunk")

    def set_stage_variant(self, var: int):
        """Select stage-kernel variant var (0: the scheme's default kernel)."""
        _lib.check(self.L.amrvac_gpu_set_stage_variant(self.h, var), "set_stage_variant")

    def stage_variant(self) -> dict:
        """The current stage-kernel variant: its index, the number of
        variants, threads per CTA, CTAs per SM, asynchronous staging."""
        v = [ctypes.c_int() for _ in range(5)]
        _lib.check(self.L.amrvac_gpu_stage_variant(self.h, *[ctypes.byref(x) for x in v]), "stage_variant")
        return dict(variant=v[0].value, nvariants=v[1].value, threads=v[2].value, ctas_per_sm=v[3].value,
                    async_staging=bool(v[4].value))

    def get_time(self):
        dt, cm, t = ctypes.c_double(), ctypes.c_double(), ctypes.c_double()
        _lib.check(self.L.amrvac_gpu_get_time(self.h, ctypes.byref(dt), ctypes.byref(cm), ctypes.byref(t)),
                   "get_time")
        return dt.value, cm.value, t.value

    def status(self) -> int:
        f = ctypes.c_uint32()
        _lib.check(self.L.amrvac_gpu_status(self.h, ctypes.byref(f)), "status")
        return f.value

    def clear_status(self):
        _lib.check(self.L.amrvac_gpu_clear_status(self.h), "clear_status")

    def synchronize(self):
        _lib.check(self.L.amrvac_gpu_synchronize(self.h), "synchronize")

    def stream_ptr(self) -> int:
        p = ctypes.c_void_p()
        _lib.check(self.L.amrvac_gpu_stream(self.h, ctypes.byref(p)), "stream")
        return p.value or 0

    def register_ptr(self, reg="ps") -> int:
        p = ctypes.POINTER(ctypes.c_double)()
        _lib.check(self.L.amrvac_gpu_register_ptr(self.h, REG.get(reg, reg), ctypes.byref(p)), "register_ptr")
        return ctypes.cast(p, ctypes.c_void_p).value

    def lohner(self, weight, logflag=None, refine_max_level=2, refine_threshold=0.1, derefine_ratio=0.125,
               amr_wavefilter=1e-2, block_level=None, reg="ps"):
        """Löhner estimator on all blocks: (flags, errmax) with flags 1 refine | 2 coarsen."""
        nl = refine_max_level
        per = lambda x: np.ascontiguousarray(np.broadcast_to(np.asarray(x, np.float64), (nl,)))  # noqa: E731
        w = np.ascontiguousarray(weight, np.float64)
        lf = None if logflag is None else np.ascontiguousarray(logflag, np.int32)
        lv = None if block_level is None else np.ascontiguousarray(block_level, np.int32)
        flags = np.zeros(self.nblocks, np.int32)
        errmax = np.zeros(self.nblocks, np.float64)
        ip = ctypes.POINTER(ctypes.c_int)
        _lib.check(self.L.amrvac_gpu_lohner(self.h, REG.get(reg, reg), _dp(w), lf.ctypes.data_as(ip) if lf is not None
                                            else None, nl, _dp(per(refine_threshold)), _dp(per(derefine_ratio)),
                                            _dp(per(amr_wavefilter)), lv.ctypes.data_as(ip) if lv is not None else None,
                                            flags.ctypes.data_as(ip), _dp(errmax)), "lohner")
        return flags, errmax

    def launch_count(self) -> int:
        return int(self.L.amrvac_gpu_launch_count(self.h))

    # ---------------------------------------------------------------- per routine
    def riemann_points(self, wlp, wrp, idim, cmax_global=0.0):
        wlp = np.ascontiguousarray(wlp, dtype=np.float64)
        wrp = np.ascontiguousarray(wrp, dtype=np.float64)
        f = np.empty_like(wlp)
        _lib.check(self.L.amrvac_gpu_riemann_points(self.h, wlp.shape[0], _dp(wlp), _dp(wrp), idim, cmax_global,
                                                     _dp(f)), "riemann_points")
        return f

    def get_flux_points(self, wc, wp, idim, cmax_global=0.0):
        wc = np.ascontiguousarray(wc, dtype=np.float64)
        wp = np.ascontiguousarray(wp, dtype=np.float64)
        f = np.empty_like(wc)
        _lib.check(self.L.amrvac_gpu_get_flux_points(self.h, wc.shape[0], _dp(wc), _dp(wp), idim, cmax_global,
                                                      _dp(f)), "get_flux_points")
        return f

    def get_cbounds_points(self, wlc, wrc, wlp, wrp, idim, with_cmin=True):
        arrs = [np.ascontiguousarray(a, dtype=np.float64) for a in (wlc, wrc, wlp, wrp)]
        n = arrs[0].shape[0]
        cmax = np.empty(n)
        cmin = np.empty(n) if with_cmin else None
        _lib.check(self.L.amrvac_gpu_get_cbounds_points(
            self.h, n, *[_dp(a) for a in arrs], idim, _dp(cmax),
            _dp(cmin) if with_cmin else ctypes.POINTER(ctypes.c_double)()), "get_cbounds_points")
        return (cmax, cmin) if with_cmin else cmax

    # ---------------------------------------------------------------- drivers
    def advance(self):
        """One full step: setdt on the device, RK stages, time update."""
        self.step()


def fp64_peak_tflops() -> float:
    """Measured FP64 FMA throughput of the current device (TFLOP/s)."""
    v = ctypes.c_double()
    _lib.check(_lib.load().amrvac_gpu_fp64_peak(ctypes.byref(v)), "fp64_peak")
    return v.value


def srl_maps(nghost: int, block_nx: int):
    """ixS_srl_/ixR_srl_ of init_bc, 0-based (s_min, s_max, r_min, r_max)."""
    L = _lib.load()
    a = [np.zeros(3, np.int32) for _ in range(4)]
    _lib.check(L.amrvac_gpu_srl_maps(nghost, block_nx, *[x.ctypes.data_as(ctypes.POINTER(ctypes.c_int)) for x in a]),
               "srl_maps")
    return a
