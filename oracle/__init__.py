"""ctypes binding of the CPU oracle (test infrastructure only).

The oracle is a C++ restatement of the reference's finite-volume path
(``oracle/amrvac_oracle.cpp``).  It is the checker for the CUDA product path;
only ``tests/``, ``__graft_entry__.smoke`` and the CPU-baseline leg of
``bench.py`` may import this module.
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "_build", "liboracle.so")

FS = {"tvdlf": 1, "hll": 2, "hllc": 3, "hlld": 4, "tvdmu": 5}
LIMITER = {"minmod": 1, "woodward": 2, "mcbeta": 3, "superbee": 4, "vanleer": 5,
           "albada": 6, "koren": 7, "cada": 8, "cada3": 9, "schmid1": 10, "schmid2": 10, "venk": 11, "mp5": 13, "weno3": 14, "wenoyc3": 15, "weno5": 16, "wenoz5": 18, "wenozp5": 20}
BOUNDSPEED = {"Einfeldt": 1, "cmaxmean": 2, "cmaxleftright": 3}
DIVB = {"none": 0, "glm": 1, "linde": 4}
BC = {"periodic": 0, "cont": 1, "symm": 2, "asymm": 3}
ST_SMALL_VALUE = 1


class OrcCfg(ctypes.Structure):
    _fields_ = [
        ("ndim", ctypes.c_int), ("ndir", ctypes.c_int), ("physics", ctypes.c_int),
        ("nw", ctypes.c_int), ("nghost", ctypes.c_int), ("block_nx", ctypes.c_int * 3),
        ("gamma", ctypes.c_double), ("flux_scheme", ctypes.c_int), ("limiter", ctypes.c_int),
        ("boundspeed", ctypes.c_int), ("divb", ctypes.c_int), ("glm_alpha", ctypes.c_double),
        ("glm_extended", ctypes.c_int), ("courantpar", ctypes.c_double),
        ("type_courant", ctypes.c_int), ("cada3_radius", ctypes.c_double),
        ("tvdlfeps", ctypes.c_double), ("fix_small_values", ctypes.c_int),
        ("check_small_values", ctypes.c_int), ("small_values_method", ctypes.c_int),
        ("small_density", ctypes.c_double), ("small_pressure", ctypes.c_double),
        ("divbdiff", ctypes.c_double), ("ssprk_order", ctypes.c_int),
        ("time_stepper", ctypes.c_int), ("time_integrator", ctypes.c_int),
        ("dimsplit", ctypes.c_int),
        ("schmid_rad", ctypes.c_double * 3),
        ("schmid_global", ctypes.c_int),
        ("small_values_daverage", ctypes.c_int),
    ]


def build() -> str:
    """Compile the oracle with its Makefile (g++ only, seconds)."""
    subprocess.run(["make", "-s", "-C", _HERE], check=True)
    return _LIB_PATH


_lib = None


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(_LIB_PATH):
            build()
        L = ctypes.CDLL(_LIB_PATH)
        P = ctypes.POINTER
        d = ctypes.c_double
        dp = P(ctypes.c_double)
        ip = P(ctypes.c_int)
        cp = P(OrcCfg)
        L.orc_cfg_finalize.argtypes = [cp]
        L.orc_finite_volume.argtypes = [cp, dp, dp, d, d, dp, d]
        L.orc_getdt_block.argtypes = [cp, dp, dp, dp, dp]
        L.orc_to_primitive.argtypes = [cp, dp]
        L.orc_to_conserved.argtypes = [cp, dp]
        L.orc_get_flux_points.argtypes = [cp, ctypes.c_int, dp, dp, ctypes.c_int, d, dp]
        L.orc_get_cbounds_points.argtypes = [cp, ctypes.c_int, dp, dp, dp, dp, ctypes.c_int, dp, dp]
        L.orc_riemann_points.argtypes = [cp, ctypes.c_int, dp, dp, ctypes.c_int, d, dp]
        L.orc_limiter_line.argtypes = [cp, ctypes.c_int, dp, d, dp, dp]
        L.orc_grid_create.restype = ctypes.c_void_p
        L.orc_grid_create.argtypes = [cp, ip, dp, dp, ip]
        L.orc_grid_destroy.argtypes = [ctypes.c_void_p]
        L.orc_grid_nblocks.argtypes = [ctypes.c_void_p]
        L.orc_grid_block_index.argtypes = [ctypes.c_void_p, ctypes.c_int, ip]
        L.orc_grid_dx.argtypes = [ctypes.c_void_p, dp]
        L.orc_grid_x.restype = d
        L.orc_grid_x.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.c_int]
        L.orc_grid_set_block.argtypes = [ctypes.c_void_p, ctypes.c_int, dp]
        L.orc_grid_get_block.argtypes = [ctypes.c_void_p, ctypes.c_int, dp]
        L.orc_grid_getbc.argtypes = [ctypes.c_void_p]
        L.orc_grid_getdt.argtypes = [ctypes.c_void_p, dp, dp]
        L.orc_grid_advance.argtypes = [ctypes.c_void_p, d, d, ctypes.c_int]
        L.orc_grid_advect1.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_int, d, d, d, ctypes.c_int]
        L.orc_grid_copy_reg.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_int]
        L.orc_grid_combine_reg.argtypes = [ctypes.c_void_p, ctypes.c_int, d, ctypes.c_int, d, ctypes.c_int]
        L.orc_grid_volume_average.argtypes = [ctypes.c_void_p, ctypes.c_int, dp]
        L.orc_srl_maps.argtypes = [ctypes.c_int, ctypes.c_int, ip, ip, ip, ip]
        L.orc_run_field_loop.argtypes = [cp, d, d, d, ctypes.c_int, dp, ctypes.c_int]
        L.orc_count_flops_stage.restype = d
        L.orc_count_flops_stage.argtypes = [cp, dp, dp, d, dp, d]
        L.orc_count_flops_getdt.restype = d
        L.orc_count_flops_getdt.argtypes = [cp, dp, dp]
        vp = ctypes.c_void_p
        L.orc_amr_create.restype = vp
        L.orc_amr_create.argtypes = [cp, ip, dp, dp, ctypes.c_int, ip, ip]
        L.orc_amr_destroy.argtypes = [vp]
        L.orc_amr_neighbors.argtypes = [vp, ip, ip, ip]
        L.orc_amr_set_block.argtypes = [vp, ctypes.c_int, dp]
        L.orc_amr_get_block.argtypes = [vp, ctypes.c_int, ctypes.c_int, dp]
        L.orc_amr_getbc.argtypes = [vp]
        L.orc_amr_getdt.argtypes = [vp, dp, dp]
        L.orc_amr_advect1.argtypes = [vp, ctypes.c_int, ctypes.c_int, d, d, d, ctypes.c_int]
        L.orc_amr_combine_reg.argtypes = [vp, ctypes.c_int, d, ctypes.c_int, d, ctypes.c_int]
        L.orc_amr_advance.argtypes = [vp, d, d, ctypes.c_int]
        L.orc_amr_remap.restype = vp
        L.orc_amr_remap.argtypes = [vp, ctypes.c_int, ip, ip]
        L.orc_lohner_block.restype = None
        L.orc_lohner_block.argtypes = [cp, dp, dp, ip, d, d, d, ctypes.c_int, ctypes.c_int, dp, ip, ip]
        L.orc_dual_run.restype = ctypes.c_int
        L.orc_dual_run.argtypes = [cp, ip, dp, dp, ip, dp, dp, d, ctypes.c_int, dp, dp, ctypes.c_int, dp, dp, dp]
        _lib = L
    return _lib


def _dp(a: np.ndarray):
    assert a.dtype == np.float64 and a.flags["C_CONTIGUOUS"]
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))


def _ip(a: np.ndarray):
    assert a.dtype == np.int32 and a.flags["C_CONTIGUOUS"]
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_int))


def make_cfg(*, ndim=2, ndir=None, physics="hd", block_nx=16, nghost=2, gamma=None,
             flux_scheme="hll", limiter="minmod", typeboundspeed="Einfeldt", divb="linde",
             glm_alpha=0.5, glm_extended=True, courantpar=0.8, type_courant=1,
             cada3_radius=0.1, tvdlfeps=1.0, fix_small_values=False, check_small_values=True,
             small_values_method="error", small_density=0.0, small_pressure=0.0,
             divbdiff=0.8, ssprk_order=3, time_stepper="threestep", time_integrator="default",
             dimsplit=False, typedimsplit="xyyx", schmid_rad=(1.0, 1.0, 1.0),
             small_values_daverage=1) -> OrcCfg:
    c = OrcCfg()
    c.ndim = ndim
    c.ndir = ndim if ndir is None else ndir
    c.physics = 1 if physics == "mhd" else 0
    c.nghost = nghost
    bn = [block_nx] * 3 if isinstance(block_nx, int) else list(block_nx) + [1] * (3 - len(block_nx))
    for d in range(3):
        c.block_nx[d] = bn[d] if d < ndim else 1
    c.gamma = (5.0 / 3.0) if gamma is None else gamma
    c.flux_scheme = FS[flux_scheme]
    c.limiter = LIMITER[limiter]
    c.boundspeed = BOUNDSPEED[typeboundspeed]
    c.divb = DIVB[divb] if (physics == "mhd" and ndim > 1) else 0
    c.glm_alpha = glm_alpha
    c.glm_extended = int(glm_extended)
    c.courantpar = courantpar
    c.type_courant = type_courant
    c.cada3_radius = cada3_radius
    c.tvdlfeps = tvdlfeps
    c.fix_small_values = int(fix_small_values)
    c.check_small_values = int(check_small_values)
    c.small_values_method = {"error": 0, "replace": 1, "average": 2}[small_values_method]
    c.small_density = small_density
    c.small_pressure = small_pressure
    c.divbdiff = divbdiff
    c.ssprk_order = ssprk_order
    c.time_stepper = {"twostep": 2, "threestep": 3, "fourstep": 4, "fivestep": 5}[time_stepper]
    c.time_integrator = {"default": 0, "Predictor_Corrector": 0, "ssprk4": 0, "rk4": 1, "ssprk2": 2}[time_integrator]
    c.dimsplit = 0 if not dimsplit else (2 if typedimsplit == "xy" else 1)
    for d in range(3):
        c.schmid_rad[d] = float(schmid_rad[d])
    c.schmid_global = int(limiter == "schmid1")
    c.small_values_daverage = int(small_values_daverage)
    lib().orc_cfg_finalize(ctypes.byref(c))
    return c


def block_shape(c: OrcCfg):
    """Fortran array w(ixG^S,1:nw) as a numpy shape in C order (nw, nz, ny, nx)."""
    n = [c.block_nx[d] + 2 * c.nghost if d < c.ndim else 1 for d in range(3)]
    return (c.nw, n[2], n[1], n[0])


def finite_volume(c: OrcCfg, wct: np.ndarray, wnew: np.ndarray, qdt: float, dx, cmax_global=0.0,
                  dtfactor=1.0) -> int:
    dxa = np.ascontiguousarray(np.asarray(dx, dtype=np.float64))
    return lib().orc_finite_volume(ctypes.byref(c), _dp(wct), _dp(wnew), qdt, dtfactor, _dp(dxa),
                                   cmax_global)


def getdt_block(c: OrcCfg, w: np.ndarray, dx):
    dxa = np.ascontiguousarray(np.asarray(dx, dtype=np.float64))
    dt = ctypes.c_double(0.0)
    cm = ctypes.c_double(0.0)
    lib().orc_getdt_block(ctypes.byref(c), _dp(w), _dp(dxa), ctypes.byref(dt), ctypes.byref(cm))
    return dt.value, cm.value


def srl_maps(nghost: int, block_nx: int):
    a = [np.zeros(3, np.int32) for _ in range(4)]
    lib().orc_srl_maps(nghost, block_nx, *[_ip(x) for x in a])
    return a


class Grid:
    """Uniform level-1 block grid of the oracle (periodic/cont boundaries)."""

    def __init__(self, c: OrcCfg, domain_nx, xprobmin, xprobmax, bc):
        self.c = c
        dn = np.array(list(domain_nx) + [1] * (3 - len(domain_nx)), np.int32)
        xmn = np.array(list(xprobmin) + [0.0] * (3 - len(xprobmin)), np.float64)
        xmx = np.array(list(xprobmax) + [1.0] * (3 - len(xprobmax)), np.float64)
        bca = np.array([BC[b] if isinstance(b, str) else b for b in bc] + [0] * (6 - len(bc)), np.int32)
        self.h = lib().orc_grid_create(ctypes.byref(c), _ip(dn), _dp(xmn), _dp(xmx), _ip(bca))
        self.nblocks = lib().orc_grid_nblocks(self.h)
        self.shape = block_shape(c)

    def __del__(self):
        if getattr(self, "h", None):
            lib().orc_grid_destroy(self.h)
            self.h = None

    def dx(self):
        a = np.zeros(3, np.float64)
        lib().orc_grid_dx(self.h, _dp(a))
        return a[: self.c.ndim]

    def block_index(self, ib):
        a = np.zeros(3, np.int32)
        lib().orc_grid_block_index(self.h, ib, _ip(a))
        return a

    def x(self, ib, idim, i):
        return lib().orc_grid_x(self.h, ib, idim, i)

    def set_block(self, ib, w):
        w = np.ascontiguousarray(w, dtype=np.float64)
        lib().orc_grid_set_block(self.h, ib, _dp(w))

    def get_block(self, ib):
        w = np.zeros(self.shape, np.float64)
        lib().orc_grid_get_block(self.h, ib, _dp(w))
        return w

    def getbc(self):
        lib().orc_grid_getbc(self.h)

    def getdt(self):
        dt = ctypes.c_double(0)
        cm = ctypes.c_double(0)
        lib().orc_grid_getdt(self.h, ctypes.byref(dt), ctypes.byref(cm))
        return dt.value, cm.value

    def advance(self, dt, cmax_global=0.0, nthreads=0):
        return lib().orc_grid_advance(self.h, dt, cmax_global, nthreads)

    def volume_average(self, power):
        a = np.zeros(self.c.nw, np.float64)
        lib().orc_grid_volume_average(self.h, power, _dp(a))
        return a


def run_field_loop(c: OrcCfg, courantpar: float, time_max=0.5, dtsave=0.01, nthreads=0):
    ncol = 1 + 2 * (c.nw + 3)
    nmax = int(round(time_max / dtsave)) + 5
    rows = np.zeros((nmax, ncol), np.float64)
    n = lib().orc_run_field_loop(ctypes.byref(c), courantpar, time_max, dtsave, nmax, _dp(rows), nthreads)
    if n < 0:
        raise RuntimeError(f"oracle field loop crashed: status {-n}")
    return rows[:n]


def count_flops_stage(c, wct, wnew, qdt, dx, cmax_global=0.0):
    dxa = np.ascontiguousarray(np.asarray(dx, dtype=np.float64))
    return lib().orc_count_flops_stage(ctypes.byref(c), _dp(wct), _dp(wnew), qdt, _dp(dxa), cmax_global)


def count_flops_getdt(c, w, dx):
    dxa = np.ascontiguousarray(np.asarray(dx, dtype=np.float64))
    return lib().orc_count_flops_getdt(ctypes.byref(c), _dp(w), _dp(dxa))


def read_log(path):
    """Read a regression log (header lines start with # or !)."""
    rows = []
    with open(path) as f:
        for line in f:
            s = line.strip()
            if not s or s[0] in "#!":
                continue
            rows.append([float(v) for v in s.replace(",", " ").split()])
    return np.array(rows, np.float64)


def compare_logs(a: np.ndarray, b: np.ndarray, rtol=1.0e-5, atol=1.0e-8) -> bool:
    """compare_logs rule (tools/fortran/compare_logs.f:44-48)."""
    if a.shape != b.shape:
        return False
    return bool(np.all(np.abs(a - b) <= atol + 0.5 * rtol * (np.abs(a) + np.abs(b))))


def dual_run(c: OrcCfg, domain_nx, xprobmin, xprobmax, bc, w0, dw0, dgamma, dts, mask, nthreads=0,
             want_final=False):
    """Forward-mode reference gradient (orc_dual_run): loss = sum(mask * rho^2)
    after len(dts) SSP-RK3 steps with the frozen dt sequence, and its
    derivative along (dw0, dgamma).  w0, dw0: conserved block arrays
    (nblocks, nw, nz, ny, nx); mask: (nblocks, nz, ny, nx)."""
    nd = c.ndim
    dn = np.array(list(domain_nx) + [1] * (3 - nd), np.int32)
    xmn = np.array(list(xprobmin) + [0.0] * (3 - nd), np.float64)
    xmx = np.array(list(xprobmax) + [1.0] * (3 - nd), np.float64)
    bca = np.array([BC[b] if isinstance(b, str) else b for b in bc] + [0] * (6 - len(bc)), np.int32)
    w0 = np.ascontiguousarray(w0, np.float64)
    dw = None if dw0 is None else np.ascontiguousarray(dw0, np.float64)
    dts = np.ascontiguousarray(dts, np.float64)
    mask = np.ascontiguousarray(mask, np.float64)
    loss = ctypes.c_double()
    dloss = ctypes.c_double()
    wf = np.empty_like(w0) if want_final else None
    st = lib().orc_dual_run(ctypes.byref(c), _ip(dn), _dp(xmn), _dp(xmx), _ip(bca), _dp(w0),
                            _dp(dw) if dw is not None else None, float(dgamma), len(dts), _dp(dts), _dp(mask),
                            nthreads, ctypes.byref(loss), ctypes.byref(dloss), _dp(wf) if wf is not None else None)
    return (loss.value, dloss.value, st) + ((wf,) if want_final else ())


def lohner_block(c: OrcCfg, w, weight, logflag, wavefilter=1e-2, threshold=0.1, derefine=0.125, level=1,
                 refine_max_level=2):
    """Löhner error of one ghosted block: (error over the interior, refine, coarsen)."""
    w = np.ascontiguousarray(w, np.float64)
    wt = np.ascontiguousarray(weight, np.float64)
    lf = np.ascontiguousarray(logflag, np.int32)
    n = 1
    for d in range(c.ndim):
        n *= c.block_nx[d]
    err = np.zeros(n)
    r = ctypes.c_int()
    co = ctypes.c_int()
    lib().orc_lohner_block(ctypes.byref(c), _dp(w), _dp(wt), _ip(lf), wavefilter, threshold, derefine, level,
                           refine_max_level, _dp(err), ctypes.byref(r), ctypes.byref(co))
    return err, bool(r.value), bool(co.value)


class AmrGrid:
    """Static multi-level grid of the oracle: leaves [(level, ig0, ig1, ig2)],
    periodic boundaries, the reference's multi-level getbc and flux fix."""

    def __init__(self, c: OrcCfg, nbase, xprobmin, xprobmax, leaves, bc=None):
        self.c = c
        nd = c.ndim
        nb = np.array(list(nbase) + [1] * (3 - nd), np.int32)
        xmn = np.array(list(xprobmin) + [0.0] * (3 - nd), np.float64)
        xmx = np.array(list(xprobmax) + [1.0] * (3 - nd), np.float64)
        lv = np.ascontiguousarray(np.array([list(t) + [0] * (4 - len(t)) for t in leaves], np.int32).reshape(-1))
        bc = ["periodic"] * (2 * nd) if bc is None else list(bc)
        self.bca = np.array([BC[b] if isinstance(b, str) else b for b in bc] + [0] * (6 - len(bc)), np.int32)
        self.h = lib().orc_amr_create(ctypes.byref(c), _ip(nb), _dp(xmn), _dp(xmx), len(leaves), _ip(lv),
                                      _ip(self.bca))
        self.nblocks = len(leaves)
        self.shape = block_shape(c)

    def __del__(self):
        if getattr(self, "h", None):
            lib().orc_amr_destroy(self.h)
            self.h = None

    def neighbors(self):
        t = np.zeros(27 * self.nblocks, np.int32)
        i = np.zeros(27 * self.nblocks, np.int32)
        ch = np.zeros(27 * 8 * self.nblocks, np.int32)
        lib().orc_amr_neighbors(self.h, _ip(t), _ip(i), _ip(ch))
        return t.reshape(-1, 27), i.reshape(-1, 27), ch.reshape(-1, 27, 8)

    def set_block(self, b, w):
        lib().orc_amr_set_block(self.h, b, _dp(np.ascontiguousarray(w, np.float64)))

    def get_block(self, b, reg=0):
        w = np.zeros(self.shape, np.float64)
        lib().orc_amr_get_block(self.h, reg, b, _dp(w))
        return w

    def getbc(self):
        lib().orc_amr_getbc(self.h)

    def getdt(self):
        dt = ctypes.c_double()
        cm = ctypes.c_double()
        lib().orc_amr_getdt(self.h, ctypes.byref(dt), ctypes.byref(cm))
        return dt.value, cm.value

    def advect1(self, ra, rb, qdt, dtfactor=1.0, cmax_global=0.0, nthreads=0):
        return lib().orc_amr_advect1(self.h, ra, rb, qdt, dtfactor, cmax_global, nthreads)

    def combine_reg(self, dst, ca, ra, cb, rb):
        lib().orc_amr_combine_reg(self.h, dst, ca, ra, cb, rb)

    def advance(self, dt, cmax_global=0.0, nthreads=0):
        return lib().orc_amr_advance(self.h, dt, cmax_global, nthreads)

    def remap(self, leaves, ops):
        """The regridded grid (amr_coarsen_refine): new leaves, and per new
        leaf the op row of amrvac_b200.amr.ops; getbc is run on it."""
        lv = np.ascontiguousarray(np.array([list(t) + [0] * (4 - len(t)) for t in leaves], np.int32).reshape(-1))
        op = np.ascontiguousarray(np.asarray(ops, np.int32).reshape(-1))
        new = AmrGrid.__new__(AmrGrid)
        new.c = self.c
        new.bca = self.bca
        new.h = lib().orc_amr_remap(self.h, len(leaves), _ip(lv), _ip(op))
        new.nblocks = len(leaves)
        new.shape = self.shape
        lib().orc_amr_getbc(new.h)
        return new
