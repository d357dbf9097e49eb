"""ctypes binding of libamrvac_gpu.so (C ABI in include/amrvac_gpu.h).

The shared library is built in-tree by ``python -m amrvac_b200.build``.  There
is no fallback: if the library is missing or cannot be loaded, importing the
product API raises, and a context cannot be created without a CUDA device.
"""
from __future__ import annotations

import ctypes
import os

HERE = os.path.dirname(os.path.abspath(__file__))
# AMRVAC_GPU_LIB selects another build of the same library (e.g. a tuning variant).
LIB_PATH = os.environ.get("AMRVAC_GPU_LIB", os.path.join(HERE, "libamrvac_gpu.so"))
HEADER = os.path.join(os.path.dirname(HERE), "include", "amrvac_gpu.h")

MAX_NW = 16

E_ARG, E_UNSUPPORTED, E_CUDA, E_STATE = -1, -2, -3, -4
ST_SMALL_VALUE, ST_NAN, ST_DT_TOO_SMALL = 1, 2, 4

FS = {"tvdlf": 1, "hll": 2, "hllc": 3, "hlld": 4, "tvdmu": 5}
LIMITER = {"minmod": 1, "woodward": 2, "mcbeta": 3, "superbee": 4, "vanleer": 5,
           "albada": 6, "koren": 7, "cada": 8, "cada3": 9, "schmid1": 10, "schmid2": 10, "venk": 11, "mp5": 13,
           "weno3": 14, "wenoyc3": 15,
           "weno5": 16, "wenoz5": 18, "wenozp5": 20}
BOUNDSPEED = {"Einfeldt": 1, "cmaxmean": 2, "cmaxleftright": 3}
DIVB = {"none": 0, "glm": 1, "linde": 4}
COURANT = {"maxsum": 1, "summax": 2, "minimum": 3}
BC = {"periodic": 0, "cont": 1, "symm": 2, "asymm": 3}
TIME_STEPPER = {"onestep": 1, "twostep": 2, "threestep": 3, "fourstep": 4, "fivestep": 5}
TIME_INTEGRATOR = {"default": 0, "Predictor_Corrector": 0, "ssprk5": 0, "ssprk4": 0, "ssprk3": 0, "Forward_Euler": 0, "rk4": 1,
                   "ssprk2": 2}
PRECISION = {"fp64": 0, "mixed": 1}


class AmrvacCfg(ctypes.Structure):
    """Mirror of ``amrvac_cfg`` (field order and types must match the header)."""

    _fields_ = [
        ("ndim", ctypes.c_int), ("ndir", ctypes.c_int), ("physics", ctypes.c_int),
        ("block_nx", ctypes.c_int * 3), ("nghostcells", ctypes.c_int),
        ("gamma", ctypes.c_double),
        ("flux_scheme", ctypes.c_int), ("limiter", ctypes.c_int),
        ("typeboundspeed", ctypes.c_int), ("typedivbfix", ctypes.c_int),
        ("mhd_glm_alpha", ctypes.c_double), ("mhd_glm_extended", ctypes.c_int),
        ("divbdiff", ctypes.c_double), ("courantpar", ctypes.c_double),
        ("type_courant", ctypes.c_int), ("cada3_radius", ctypes.c_double),
        ("tvdlfeps", ctypes.c_double), ("fix_small_values", ctypes.c_int),
        ("check_small_values", ctypes.c_int), ("small_values_method", ctypes.c_int),
        ("small_density", ctypes.c_double), ("small_pressure", ctypes.c_double),
        ("time_stepper", ctypes.c_int), ("ssprk_order", ctypes.c_int),
        ("dtmin", ctypes.c_double),
        ("typeboundary", (ctypes.c_int * MAX_NW) * 6),
        ("zchunk", ctypes.c_int),
        ("precision", ctypes.c_int),
        ("slowsteps", ctypes.c_int),
        ("time_integrator", ctypes.c_int),
        ("dimsplit", ctypes.c_int),
        ("schmid_rad", ctypes.c_double * 3),
        ("schmid_global", ctypes.c_int),
        ("small_values_daverage", ctypes.c_int),
    ]


class AmrvacEnsInstance(ctypes.Structure):
    """Mirror of ``amrvac_ens_instance``."""

    _fields_ = [
        ("ndim", ctypes.c_int), ("domain_nx", ctypes.c_int * 2),
        ("xprobmin", ctypes.c_double * 2), ("xprobmax", ctypes.c_double * 2),
        ("flux_scheme", ctypes.c_int), ("limiter", ctypes.c_int),
        ("time_max", ctypes.c_double),
    ]


# (name, restype, argtypes) for every function declared in the header.
_P = ctypes.POINTER
_d, _i, _u32, _i64, _vp = ctypes.c_double, ctypes.c_int, ctypes.c_uint32, ctypes.c_int64, ctypes.c_void_p
_dp, _ip = _P(ctypes.c_double), _P(ctypes.c_int)
_cfgp = _P(AmrvacCfg)
SIGNATURES = [
    ("amrvac_gpu_default_cfg", None, [_cfgp]),
    ("amrvac_gpu_nw", _i, [_cfgp]),
    ("amrvac_gpu_create", _i, [_cfgp, _P(_vp)]),
    ("amrvac_gpu_destroy", _i, [_vp]),
    ("amrvac_gpu_set_blocks", _i, [_vp, _i, _dp, _ip]),
    ("amrvac_gpu_set_uniform_grid", _i, [_vp, _ip, _dp, _dp]),
    ("amrvac_gpu_nblocks", _i, [_vp]),
    ("amrvac_gpu_set_amr_grid", _i, [_vp, _i, _ip, _ip, _dp, _dp]),
    ("amrvac_gpu_amr_slots", _i, [_vp]),
    ("amrvac_gpu_amr_regrid", _i, [_vp, _i, _ip, _ip]),
    ("amrvac_gpu_amr_resettree", _i, [_vp, _dp, _ip, _i, _dp, _dp, _dp, _ip]),
    ("amrvac_gpu_amr_leaves", _i, [_vp, _ip]),
    ("amrvac_amr_plan", _i, [_i, _ip, _ip, _i, _i, _ip, _P(ctypes.c_ubyte), _P(ctypes.c_ubyte), _i, _ip, _ip, _ip]),
    ("amrvac_gpu_amr_kernel_ms", _i, [_vp, _i, _dp, _dp]),
    ("amrvac_gpu_upload", _i, [_vp, _i, _i, _i, _dp]),
    ("amrvac_gpu_download", _i, [_vp, _i, _i, _i, _dp]),
    ("amrvac_gpu_getdt", _i, [_vp, _i, _dp, _dp]),
    ("amrvac_gpu_getdt_noalloc", _i, [_cfgp, _vp, _i, _dp, _vp, _dp, _dp]),
    ("amrvac_gpu_advect1", _i, [_vp, _i, _i, _i, _d, _d, _d, _d]),
    ("amrvac_gpu_advect1_dim", _i, [_vp, _i, _i, _i, _d, _d, _d, _d, _i]),
    ("amrvac_gpu_set_cmax_global", _i, [_vp, _d]),
    ("amrvac_gpu_set_time", _i, [_vp, _d, _d, _d]),
    ("amrvac_gpu_step", _i, [_vp]),
    ("amrvac_gpu_run", _i, [_vp, _i]),
    ("amrvac_gpu_get_time", _i, [_vp, _dp, _dp, _dp]),
    ("amrvac_gpu_run_timed", _i, [_vp, _i, _dp, _dp, _dp]),
    ("amrvac_gpu_fp64_peak", _i, [_dp]),
    ("amrvac_gpu_wait_probe", _i, [_i, _P(_u32)]),
    ("amrvac_gpu_autotune", _i, [_vp, _i, _ip, _dp]),
    ("amrvac_gpu_set_zchunk", _i, [_vp, _i]),
    ("amrvac_gpu_set_stage_variant", _i, [_vp, _i]),
    ("amrvac_gpu_stage_variant", _i, [_vp, _ip, _ip, _ip, _ip, _ip]),
    ("amrvac_gpu_status", _i, [_vp, _P(_u32)]),
    ("amrvac_gpu_clear_status", _i, [_vp]),
    ("amrvac_gpu_synchronize", _i, [_vp]),
    ("amrvac_gpu_stream", _i, [_vp, _P(_vp)]),
    ("amrvac_gpu_register_ptr", _i, [_vp, _i, _P(_dp)]),
    ("amrvac_gpu_launch_count", _i64, [_vp]),
    ("amrvac_gpu_last_error", ctypes.c_char_p, []),
    ("amrvac_gpu_get_flux_points", _i, [_vp, _i, _dp, _dp, _i, _d, _dp]),
    ("amrvac_gpu_get_cbounds_points", _i, [_vp, _i, _dp, _dp, _dp, _dp, _i, _dp, _dp]),
    ("amrvac_gpu_riemann_points", _i, [_vp, _i, _dp, _dp, _i, _d, _dp]),
    ("amrvac_gpu_div_points", _i, [_i, _dp, _dp, _dp, _dp, _dp]),
    ("amrvac_gpu_srl_maps", _i, [_i, _i, _ip, _ip, _ip, _ip]),
    ("amrvac_gpu_lohner", _i, [_vp, _i, _dp, _ip, _i, _dp, _dp, _dp, _ip, _ip, _dp]),
    ("amrvac_gpu_step_dt", _i, [_vp, _d]),
    ("amrvac_gpu_register_copy", _i, [_vp, _i, _vp, _i]),
    ("amrvac_gpu_step_dt_states", _i, [_vp, _d, _vp, _vp, _vp, _vp]),
    ("amrvac_gpu_adjoint_step", _i, [_vp, _vp, _d, _vp]),
    ("amrvac_gpu_adjoint_step_states", _i, [_vp, _vp, _vp, _vp, _vp, _d, _vp]),
    ("amrvac_ens_create", _i, [_cfgp, _i, _P(AmrvacEnsInstance), _P(_vp)]),
    ("amrvac_ens_destroy", _i, [_vp]),
    ("amrvac_ens_nblocks", _i, [_vp, _i]),
    ("amrvac_ens_upload", _i, [_vp, _i, _dp]),
    ("amrvac_ens_download", _i, [_vp, _i, _dp]),
    ("amrvac_ens_reset_time", _i, [_vp]),
    ("amrvac_ens_step", _i, [_vp]),
    ("amrvac_ens_run", _i, [_vp, _i, _i, _ip, _ip]),
    ("amrvac_ens_state", _i, [_vp, _dp, _dp, _ip, _ip]),
    ("amrvac_ens_status", _i, [_vp, _P(_u32), _P(_u32)]),
    ("amrvac_ens_set_grid", _i, [_vp, _i]),
    ("amrvac_ens_grid", _i, [_vp, _ip, _ip]),
    ("amrvac_ens_autotune", _i, [_vp, _i, _ip, _dp]),
    ("amrvac_ens_set_variant", _i, [_vp, _i]),
    ("amrvac_ens_variant", _i, [_vp, _ip, _ip, _ip]),
    ("amrvac_ens_stream", _i, [_vp, _P(_vp)]),
    ("amrvac_ens_launch_count", _i64, [_vp]),
]

_lib = None


def load() -> ctypes.CDLL:
    """Load the in-tree library; raise if it has not been built."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError(
                f"{LIB_PATH} not found: build it with `python -m amrvac_b200.build` "
                "(nvcc, sm_100a). There is no CPU fallback.")
        L = ctypes.CDLL(LIB_PATH)
        for name, res, args in SIGNATURES:
            fn = getattr(L, name)
            fn.restype = res
            fn.argtypes = args
        _lib = L
    return _lib


class AmrvacError(RuntimeError):
    def __init__(self, code: int, where: str):
        msg = load().amrvac_gpu_last_error().decode(errors="replace")
        super().__init__(f"{where} failed with code {code}: {msg}")
        self.code = code


def check(code: int, where: str) -> int:
    """Raise on configuration errors (negative codes); return status bits."""
    if code < 0:
        raise AmrvacError(code, where)
    return code
