"""Par-file namelist reader and mapping to ``amrvac_cfg``.

Reads the reference's Fortran namelist par files (``&methodlist``,
``&boundlist``, ``&meshlist``, ``&paramlist``, ``&stoplist``, ``&savelist``,
``&hd_list`` / ``&mhd_list``; read_par_files in src/io/mod_input_output.t:
173-1687) and fills the C configuration with the same defaults
(src/io/mod_input_output.t:284-480, src/hd/mod_hd_phys.t:66-81,
src/mhd/mod_mhd_phys.t:13-268).  Later files override earlier ones, as with
``amrvac -i a.par b.par``.
"""
from __future__ import annotations

import re
from dataclasses import dataclass, field

from . import _lib

_TOKEN = re.compile(r"""('[^']*'|"[^"]*"|[^,\s]+)""")


def _parse_value(tok: str):
    t = tok.strip()
    if not t:
        return None
    if t[0] in "'\"":
        return t[1:-1]
    low = t.lower()
    if low in (".true.", "t", "true", ".t."):
        return True
    if low in (".false.", "f", "false", ".f."):
        return False
    num = low.replace("d", "e")
    try:
        if re.fullmatch(r"[+-]?\d+", num):
            return int(num)
        return float(num)
    except ValueError:
        return t


def _expand(values: str):
    out = []
    for tok in _TOKEN.findall(values):
        m = re.fullmatch(r"(\d+)\*(.+)", tok)
        if m:
            out.extend([_parse_value(m.group(2))] * int(m.group(1)))
        else:
            out.append(_parse_value(tok))
    return out


def parse_namelists(text: str) -> dict:
    """Return {list_name: {key: value-or-list}} from namelist text."""
    lists: dict = {}
    text = re.sub(r"!.*", "", text)
    for m in re.finditer(r"&(\w+)(.*?)(?:^\s*/\s*$|/\s*$)", text, re.S | re.M):
        name = m.group(1).lower()
        body = m.group(2)
        d = lists.setdefault(name, {})
        parts = re.split(r"(\b[\w%]+(?:\(\s*[\d:,\s]+\))?)\s*=", body)
        for i in range(1, len(parts) - 1, 2):
            key = parts[i].strip().lower()
            vals = _expand(parts[i + 1].strip().rstrip(","))
            km = re.fullmatch(r"(\w+)\(\s*(\d+)\s*\)", key)
            if km:
                base, idx = km.group(1), int(km.group(2))
                arr = d.setdefault(base, {})
                if isinstance(arr, dict):
                    arr[idx] = vals[0] if len(vals) == 1 else vals
                continue
            d[key] = vals[0] if len(vals) == 1 else vals
    return lists


def read_par_files(paths) -> dict:
    merged: dict = {}
    for p in paths:
        with open(p) as f:
            nl = parse_namelists(f.read())
        for name, kv in nl.items():
            merged.setdefault(name, {}).update(kv)
    return merged


def _first(v):
    return v[0] if isinstance(v, list) else v


@dataclass
class RunConfig:
    """Everything a standalone run needs beyond ``amrvac_cfg``."""

    cfg: _lib.AmrvacCfg
    domain_nx: list = field(default_factory=list)
    xprobmin: list = field(default_factory=list)
    xprobmax: list = field(default_factory=list)
    time_max: float = 1.0e99
    it_max: int = 2 ** 62
    dtsave_log: float = 0.0
    physics: str = "hd"


# small_values_method names in the order of amrvac_cfg.small_values_method
# (src/mod_small_values.t:9)
SMALL_VALUES_METHODS = ("error", "replace", "average")


def make_cfg(*, physics="hd", ndim=2, ndir=None, gamma=None, flux_scheme="tvdlf",
             limiter="minmod", typeboundspeed="Einfeldt", typedivbfix=None,
             mhd_glm_alpha=0.5, mhd_glm_extended=True, divbdiff=0.8, courantpar=0.8,
             typecourant="maxsum", cada3_radius=0.1, tvdlfeps=1.0, fix_small_values=False,
             check_small_values=True, small_values_method="error", small_density=0.0,
             small_pressure=0.0, time_stepper="threestep", ssprk_order=3, dtmin=1.0e-10,
             typeboundary=None, zchunk=0, precision="fp64", slowsteps=-1,
             time_integrator="default", nghostcells=None, dimsplit=False,
             typedimsplit="xyyx", schmid_rad=(1.0, 1.0, 1.0), block_nx=16,
             small_values_daverage=1) -> _lib.AmrvacCfg:
    """Build an ``amrvac_cfg`` from reference-style parameter names.

    typeboundary: list of 2*ndim entries (min1, max1, min2, ...), each a name
    applied to all variables or a list of per-variable names.  nghostcells
    defaults to 3 for the fifth-order reconstructions (mp5, weno5, wenoz5,
    wenozp5: they need them) and 2 otherwise.  block_nx: cells per block
    edge, the same in every direction (the library runs 8, 10, 12, 16, 32).
    """
    L = _lib.load()
    c = _lib.AmrvacCfg()
    L.amrvac_gpu_default_cfg(c)
    c.ndim = ndim
    c.ndir = ndim if ndir is None else ndir
    c.physics = 1 if physics == "mhd" else 0
    for d in range(3):
        c.block_nx[d] = int(block_nx)
    c.gamma = (5.0 / 3.0) if gamma is None else float(gamma)
    c.flux_scheme = _lib.FS[flux_scheme]
    c.limiter = _lib.LIMITER[limiter]
    five = limiter in ("mp5", "weno5", "wenoz5", "wenozp5")
    c.nghostcells = int(nghostcells) if nghostcells is not None else (3 if five else 2)
    c.typeboundspeed = _lib.BOUNDSPEED[typeboundspeed]
    if typedivbfix is None:
        typedivbfix = "linde" if physics == "mhd" else "none"
    c.typedivbfix = _lib.DIVB[typedivbfix] if (physics == "mhd" and ndim > 1) else 0
    c.mhd_glm_alpha = mhd_glm_alpha
    c.mhd_glm_extended = int(mhd_glm_extended)
    c.divbdiff = divbdiff
    c.courantpar = courantpar
    c.type_courant = _lib.COURANT[typecourant]
    c.cada3_radius = cada3_radius
    c.tvdlfeps = tvdlfeps
    c.fix_small_values = int(fix_small_values)
    c.check_small_values = int(check_small_values)
    if small_values_method not in SMALL_VALUES_METHODS:
        raise ValueError(f"small_values_method {small_values_method!r}: the library runs "
                         f"{', '.join(SMALL_VALUES_METHODS)}")
    c.small_values_method = SMALL_VALUES_METHODS.index(small_values_method)
    c.small_density = small_density
    c.small_pressure = small_pressure
    c.time_stepper = _lib.TIME_STEPPER[time_stepper]
    c.ssprk_order = ssprk_order
    c.dtmin = dtmin
    c.zchunk = zchunk
    c.precision = _lib.PRECISION[precision]
    c.slowsteps = int(slowsteps)
    c.time_integrator = _lib.TIME_INTEGRATOR[time_integrator]
    c.dimsplit = 0 if not dimsplit else (2 if typedimsplit == "xy" else 1)
    for d in range(3):
        c.schmid_rad[d] = float(schmid_rad[d])
    c.schmid_global = int(limiter == "schmid1")
    c.small_values_daverage = int(small_values_daverage)
    nw = L.amrvac_gpu_nw(c)
    tb = typeboundary or ["periodic"] * (2 * ndim)
    for s in range(6):
        for v in range(_lib.MAX_NW):
            c.typeboundary[s][v] = 0
        if s < 2 * ndim:
            spec = tb[s]
            for v in range(nw):
                name = spec[v] if isinstance(spec, (list, tuple)) else spec
                c.typeboundary[s][v] = _lib.BC[name]
    return c


def config_from_par(paths) -> RunConfig:
    """Translate par files into a RunConfig (the subset the path reads)."""
    nl = read_par_files(paths)
    meth = nl.get("methodlist", {})
    mesh = nl.get("meshlist", {})
    bound = nl.get("boundlist", {})
    param = nl.get("paramlist", {})
    stop = nl.get("stoplist", {})
    save = nl.get("savelist", {})
    physics = "mhd" if "mhd_list" in nl else "hd"
    plist = nl.get("mhd_list" if physics == "mhd" else "hd_list", {})
    ndim = 1 + sum(1 for k in ("domain_nx2", "domain_nx3") if k in mesh)
    domain_nx = [int(mesh.get(f"domain_nx{d + 1}", 32)) for d in range(ndim)]
    # block_nx1..3 (default 16, src/io/mod_input_output.t:301); the library
    # needs the same edge in every direction
    bnxs = [int(mesh.get(f"block_nx{d + 1}", 16)) for d in range(ndim)]
    if len(set(bnxs)) != 1:
        raise ValueError("block_nx must be the same in every direction for the B200 path")
    bnx = bnxs[0]
    tb = []
    for d in range(ndim):
        for side in ("min", "max"):
            v = bound.get(f"typeboundary_{side}{d + 1}", "periodic")
            tb.append(v if isinstance(v, list) else [v])
    ts = _first(meth.get("time_stepper", "twostep"))
    integ = _first(meth.get("time_integrator", None))
    if ts == "twostep" and integ not in (None, "ssprk2", "Predictor_Corrector"):
        raise ValueError(f"time_integrator {integ} not supported")
    if ts == "threestep" and integ not in (None, "ssprk3"):
        raise ValueError(f"time_integrator {integ} not supported")
    if ts == "fourstep" and integ not in (None, "ssprk4", "rk4"):
        raise ValueError(f"time_integrator {integ} not supported")
    if ts == "fivestep" and integ not in (None, "ssprk5"):
        raise ValueError(f"time_integrator {integ} not supported")
    cfg_kw = dict(
        physics=physics, ndim=ndim,
        gamma=plist.get(f"{physics}_gamma", None),
        flux_scheme=_first(meth.get("flux_scheme", "tvdlf")),
        limiter=_first(meth.get("limiter", "minmod")),
        typeboundspeed=meth.get("typeboundspeed", "Einfeldt"),
        courantpar=float(param.get("courantpar", 0.8)),
        typecourant=param.get("typecourant", "maxsum"),
        slowsteps=int(param.get("slowsteps", -1)),
        cada3_radius=float(meth.get("cada3_radius", 0.1)),
        tvdlfeps=float(meth.get("tvdlfeps", 1.0)),
        fix_small_values=bool(meth.get("fix_small_values", False)),
        check_small_values=bool(meth.get("check_small_values", True)),
        small_values_method=meth.get("small_values_method", "error"),
        small_values_daverage=int(meth.get("small_values_daverage", 1)),
        small_density=float(meth.get("small_density", 0.0)),
        small_pressure=float(meth.get("small_pressure", 0.0)),
        time_stepper=ts,
        ssprk_order=int(meth.get("ssprk_order", 3)),
        time_integrator=integ or "default",
        nghostcells=int(mesh["nghostcells"]) if "nghostcells" in mesh else None,
        dimsplit=bool(meth.get("dimsplit", False)),
        schmid_rad=tuple(float(meth.get(f"schmid_rad{d + 1}", 1.0)) for d in range(3)),
        typedimsplit=meth.get("typedimsplit", "xyyx"),
        block_nx=bnx,
    )
    if physics == "mhd":
        cfg_kw.update(typedivbfix=plist.get("typedivbfix", "linde"),
                      mhd_glm_alpha=float(plist.get("mhd_glm_alpha", 0.5)),
                      mhd_glm_extended=bool(plist.get("mhd_glm_extended", True)),
                      divbdiff=float(plist.get("divbdiff", 0.8)))
        ndir = 3 if any(isinstance(v, str) and "2.5" in v for v in nl.get("usr", {}).values()) else ndim
        cfg_kw["ndir"] = ndir
    names = [t if len(t) > 1 else t[0] for t in tb]
    cfg = make_cfg(typeboundary=names, **cfg_kw)
    return RunConfig(
        cfg=cfg, domain_nx=domain_nx,
        xprobmin=[float(mesh.get(f"xprobmin{d + 1}", 0.0)) for d in range(ndim)],
        xprobmax=[float(mesh.get(f"xprobmax{d + 1}", 1.0)) for d in range(ndim)],
        time_max=float(stop.get("time_max", 1.0e99)),
        it_max=int(stop.get("it_max", 2 ** 62)),
        dtsave_log=float(save.get("dtsave_log", 0.0)),
        physics=physics)
