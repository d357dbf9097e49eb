"""Autotuner for the stage-kernel tiling, with an on-disk cache.

The 3-D stage kernel splits each 16^3 block into z-chunks of 16, 8 or 4
planes per CTA.  Small chunks fill the last wave of CTAs better (the number
of blocks is rarely a multiple of 2 x 148 CTAs) but repeat more z-faces and
stage more halo planes.  ``amrvac_gpu_autotune`` times one stage for each
candidate on the context's current state; the best value is cached per
(physics, dimensions, solver, limiter, bound speed, block count, device) in
``$AMRVAC_TUNE_CACHE`` (default ``~/.cache/amrvac_b200/tune.json``).
"""
from __future__ import annotations

import ctypes
import json
import os

from . import _lib


def _cache_path() -> str:
    return os.environ.get("AMRVAC_TUNE_CACHE",
                          os.path.join(os.path.expanduser("~"), ".cache", "amrvac_b200", "tune.json"))


def _key(ctx) -> str:
    c = ctx.cfg
    dev = "gpu"
    try:
        import torch
        if torch.cuda.is_available():
            dev = torch.cuda.get_device_name(torch.cuda.current_device()).replace(" ", "_")
    except Exception:
        pass
    return (f"{dev}|phys{c.physics}|nd{c.ndim}|ndir{c.ndir}|divb{c.typedivbfix}|fs{c.flux_scheme}|"
            f"lim{c.limiter}|bs{c.typeboundspeed}|nb{ctx.nblocks}")


def autotune(ctx, reps: int = 3, cache: bool = True):
    """Return (zchunk, ms_per_stage or None if taken from the cache)."""
    path = _cache_path()
    key = _key(ctx)
    table = {}
    if cache and os.path.exists(path):
        try:
            with open(path) as f:
                table = json.load(f)
        except (OSError, ValueError):
            table = {}
    if cache and key in table:
        ctx.set_zchunk(int(table[key]["zchunk"]))
        return int(table[key]["zchunk"]), None
    z = ctypes.c_int()
    ms = ctypes.c_double()
    _lib.check(ctx.L.amrvac_gpu_autotune(ctx.h, reps, ctypes.byref(z), ctypes.byref(ms)), "autotune")
    if cache:
        table[key] = {"zchunk": z.value, "ms_per_stage": ms.value}
        try:
            os.makedirs(os.path.dirname(path), exist_ok=True)
            with open(path, "w") as f:
                json.dump(table, f, indent=1, sort_keys=True)
        except OSError:
            pass
    return z.value, ms.value
