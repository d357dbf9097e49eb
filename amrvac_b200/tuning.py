"""Autotuner for the stage kernel's launch shape, with an on-disk cache.

Two knobs.  The work distribution: the 3-D stage kernel either runs one
wave of persistent CTAs marching plane ranges across blocks, or splits each
block into z-chunks of block_nx, block_nx/2 or block_nx/4 planes per CTA;
small chunks fill the last wave better (the number of blocks is rarely a
multiple of 2 x 148 CTAs) but repeat more z-faces and stage more halo
planes.  The kernel variant (amrvac_gpu_stage_variant): for the 3-D MHD
HLLD + cada3 + GLM scheme, threads per CTA (256 / 288), CTAs per SM the
registers are capped for (1 / 2 / 3 / 4) and the staging mode (gathered
loads, or asynchronous bulk copies of the next conserved plane).
``amrvac_gpu_autotune`` times one stage for every pair on the context's
current state; the best pair is cached per (physics, dimensions, solver,
limiter, bound speed, precision, block_nx, block count, device) in
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
            f"lim{c.limiter}|bs{c.typeboundspeed}|prec{c.precision}|bn{c.block_nx[0]}|nb{ctx.nblocks}")


def autotune(ctx, reps: int = 3, cache: bool = True):
    """Return (zchunk, ms_per_stage or None if taken from the cache); the
    chosen kernel variant is set on the context (ctx.stage_variant())."""
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
        ctx.set_stage_variant(int(table[key].get("variant", 0)))
        return int(table[key]["zchunk"]), None
    z = ctypes.c_int()
    ms = ctypes.c_double()
    _lib.check(ctx.L.amrvac_gpu_autotune(ctx.h, reps, ctypes.byref(z), ctypes.byref(ms)), "autotune")
    if cache:
        table[key] = {"zchunk": z.value, "variant": ctx.stage_variant()["variant"], "ms_per_stage": ms.value}
        try:
            os.makedirs(os.path.dirname(path), exist_ok=True)
            with open(path, "w") as f:
                json.dump(table, f, indent=1, sort_keys=True)
        except OSError:
            pass
    return z.value, ms.value
