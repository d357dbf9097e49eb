"""amrvac_gpu_getdt_noalloc against amrvac_gpu_getdt.

The no-allocation entry point serves host codes that may not call cudaMalloc
themselves (their device memory belongs to another runtime, such as OpenACC
data regions or a framework's caching allocator), so they cannot create a
context.  It must give the same dt and cmax_global as the context's getdt on
the same blocks, and the oracle's getdt_courant on the same state.  Two
calls in a row on different block sets check that nothing from the previous
call's scratch leaks into the next.  This file is named to be collected last.
"""
import ctypes

import numpy as np
import pytest

from tests import _problems as P

pytestmark = pytest.mark.gpu

RTOL = 1e-12

CASES = [
    ("mhd3_glm", dict(physics="mhd", ndim=3, flux_scheme="hlld", limiter="cada3", typedivbfix="glm"), 48, 11),
    ("mhd3_glm_summax", dict(physics="mhd", ndim=3, flux_scheme="hlld", limiter="cada3", typedivbfix="glm",
                             typecourant="summax"), 32, 12),
    ("hd2", dict(physics="hd", ndim=2, gamma=1.4, flux_scheme="hllc", limiter="vanleer"), 64, 13),
    ("hd2_minimum", dict(physics="hd", ndim=2, gamma=1.4, flux_scheme="hllc", limiter="vanleer",
                         typecourant="minimum"), 32, 14),
    ("mhd25_linde", dict(physics="mhd", ndim=2, ndir=3, flux_scheme="hll", limiter="cada3", typedivbfix="linde"),
     48, 15),
]


def _cuda():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")


def _context(kw, n, seed, amp):
    from amrvac_b200 import Context, make_cfg
    ndim = kw["ndim"]
    ndir = kw.get("ndir", ndim)
    cfg = make_cfg(**kw)
    prim = P.random_smooth(kw["physics"], ndim, ndir, n, seed=seed, glm=kw.get("typedivbfix") == "glm", amp=amp)
    cons = P.prim_to_cons(prim, kw["physics"], ndir, cfg.gamma)
    ctx = Context(cfg)
    lo, hi = [0.0] * ndim, [1.0 + 0.25 * d for d in range(ndim)]
    ctx.set_uniform_grid([n] * ndim, lo, hi)
    blocks = P.to_blocks(cons, ndim)
    ctx.upload(blocks)
    dx = np.zeros((ctx.nblocks, 3))
    for d in range(ndim):
        dx[:, d] = (hi[d] - lo[d]) / n
    ctx.case = (kw, n, lo, hi, blocks)
    return cfg, ctx, dx


def _oracle_getdt(O, ctx):
    """getdt_courant of the oracle (src/mod_dt.t:160-287) on the same blocks."""
    kw, n, lo, hi, blocks = ctx.case
    k = dict(kw)
    div = k.pop("typedivbfix", "none")
    tc = {"maxsum": 1, "summax": 2, "minimum": 3}[k.pop("typecourant", "maxsum")]
    c = O.make_cfg(divb=div, type_courant=tc, **k)
    nd = kw["ndim"]
    g = O.Grid(c, [n] * nd, lo, hi, ["periodic"] * (2 * nd))
    for ib in range(g.nblocks):
        g.set_block(ib, blocks[ib])
    g.getbc()
    return g.getdt()


def _noalloc(cfg, ctx, dx, stream):
    from amrvac_b200 import _lib
    L = _lib.load()
    dt = ctypes.c_double(-1.0)
    cm = ctypes.c_double(-1.0)
    rc = L.amrvac_gpu_getdt_noalloc(ctypes.byref(cfg), ctypes.c_void_p(ctx.register_ptr("ps")), ctx.nblocks,
                                    dx.ctypes.data_as(ctypes.POINTER(ctypes.c_double)), ctypes.c_void_p(stream),
                                    ctypes.byref(dt), ctypes.byref(cm))
    assert rc >= 0, L.amrvac_gpu_last_error()
    return dt.value, cm.value, rc


def _close(a, b):
    return abs(a - b) <= RTOL * max(abs(a), abs(b))


@pytest.mark.parametrize("name,kw,n,seed", CASES, ids=[c[0] for c in CASES])
def test_noalloc_getdt_matches_context_getdt_twice(oracle_lib, name, kw, n, seed):
    _cuda()
    # first a larger block set, then a smaller one on the same domain (coarser
    # cells, so smaller courant numbers): stale per-block partials left by the
    # first call would raise the second call's maximum
    cfg1, ctx1, dx1 = _context(kw, n, seed, amp=0.25)
    cfg2, ctx2, dx2 = _context(kw, n // 2 if n >= 64 else 16, seed + 100, amp=0.1)
    assert ctx2.nblocks < ctx1.nblocks
    for cfg, ctx, dx, stream in ((cfg1, ctx1, dx1, ctx1.stream_ptr()), (cfg2, ctx2, dx2, 0)):
        dt_ref, cm_ref, st_ref = ctx.getdt()
        dt, cm, st = _noalloc(cfg, ctx, dx, stream)
        assert _close(dt, dt_ref) and _close(cm, cm_ref), (name, dt, dt_ref, cm, cm_ref)
        assert st == st_ref
        dt_o, cm_o = _oracle_getdt(oracle_lib, ctx)
        assert _close(dt, dt_o) and _close(cm, cm_o), (name, "oracle", dt, dt_o, cm, cm_o)
        assert 0.0 < dt < 1.0e99


def test_noalloc_getdt_refuses_too_many_blocks():
    _cuda()
    from amrvac_b200 import _lib, make_cfg
    L = _lib.load()
    cfg = make_cfg(physics="hd", ndim=2, gamma=1.4)
    dummy = (ctypes.c_double * 3)()
    dt = ctypes.c_double()
    cm = ctypes.c_double()
    # refused by the size check, before either pointer is used
    rc = L.amrvac_gpu_getdt_noalloc(ctypes.byref(cfg), ctypes.cast(dummy, ctypes.c_void_p), 32768 + 1,
                                    ctypes.cast(dummy, ctypes.POINTER(ctypes.c_double)), None,
                                    ctypes.byref(dt), ctypes.byref(cm))
    assert rc == _lib.E_ARG
    assert b"AMRVAC_NOALLOC_MAX_BLOCKS" in L.amrvac_gpu_last_error()
