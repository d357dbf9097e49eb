"""The algorithmic flop counts quoted by bench.py come from the oracle.

Counting scalar: +,-,*,/,sqrt,exp count 1 each (the oracle never contracts to
FMA).  Halo overhead of the oracle's own array sweeps is removed by
Richardson extrapolation in the block size: count(2N) * 2 - count(N).
"""
import numpy as np
import pytest

from tests import _problems as P


def _count(O, physics, ndim, ndir, bn, **kw):
    c = O.make_cfg(physics=physics, ndim=ndim, ndir=ndir, block_nx=bn, **kw)
    prim = P.random_smooth(physics, ndim, ndir, bn, glm=kw.get("divb") == "glm")
    cons = P.prim_to_cons(prim, physics, ndir, c.gamma)
    blocks = P.to_blocks(cons, ndim, bn=bn)
    g = O.Grid(c, [bn] * ndim, [0] * ndim, [1] * ndim, ["periodic"] * (2 * ndim))
    g.set_block(0, blocks[0])
    g.getbc()
    w = g.get_block(0)
    dt, cg = g.getdt()
    return O.count_flops_stage(c, w, w.copy(), dt, g.dx(), cg), O.count_flops_getdt(c, w, g.dx())


@pytest.mark.parametrize("wl,args,sizes", [
    ("ot128", ("mhd", 3, 3), (32, 64)),
    ("kh256", ("hd", 2, 2), (128, 256)),
    ("amrblast3d", ("mhd", 3, 3), (32, 64)),
])
def test_alg_flops_constants(oracle_lib, wl, args, sizes):
    import bench
    kw = dict(flux_scheme="hlld", limiter="vanleer" if wl == "amrblast3d" else "cada3", divb="glm") \
        if args[0] == "mhd" else dict(flux_scheme="hllc", limiter="vanleer", gamma=1.4)
    a = _count(oracle_lib, *args, sizes[0], **kw)
    b = _count(oracle_lib, *args, sizes[1], **kw)
    stage = 2 * b[0] - a[0]
    getdt = 2 * b[1] - a[1]
    assert abs(stage - bench.ALG_FLOPS[wl]["stage"]) <= 0.01 * stage
    assert abs(getdt - bench.ALG_FLOPS[wl]["getdt"]) <= 0.02 * getdt
