"""CPU checks of the oracle's restatements of the split and TVD schemes.

The GPU tests compare the device against these restatements; here they are
checked on their own: conservation on a periodic domain (the flux form of
TVD-MUSCL's characteristic limiter, the Hancock predictor, the split sweeps),
the sweep order of typedimsplit ('xyyx' reverses on odd steps, 'xy' never
does, src/mod_advance.t:23-45), and that the split sweeps really are one
direction each (a field varying only along y is left unchanged by the x
sweep: the split step of such a field equals one y-only step).
"""
import numpy as np
import pytest

from tests import _problems as P


def _grid(O, kw, n=32, prim=None, bc=None):
    c = O.make_cfg(**kw)
    nd = kw["ndim"]
    ndir = kw.get("ndir", nd)
    if prim is None:
        prim = P.random_smooth(kw["physics"], nd, ndir, n, seed=P.SEED)
    blocks = P.to_blocks(P.prim_to_cons(prim, kw["physics"], ndir, c.gamma), nd)
    g = O.Grid(c, [n] * nd, [0.0] * nd, [1.0] * nd, bc or ["periodic"] * (2 * nd))
    for ib in range(g.nblocks):
        g.set_block(ib, blocks[ib])
    g.getbc()
    return g


def _state(g, nd):
    return P.interior(np.array([g.get_block(ib) for ib in range(g.nblocks)]), nd)


@pytest.mark.parametrize("kw", [
    dict(physics="hd", ndim=2, gamma=1.4, flux_scheme="tvdmu", limiter="albada", time_stepper="twostep",
         dimsplit=True),
    dict(physics="hd", ndim=3, gamma=1.4, flux_scheme="tvdmu", limiter="minmod", dimsplit=True),
    dict(physics="mhd", ndim=2, ndir=3, flux_scheme="tvdmu", limiter="vanleer", divb="none", time_stepper="twostep",
         dimsplit=True),
    dict(physics="hd", ndim=2, gamma=1.4, flux_scheme="tvdlf", limiter="koren", time_stepper="twostep"),
    dict(physics="hd", ndim=2, gamma=1.4, flux_scheme="hllc", limiter="mp5", nghost=3, time_stepper="fivestep"),
], ids=["hd2_tvdmu", "hd3_tvdmu", "mhd25_tvdmu", "hd2_hancock", "hd2_mp5_fivestep"])
def test_schemes_conserve_on_a_periodic_domain(oracle_lib, kw):
    O = oracle_lib
    nd = kw["ndim"]
    n = 16 if nd == 3 else 32
    prim = P.random_smooth(kw["physics"], nd, kw.get("ndir", nd), n, seed=P.SEED)
    c = O.make_cfg(**kw)
    ng = c.nghost
    blocks = P.to_blocks(P.prim_to_cons(prim, kw["physics"], kw.get("ndir", nd), c.gamma), nd, nghost=ng)
    g = O.Grid(c, [n] * nd, [0.0] * nd, [1.0] * nd, ["periodic"] * (2 * nd))
    for ib in range(g.nblocks):
        g.set_block(ib, blocks[ib])
    g.getbc()
    w0 = P.interior(np.array([g.get_block(ib) for ib in range(g.nblocks)]), nd, nghost=ng)
    for _ in range(3):
        dt, cg = g.getdt()
        g.advance(dt, cg)
    w1 = P.interior(np.array([g.get_block(ib) for ib in range(g.nblocks)]), nd, nghost=ng)
    assert np.isfinite(w1).all()
    before, after = w0.sum(axis=(0, 2, 3, 4)), w1.sum(axis=(0, 2, 3, 4))
    scale = np.abs(w1).sum(axis=(0, 2, 3, 4))
    assert np.all(np.abs(after - before) <= 1e-13 * scale), (after - before) / scale


def test_sweep_order_xyyx_and_xy(oracle_lib):
    """First step: both orders sweep x then y (identical).  Second step:
    'xyyx' sweeps y then x, 'xy' again x then y (different)."""
    O = oracle_lib
    base = dict(physics="hd", ndim=2, gamma=1.4, flux_scheme="hll", limiter="minmod", dimsplit=True)
    ga = _grid(O, dict(base, typedimsplit="xyyx"))
    gb = _grid(O, dict(base, typedimsplit="xy"))
    for step in range(2):
        dt, cg = ga.getdt()
        ga.advance(dt, cg)
        gb.advance(dt, cg)
        a, b = _state(ga, 2), _state(gb, 2)
        if step == 0:
            assert np.array_equal(a, b)
        else:
            assert np.abs(a - b).max() > 1e-10


def test_x_sweep_leaves_a_y_only_field_alone(oracle_lib):
    """rho, p vary with y only and the velocity is along y: the x sweep sees
    no gradients, so the split step equals the unsplit step of the same
    field (which then has no x fluxes either) to rounding."""
    O = oracle_lib
    n = 32
    y = (np.arange(n) + 0.5) / n
    prim = np.zeros((4, 1, n, n))
    prim[0, 0] = (1.0 + 0.3 * np.sin(2 * np.pi * y))[:, None]
    prim[2, 0] = (0.2 * np.cos(2 * np.pi * y))[:, None]
    prim[3, 0] = (1.0 + 0.1 * np.cos(4 * np.pi * y))[:, None]
    base = dict(physics="hd", ndim=2, gamma=1.4, flux_scheme="hllc", limiter="vanleer")
    gs = _grid(O, dict(base, dimsplit=True), prim=prim.copy())
    gu = _grid(O, base, prim=prim.copy())
    dt, cg = gu.getdt()
    gs.advance(dt, cg)
    gu.advance(dt, cg)
    a, b = _state(gs, 2), _state(gu, 2)
    assert np.abs(a - b).max() <= 1e-13 * np.abs(b).max()
    assert np.abs(a - _state(_grid(O, base, prim=prim.copy()), 2)).max() > 1e-6  # the y sweep did work
