"""Known-answer accuracy pin of the oracle's MP5 and WENO5 restatements.

A density wave rho = 1 + 0.2 sin(2 pi x) advected at v = (1, 0) with
constant pressure is an exact solution of the Euler equations (translation);
starting from exact cell averages, a fifth-order reconstruction (MP5limiter,
src/limiter/mod_mp5.t:16-201: the (2, -13, 47, 27, -3)/60 interpolant with
its monotonicity limits inactive on smooth data) must cut the L1 error of the
cell averages by about 2^5 per doubling of the resolution when the time
error is small (CFL 0.1); so must the WENO5 family (WENO5limiter,
src/limiter/mod_weno.t:254-377: WENO-JS, WENO-Z, WENO-Z+).  WENO-YC3
(WENO3limiter var 2, mod_weno.t:165-252) is third order (2^3); the
Venkatakrishnan limiter (src/limiter/mod_venk.t) and the slope limiters stay
near second order.
"""
import numpy as np
import pytest

from tests import _problems as P


def _l1_error(O, n, limiter, nghost, cfl=0.1, tend=0.1, time_stepper="threestep"):
    c = O.make_cfg(physics="hd", ndim=2, gamma=1.4, flux_scheme="hll", limiter=limiter, nghost=nghost,
                   courantpar=cfl, time_stepper=time_stepper)
    x = (np.arange(n) + 0.5) / n
    X, _ = np.meshgrid(x, x, indexing="xy")
    k, h = 2.0 * np.pi, 1.0 / n
    sinc = np.sin(k * h / 2) / (k * h / 2)

    def cons_of(rho_avg):
        prim = np.zeros((4, 1, n, n))
        prim[0, 0] = rho_avg
        prim[1], prim[3] = 1.0, 1.0
        return P.prim_to_cons(prim, "hd", 2, 1.4)  # linear in rho at fixed v, p
    blocks = P.to_blocks(cons_of(1.0 + 0.2 * np.sin(k * X) * sinc), 2, nghost=nghost)
    g = O.Grid(c, [n, n], [0.0, 0.0], [1.0, 1.0], ["periodic"] * 4)
    for ib in range(g.nblocks):
        g.set_block(ib, blocks[ib])
    g.getbc()
    t = 0.0
    while t < tend - 1e-14:
        dt, cg = g.getdt()
        dt = min(dt, tend - t)
        g.advance(dt, cg)
        t += dt
    got = P.interior(np.array([g.get_block(ib) for ib in range(g.nblocks)]), 2, nghost=nghost)
    ex = P.interior(P.to_blocks(cons_of(1.0 + 0.2 * np.sin(k * (X - tend)) * sinc), 2, nghost=nghost), 2,
                    nghost=nghost)
    return float(np.abs(got[:, 0] - ex[:, 0]).mean())


@pytest.mark.parametrize("limiter,nghost,lo,hi", [("mp5", 3, 24.0, 40.0), ("weno5", 3, 24.0, 40.0),
                                                   ("wenoz5", 3, 24.0, 40.0), ("wenozp5", 3, 24.0, 40.0),
                                                   ("wenoyc3", 2, 6.5, 9.5), ("venk", 2, 3.8, 5.8),
                                                   ("minmod", 2, 2.5, 4.5)])
def test_convergence_order_on_smooth_wave(oracle_lib, limiter, nghost, lo, hi):
    e32 = _l1_error(oracle_lib, 32, limiter, nghost)
    e64 = _l1_error(oracle_lib, 64, limiter, nghost)
    assert lo < e32 / e64 < hi, (e32, e64, e32 / e64)


@pytest.mark.parametrize("time_stepper,lo,hi", [("fivestep", 24.0, 40.0), ("threestep", 8.0, 16.0)])
def test_fivestep_keeps_fifth_order_at_large_cfl(oracle_lib, time_stepper, lo, hi):
    """At CFL 0.9 the time error shows: SSP-RK3 (third order) falls to about
    2^3.8 per doubling with MP5, SSPRK(5,4) (fivestep, fourth order,
    src/mod_advance.t:513-557) keeps the spatial 2^5."""
    e32 = _l1_error(oracle_lib, 32, "mp5", 3, cfl=0.9, time_stepper=time_stepper)
    e64 = _l1_error(oracle_lib, 64, "mp5", 3, cfl=0.9, time_stepper=time_stepper)
    assert lo < e32 / e64 < hi, (e32, e64, e32 / e64)
