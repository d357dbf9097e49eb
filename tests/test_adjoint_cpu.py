"""Reference gradient of the adjoint workload, without a GPU.

The forward-mode (dual-number) run of the oracle is the reference gradient
for the GPU discrete adjoint.  Here it is pinned against central finite
differences of the oracle's own FP64 runs on a small blast wave: along a
random density direction and along gamma, with the dt sequence of the
unperturbed run held fixed (the differentiated map is the scheme at frozen
time steps).
"""
import numpy as np
import pytest

from tests import _blast as B

N = 32
NSTEPS = 20  # the blast reaches the loss annulus
# central-difference steps: small enough not to cross limiter or upwind
# kinks of the perturbed cells (a random density direction moves every cell),
# large enough to stay above roundoff of the loss (about 200)
EPS_RHO = 1e-7
EPS_GAMMA = 1e-6
RTOL_FD = 1e-6
BC = ["cont"] * 4


def _cfg(O, gamma=B.GAMMA, fs="hll", lim="minmod"):
    return O.make_cfg(physics="hd", ndim=2, gamma=gamma, flux_scheme=fs, limiter=lim, courantpar=0.8)


def _dts(O, c, w0, nsteps):
    g = O.Grid(c, [N, N], [0.0, 0.0], [1.0, 1.0], BC)
    for ib in range(g.nblocks):
        g.set_block(ib, w0[ib])
    g.getbc()
    out = []
    for _ in range(nsteps):
        dt, _ = g.getdt()
        g.advance(dt)
        out.append(dt)
    return np.array(out)


@pytest.mark.parametrize("fs,lim", [("hll", "minmod"), ("hll", "vanleer"), ("hllc", "minmod"),
                                    ("hllc", "vanleer")])
def test_dual_gradient_matches_central_differences(oracle_lib, fs, lim):
    O = oracle_lib
    prim = B.blast_prim(N)
    c = _cfg(O, fs=fs, lim=lim)
    w0 = B.to_cons_blocks(prim)
    dts = _dts(O, c, w0, NSTEPS)
    mask = B.mask_blocks(N)
    rng = np.random.default_rng(11)
    drho = rng.standard_normal((N, N))
    # density direction
    dw = B.cons_direction(prim, drho, 0.0)
    L, dL, st = O.dual_run(c, [N, N], [0.0, 0.0], [1.0, 1.0], BC, w0, dw, 0.0, dts, mask)
    assert st == 0 and np.isfinite(dL)
    eps = EPS_RHO
    Lp = O.dual_run(c, [N, N], [0.0, 0.0], [1.0, 1.0], BC, w0 + eps * dw, None, 0.0, dts, mask)[0]
    Lm = O.dual_run(c, [N, N], [0.0, 0.0], [1.0, 1.0], BC, w0 - eps * dw, None, 0.0, dts, mask)[0]
    fd = (Lp - Lm) / (2 * eps)
    assert abs(fd - dL) <= RTOL_FD * abs(dL), (fd, dL)
    # gamma: the scheme's gamma and the initial energy e = p/(gamma-1) both move
    dwg = B.cons_direction(prim, np.zeros((N, N)), 1.0)
    _, dLg, _ = O.dual_run(c, [N, N], [0.0, 0.0], [1.0, 1.0], BC, w0, dwg, 1.0, dts, mask)
    epg = EPS_GAMMA
    vals = []
    for sgn in (1.0, -1.0):
        g = B.GAMMA + sgn * epg
        vals.append(O.dual_run(_cfg(O, gamma=g, fs=fs, lim=lim), [N, N], [0.0, 0.0], [1.0, 1.0], BC,
                               B.to_cons_blocks(prim, g), None, 0.0, dts, mask)[0])
    fdg = (vals[0] - vals[1]) / (2 * epg)
    assert abs(fdg - dLg) <= RTOL_FD * abs(dLg), (fdg, dLg)


def test_dual_value_equals_the_fp64_oracle(oracle_lib):
    """The dual run's value part is the plain FP64 oracle run, bit for bit."""
    O = oracle_lib
    prim = B.blast_prim(N)
    c = _cfg(O)
    w0 = B.to_cons_blocks(prim)
    dts = _dts(O, c, w0, 3)
    _, _, _, wf = O.dual_run(c, [N, N], [0.0, 0.0], [1.0, 1.0], BC, w0, None, 0.0, dts, B.mask_blocks(N),
                             want_final=True)
    g = O.Grid(c, [N, N], [0.0, 0.0], [1.0, 1.0], BC)
    for ib in range(g.nblocks):
        g.set_block(ib, w0[ib])
    g.getbc()
    for dt in dts:
        g.advance(dt)
    ref = np.array([g.get_block(ib) for ib in range(g.nblocks)])
    assert np.array_equal(wf, ref)
