"""Riemann-problem inputs for the batched-ensemble path, and the exact solution.

``exact_riemann`` is the exact solution of the 1-D Euler Riemann problem for
an ideal gas, written from the method in E. F. Toro, "Riemann Solvers and
Numerical Methods for Fluid Dynamics" (3rd ed., 2009), chapter 4: the star
pressure is the root of f_L(p) + f_R(p) + (u_R - u_L) = 0 (shock branch
eq. 4.6/4.7, rarefaction branch eq. 4.6/4.7), found by Newton iteration from
the primitive-variable guess, then the solution is sampled along x/t.  It is
the analytic reference of the reference's 1-D analytic test
(tests/hd/analytic_test_1d: RMSE of density against the exact solution).

``ensemble_specs`` draws the seeded ensemble of independent Riemann problems:
half 1-D with n = 16*round(logU(64, 4096)/16) cells, half 2-D with square
domains of side 16*round(logU(32, 512)/16); left/right rho, p ~ logU(0.1, 10),
normal velocity ~ U(-2, 2), interface position x0 ~ U(0.3, 0.7) on [0, 1]
(2-D: a planar interface through (x0, 0.5) with normal angle ~ U(-pi/6, pi/6));
HLL or HLLC and minmod or vanleer per instance.  Draws whose states would
open a vacuum (2/(gamma-1)(c_L + c_R) <= 1.5 (u_R - u_L)) are redrawn.
"""
from __future__ import annotations

import numpy as np

from tests import _problems as P

SEED = 20261203


# ---------------------------------------------------------------- exact solution
def _fk(p, rho, pk, ck, g):
    """Toro's f_K(p) and its derivative for one side."""
    if p > pk:  # shock
        a = 2.0 / ((g + 1.0) * rho)
        b = (g - 1.0) / (g + 1.0) * pk
        s = np.sqrt(a / (p + b))
        return (p - pk) * s, s * (1.0 - 0.5 * (p - pk) / (b + p))
    # rarefaction
    r = p / pk
    f = 2.0 * ck / (g - 1.0) * (r ** ((g - 1.0) / (2.0 * g)) - 1.0)
    df = 1.0 / (rho * ck) * r ** (-(g + 1.0) / (2.0 * g))
    return f, df


def star_state(rl, ul, pl, rr, ur, pr, g):
    """(p*, u*) of the exact Riemann solution."""
    cl, cr = np.sqrt(g * pl / rl), np.sqrt(g * pr / rr)
    if 2.0 / (g - 1.0) * (cl + cr) <= ur - ul:
        raise ValueError("vacuum is generated")
    # primitive-variable (linearised) guess, kept positive
    p = max(1e-8, 0.5 * (pl + pr) - 0.125 * (ur - ul) * (rl + rr) * (cl + cr))
    for _ in range(100):
        fl, dl = _fk(p, rl, pl, cl, g)
        fr, dr = _fk(p, rr, pr, cr, g)
        pn = p - (fl + fr + ur - ul) / (dl + dr)
        pn = max(pn, 1e-10)
        if abs(pn - p) <= 1e-14 * (pn + p):
            p = pn
            break
        p = pn
    fl, _ = _fk(p, rl, pl, cl, g)
    fr, _ = _fk(p, rr, pr, cr, g)
    return p, 0.5 * (ul + ur) + 0.5 * (fr - fl)


def exact_riemann(rl, ul, pl, rr, ur, pr, g, xi):
    """Sample (rho, u, p) at the similarity coordinates xi = (x - x0)/t."""
    ps, us = star_state(rl, ul, pl, rr, ur, pr, g)
    cl, cr = np.sqrt(g * pl / rl), np.sqrt(g * pr / rr)
    gm = (g - 1.0) / (g + 1.0)
    out = np.zeros((3, len(xi)))
    for n, s in enumerate(np.asarray(xi, dtype=np.float64)):
        if s <= us:  # left of the contact
            if ps > pl:  # left shock
                sl = ul - cl * np.sqrt((g + 1.0) / (2.0 * g) * ps / pl + (g - 1.0) / (2.0 * g))
                st = (rl, ul, pl) if s <= sl else (rl * (ps / pl + gm) / (gm * ps / pl + 1.0), us, ps)
            else:  # left rarefaction
                csl = cl * (ps / pl) ** ((g - 1.0) / (2.0 * g))
                if s <= ul - cl:
                    st = (rl, ul, pl)
                elif s >= us - csl:
                    st = (rl * (ps / pl) ** (1.0 / g), us, ps)
                else:  # inside the fan
                    f = 2.0 / (g + 1.0) + gm / cl * (ul - s)
                    st = (rl * f ** (2.0 / (g - 1.0)), 2.0 / (g + 1.0) * (cl + (g - 1.0) / 2.0 * ul + s),
                          pl * f ** (2.0 * g / (g - 1.0)))
        else:  # right of the contact
            if ps > pr:  # right shock
                sr = ur + cr * np.sqrt((g + 1.0) / (2.0 * g) * ps / pr + (g - 1.0) / (2.0 * g))
                st = (rr, ur, pr) if s >= sr else (rr * (ps / pr + gm) / (gm * ps / pr + 1.0), us, ps)
            else:  # right rarefaction
                csr = cr * (ps / pr) ** ((g - 1.0) / (2.0 * g))
                if s >= ur + cr:
                    st = (rr, ur, pr)
                elif s <= us + csr:
                    st = (rr * (ps / pr) ** (1.0 / g), us, ps)
                else:
                    f = 2.0 / (g + 1.0) - gm / cr * (ur - s)
                    st = (rr * f ** (2.0 / (g - 1.0)), 2.0 / (g + 1.0) * (-cr + (g - 1.0) / 2.0 * ur + s),
                          pr * f ** (2.0 * g / (g - 1.0)))
        out[:, n] = st
    return out


# ---------------------------------------------------------------- ensemble inputs
def _logu(rng, a, b):
    return float(np.exp(rng.uniform(np.log(a), np.log(b))))


def ensemble_specs(n_inst, seed=SEED, gamma=1.4, n1=(64, 4096), n2=(32, 512), time_max=0.2,
                   schemes=(("hll", "minmod"), ("hll", "vanleer"), ("hllc", "minmod"), ("hllc", "vanleer"))):
    rng = np.random.default_rng(seed)
    specs = []
    for k in range(n_inst):
        ndim = 1 if k % 2 == 0 else 2
        if ndim == 1:
            nx = int(16 * max(1, round(_logu(rng, *n1) / 16)))
            shape = (nx,)
        else:
            s = int(16 * max(1, round(_logu(rng, *n2) / 16)))
            shape = (s, s)
        while True:
            rl, pl, rr, pr = (_logu(rng, 0.1, 10.0) for _ in range(4))
            ul, ur = rng.uniform(-2.0, 2.0), rng.uniform(-2.0, 2.0)
            cl, cr = np.sqrt(gamma * pl / rl), np.sqrt(gamma * pr / rr)
            if 2.0 / (gamma - 1.0) * (cl + cr) > 1.5 * (ur - ul):
                break
        x0 = rng.uniform(0.3, 0.7)
        theta = rng.uniform(-np.pi / 6, np.pi / 6) if ndim == 2 else 0.0
        fs, lim = schemes[int(rng.integers(len(schemes)))]
        specs.append(dict(ndim=ndim, shape=shape, rl=rl, ul=ul, pl=pl, rr=rr, ur=ur, pr=pr, x0=x0,
                          theta=theta, flux_scheme=fs, limiter=lim, time_max=time_max))
    return specs


def initial_prim(spec):
    """Primitive fields [nw][1][ny][nx] (1-D: ny = 1) of one instance on [0, 1]^d."""
    ndim = spec["ndim"]
    if ndim == 1:
        nx = spec["shape"][0]
        x = (np.arange(nx) + 0.5) / nx
        left = x < spec["x0"]
        prim = np.zeros((3, 1, 1, nx))
        prim[0, 0, 0] = np.where(left, spec["rl"], spec["rr"])
        prim[1, 0, 0] = np.where(left, spec["ul"], spec["ur"])
        prim[2, 0, 0] = np.where(left, spec["pl"], spec["pr"])
        return prim
    ny, nx = spec["shape"][1], spec["shape"][0]
    x = ((np.arange(nx) + 0.5) / nx)[None, :]
    y = ((np.arange(ny) + 0.5) / ny)[:, None]
    c, s = np.cos(spec["theta"]), np.sin(spec["theta"])
    left = (x - spec["x0"]) * c + (y - 0.5) * s < 0.0
    vn = np.where(left, spec["ul"], spec["ur"])
    prim = np.zeros((4, 1, ny, nx))
    prim[0, 0] = np.where(left, spec["rl"], spec["rr"])
    prim[1, 0] = vn * c
    prim[2, 0] = vn * s
    prim[3, 0] = np.where(left, spec["pl"], spec["pr"])
    return prim


def initial_blocks(spec, gamma, nghost=2):
    prim = initial_prim(spec)
    cons = P.prim_to_cons(prim, "hd", spec["ndim"], gamma)
    return P.to_blocks(cons, spec["ndim"], nghost)


def instance(spec):
    from amrvac_b200 import Instance
    nd = spec["ndim"]
    return Instance(ndim=nd, domain_nx=tuple(spec["shape"]), xprobmin=(0.0,) * nd, xprobmax=(1.0,) * nd,
                    flux_scheme=spec["flux_scheme"], limiter=spec["limiter"], time_max=spec["time_max"])
