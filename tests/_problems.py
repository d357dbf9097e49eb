"""Seeded initial conditions used by the parity tests and the benchmark.

All builders return primitive interior fields on the whole uniform domain,
indexed [var][z][y][x]; ``to_blocks`` cuts them into the Fortran block arrays
w(ixG^S,1:nw) (ghost cells zero; getbc fills them).  Values come from
SplitMix64 keyed by (seed, global cell index), so they do not depend on the
block layout.
"""
from __future__ import annotations

import numpy as np

SEED = 20261203


def splitmix_uniform(seed: int, idx: np.ndarray, stream: int = 0) -> np.ndarray:
    """U(0,1) from SplitMix64 of (seed, stream, idx)."""
    with np.errstate(over="ignore"):
        z = (np.uint64(seed) * np.uint64(0x9E3779B97F4A7C15)
             + np.uint64(stream) * np.uint64(0xD1B54A32D192ED03)
             + idx.astype(np.uint64) * np.uint64(0x9E3779B97F4A7C15))
        z = (z ^ (z >> np.uint64(30))) * np.uint64(0xBF58476D1CE4E5B9)
        z = (z ^ (z >> np.uint64(27))) * np.uint64(0x94D049BB133111EB)
        z = z ^ (z >> np.uint64(31))
    return (z >> np.uint64(11)).astype(np.float64) * (1.0 / 9007199254740992.0)


def cell_centres(domain_nx, xprobmin, xprobmax):
    """Cell-centre coordinates per dimension (src/amr/mod_amr_solution_node.t:164)."""
    xs = []
    for n, a, b in zip(domain_nx, xprobmin, xprobmax):
        dx = (b - a) / n
        xs.append(a + (np.arange(n) + 0.5) * dx)
    return xs


def prim_to_cons(prim: np.ndarray, physics: str, ndir: int, gamma: float) -> np.ndarray:
    """hd_to_conserved / mhd_to_conserved_origin on whole fields (numpy)."""
    w = prim.copy()
    rho = prim[0]
    v = prim[1:1 + ndir]
    p = prim[ndir + 1]
    v2 = sum(v[c] * v[c] for c in range(ndir))
    ig1 = 1.0 / (gamma - 1.0)
    if physics == "mhd":
        b = prim[ndir + 2:2 * ndir + 2]
        b2 = sum(b[c] * b[c] for c in range(ndir))
        w[ndir + 1] = p * ig1 + 0.5 * (v2 * rho + b2)
    else:
        w[ndir + 1] = p * ig1 + 0.5 * v2 * rho
    for c in range(ndir):
        w[1 + c] = rho * v[c]
    return w


def kh_2d(n=256, seed=SEED, gamma=1.4):
    """Kelvin-Helmholtz 2-D: [0,1]x[-0.5,0.5], rho=2 inside |y|<0.25."""
    x, y = cell_centres([n, n], [0.0, -0.5], [1.0, 0.5])
    X, Y = np.meshgrid(x, y, indexing="xy")
    inside = np.abs(Y) < 0.25
    prim = np.zeros((4, n, n))
    prim[0] = np.where(inside, 2.0, 1.0)
    prim[1] = np.where(inside, 0.5, -0.5)
    idx = np.arange(n * n).reshape(n, n)
    prim[2] = 0.01 * (2.0 * splitmix_uniform(seed, idx) - 1.0)
    prim[3] = 2.5
    return prim[:, None], dict(domain_nx=[n, n], xprobmin=[0.0, -0.5], xprobmax=[1.0, 0.5])


def orszag_tang_3d(n=128, seed=SEED, gamma=5.0 / 3.0, glm=True):
    """3-D Orszag-Tang on [0,2pi]^3 with 1e-3 seeded velocity noise."""
    L = 2.0 * np.pi
    x, y, z = cell_centres([n, n, n], [0.0] * 3, [L] * 3)
    Z, Y, X = np.meshgrid(z, y, x, indexing="ij")
    nw = 9 if glm else 8
    prim = np.zeros((nw, n, n, n))
    prim[0] = 25.0 / (36.0 * np.pi)
    idx = np.arange(n ** 3).reshape(n, n, n)
    prim[1] = -np.sin(Z) + 1e-3 * (2 * splitmix_uniform(seed, idx, 1) - 1)
    prim[2] = np.sin(X) + 1e-3 * (2 * splitmix_uniform(seed, idx, 2) - 1)
    prim[3] = 1e-3 * (2 * splitmix_uniform(seed, idx, 3) - 1)
    prim[4] = 5.0 / (12.0 * np.pi)
    b0 = 1.0 / np.sqrt(4.0 * np.pi)
    prim[5] = -np.sin(Z) * b0
    prim[6] = np.sin(2.0 * X) * b0
    prim[7] = 0.0
    return prim, dict(domain_nx=[n, n, n], xprobmin=[0.0] * 3, xprobmax=[L] * 3)


def random_smooth(physics, ndim, ndir, n, seed=SEED, glm=False, amp=0.3):
    """Smooth positive random fields for stage parity (sum of seeded modes)."""
    rng = np.random.default_rng(seed)
    shape = [n] * ndim
    grids = np.meshgrid(*[np.arange(n) / n for _ in range(ndim)], indexing="ij")[::-1]
    def field(base, a):
        f = np.full(shape[::-1], base, dtype=np.float64)
        for _ in range(4):
            k = rng.integers(1, 4, size=ndim)
            ph = rng.uniform(0, 2 * np.pi)
            arg = sum(2 * np.pi * k[d] * grids[d] for d in range(ndim)) + ph
            f = f + a * rng.uniform(0.2, 1.0) * np.sin(arg)
        return f
    nw = (2 * ndir + 2 + (1 if glm else 0)) if physics == "mhd" else ndir + 2
    prim = np.zeros((nw,) + tuple(shape[::-1]))
    prim[0] = field(1.0, amp)
    for c in range(ndir):
        prim[1 + c] = field(0.0, 0.5)
    prim[ndir + 1] = field(1.0, amp)
    if physics == "mhd":
        for c in range(ndir):
            prim[ndir + 2 + c] = field(0.0, 0.4)
        if glm:
            prim[2 * ndir + 2] = field(0.0, 0.05)
    while prim.ndim < 4:
        prim = prim[:, None]
    return prim


def to_blocks(cons: np.ndarray, ndim: int, nghost: int = 2, bn: int = 16) -> np.ndarray:
    """Cut a [nw][nz][ny][nx] field into ghosted block arrays, x-fastest order."""
    nw, nz, ny, nx = cons.shape
    nb = [nx // bn, ny // bn if ndim >= 2 else 1, nz // bn if ndim >= 3 else 1]
    g = [bn + 2 * nghost if d < ndim else 1 for d in range(3)]
    out = np.zeros((nb[0] * nb[1] * nb[2], nw, g[2], g[1], g[0]))
    ng = [nghost if d < ndim else 0 for d in range(3)]
    for kb in range(nb[2]):
        for jb in range(nb[1]):
            for ib in range(nb[0]):
                b = ib + nb[0] * (jb + nb[1] * kb)
                sz = slice(kb * bn, (kb + 1) * bn) if ndim >= 3 else slice(0, 1)
                sy = slice(jb * bn, (jb + 1) * bn) if ndim >= 2 else slice(0, 1)
                sx = slice(ib * bn, (ib + 1) * bn)
                out[b, :, ng[2]:ng[2] + (bn if ndim >= 3 else 1), ng[1]:ng[1] + (bn if ndim >= 2 else 1),
                    ng[0]:ng[0] + bn] = cons[:, sz, sy, sx]
    return out


def interior(blocks: np.ndarray, ndim: int, nghost: int = 2) -> np.ndarray:
    ng = [nghost if d < ndim else 0 for d in range(3)]
    return blocks[:, :, ng[2]:blocks.shape[2] - ng[2], ng[1]:blocks.shape[3] - ng[1],
                  ng[0]:blocks.shape[4] - ng[0]]


# ---------------------------------------------------------------- field loop
# tests/mhd/field_loop_2.5D/mod_usr.t (reference): iprob=1, A0=1e-3, R0=0.3,
# v0=(2,1), B from the vector potential by central differences.
FL = dict(domain_nx=[128, 64], xprobmin=[-1.0, -0.5], xprobmax=[1.0, 0.5])


def _fl_block_x(ib, nb, dx, xmin, ng=2, bn=16):
    ig = [ib % nb[0], ib // nb[0]]
    out = []
    for d in range(2):
        rxmin = xmin[d] + ig[d] * bn * dx[d]
        out.append(rxmin + (np.arange(bn + 2 * ng) + 1 - ng - 0.5) * dx[d])
    return out


def fl_bfield(ib, t, ng=2):
    """Analytic (Bx, By) on the ghosted block ib at time t (interior valid)."""
    dn, xmn, xmx = FL["domain_nx"], FL["xprobmin"], FL["xprobmax"]
    dx = [(xmx[d] - xmn[d]) / dn[d] for d in range(2)]
    nb = [dn[0] // 16, dn[1] // 16]
    xs, ys = _fl_block_x(ib, nb, dx, xmn, ng)
    X, Y = np.meshgrid(xs, ys, indexing="xy")
    x1 = X - 2.0 * t - xmn[0]
    x1 = xmn[0] + (x1 - np.floor(x1 / (xmx[0] - xmn[0])) * (xmx[0] - xmn[0]))
    x2 = Y - 1.0 * t - xmn[1]
    x2 = xmn[1] + (x2 - np.floor(x2 / (xmx[1] - xmn[1])) * (xmx[1] - xmn[1]))
    r2 = x1 * x1 + x2 * x2
    az = np.where(r2 < 0.3 * 0.3, 1.0e-3 * (0.3 - np.sqrt(r2)), 0.0)
    bx = np.zeros_like(az)
    by = np.zeros_like(az)
    bx[1:-1, :] = ((az[2:, :] - az[:-2, :]) * 0.5) / dx[1]
    by[:, 1:-1] = -(((az[:, 2:] - az[:, :-2]) * 0.5) / dx[0])
    return bx, by


def field_loop_blocks(ng=2):
    """Conserved ghosted blocks (nw=9 with GLM psi, or 8) for the field loop."""
    dn = FL["domain_nx"]
    nb = (dn[0] // 16) * (dn[1] // 16)
    out = []
    for ib in range(nb):
        bx, by = fl_bfield(ib, 0.0, ng)
        w = np.zeros((9, 1, 16 + 2 * ng, 16 + 2 * ng))
        w[0, 0, ng:ng + 16, ng:ng + 16] = 1.0
        w[1, 0, ng:ng + 16, ng:ng + 16] = 2.0
        w[2, 0, ng:ng + 16, ng:ng + 16] = 1.0
        w[4, 0, ng:ng + 16, ng:ng + 16] = 1.0
        w[5, 0, ng:ng + 16, ng:ng + 16] = bx[ng:ng + 16, ng:ng + 16]
        w[6, 0, ng:ng + 16, ng:ng + 16] = by[ng:ng + 16, ng:ng + 16]
        out.append(w)
    prim = np.array(out)
    cons = prim.copy()
    rho, v, p, b = prim[:, 0], prim[:, 1:4], prim[:, 4], prim[:, 5:8]
    v2 = v[:, 0] ** 2 + v[:, 1] ** 2 + v[:, 2] ** 2
    b2 = b[:, 0] ** 2 + b[:, 1] ** 2 + b[:, 2] ** 2
    cons[:, 4] = p * 1.5 + 0.5 * (v2 * rho + b2)
    for c in range(3):
        cons[:, 1 + c] = rho * v[:, c]
    return cons


def field_loop_log_row(blocks, t, nwflux, ng=2):
    """One regression-log row: time, mean(w), mean(w**2) over flux vars and
    the extra output variables divb-2, divb-4, B_err (set_output_vars)."""
    dn, xmn, xmx = FL["domain_nx"], FL["xprobmin"], FL["xprobmax"]
    dx = [(xmx[d] - xmn[d]) / dn[d] for d in range(2)]
    s1 = np.zeros(nwflux + 3)
    s2 = np.zeros(nwflux + 3)
    n = 0
    I = slice(ng, ng + 16)
    for ib in range(blocks.shape[0]):
        w = blocks[ib, :, 0]
        bxw, byw = w[5], w[6]
        d2 = (0.5 * (bxw[I, ng + 1:ng + 17] - bxw[I, ng - 1:ng + 15]) * (1.0 / dx[0])
              + 0.5 * (byw[ng + 1:ng + 17, I] - byw[ng - 1:ng + 15, I]) * (1.0 / dx[1]))
        d4 = ((-bxw[I, ng + 2:ng + 18] + 8.0 * bxw[I, ng + 1:ng + 17] - 8.0 * bxw[I, ng - 1:ng + 15]
               + bxw[I, ng - 2:ng + 14]) / (12.0 * dx[0])
              + (-byw[ng + 2:ng + 18, I] + 8.0 * byw[ng + 1:ng + 17, I] - 8.0 * byw[ng - 1:ng + 15, I]
                 + byw[ng - 2:ng + 14, I]) / (12.0 * dx[1]))
        bx, by = fl_bfield(ib, t, ng)
        berr = np.sqrt((bxw[I, I] - bx[I, I]) ** 2 + (byw[I, I] - by[I, I]) ** 2)
        vals = [w[v][I, I] for v in range(nwflux)] + [d2, d4, berr]
        for q, a in enumerate(vals):
            s1[q] += a.sum()
            s2[q] += (a * a).sum()
        n += 256
    return np.concatenate([[t], s1 / n, s2 / n])
