"""2-D Euler blast wave of the adjoint workload (test and benchmark input).

Domain [0, 1]^2 with `cont` boundaries, gamma = 1.4, v = 0; density
rho = 1 + 0.1 G with G a unit-variance Gaussian random field of correlation
length 0.05 (seeded white noise convolved with a Gaussian kernel through the
FFT); pressure 0.1, and 10 inside the disk r < 0.1 around the centre.  The
loss is the sum of rho^2 over the cells whose centres lie in the annulus
0.25 < r < 0.35 at the final time.
"""
from __future__ import annotations

import numpy as np

from tests import _problems as P

SEED = 20261203
GAMMA = 1.4
R_IN, R_OUT = 0.25, 0.35


def gaussian_field(n, corr=0.05, seed=SEED):
    rng = np.random.default_rng(seed)
    noise = rng.standard_normal((n, n))
    k = 2.0 * np.pi * np.fft.fftfreq(n, d=1.0 / n)
    kx, ky = np.meshgrid(k, k, indexing="xy")
    filt = np.exp(-0.5 * (kx ** 2 + ky ** 2) * corr ** 2)
    g = np.real(np.fft.ifft2(np.fft.fft2(noise) * filt))
    g -= g.mean()
    return g / g.std()


def centres(n):
    x = (np.arange(n) + 0.5) / n
    return np.meshgrid(x, x, indexing="xy")  # [y][x]


def blast_prim(n, seed=SEED):
    """Primitive fields [4][1][n][n]: rho, vx, vy, p."""
    X, Y = centres(n)
    r = np.hypot(X - 0.5, Y - 0.5)
    prim = np.zeros((4, 1, n, n))
    prim[0, 0] = 1.0 + 0.1 * gaussian_field(n, seed=seed)
    prim[3, 0] = np.where(r < 0.1, 10.0, 0.1)
    return prim


def loss_mask(n):
    X, Y = centres(n)
    r = np.hypot(X - 0.5, Y - 0.5)
    return ((r > R_IN) & (r < R_OUT)).astype(np.float64)


def to_cons_blocks(prim, gamma=GAMMA):
    cons = P.prim_to_cons(prim, "hd", 2, gamma)
    return P.to_blocks(cons, 2)


def mask_blocks(n):
    return P.to_blocks(loss_mask(n)[None, None], 2)[:, 0]


def cons_direction(prim, drho, dgamma, gamma=GAMMA):
    """Derivative of the conserved initial blocks along (drho, dgamma) with
    v = 0: d rho = drho, d m = 0, d e = -p / (gamma-1)^2 dgamma."""
    d = np.zeros_like(prim)
    d[0, 0] = drho
    d[3, 0] = -prim[3, 0] / (gamma - 1.0) ** 2 * dgamma
    return P.to_blocks(d, 2)
