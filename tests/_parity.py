"""The per-cell parity measure shared by the GPU tests, smoke() and bench.py.

For each variable v with scale M_v = max |ref_v| and floor tau_v = 1e-3 M_v:

* cells with |ref| >= tau_v are judged by the true relative error
  |got - ref| / |ref|;
* cells with |ref| < tau_v (momenta and field components near a zero
  crossing, psi near zero) are judged on the absolute scale tau_v:
  |got - ref| / tau_v.

``percell_err`` returns the larger of the two maxima, so ``err <= rtol``
asserts both bars at once; ``percell_parts`` returns them separately.  A
non-finite value on either side is never a match.
"""
from __future__ import annotations

import numpy as np

FLOOR = 1.0e-3


def percell_parts(got: np.ndarray, ref: np.ndarray, var_axis: int = 1, floor: float = FLOOR):
    """(max relative error over cells >= floor*max, max |diff| / (floor*max) over the rest).

    ``var_axis`` is the axis of the variables: 1 for a stack of blocks
    (block, var, z, y, x), 0 for one block (var, z, y, x)."""
    got = np.asarray(got, np.float64)
    ref = np.asarray(ref, np.float64)
    if got.shape != ref.shape:
        raise ValueError(f"shape mismatch {got.shape} vs {ref.shape}")
    if not (np.isfinite(got).all() and np.isfinite(ref).all()):
        return float("inf"), float("inf")
    ax = var_axis
    g = np.moveaxis(got, ax, 0).reshape(got.shape[ax], -1)
    r = np.moveaxis(ref, ax, 0).reshape(ref.shape[ax], -1)
    rel, small = 0.0, 0.0
    tau_all = floor * float(np.abs(r).max())
    for v in range(g.shape[0]):
        tau = floor * float(np.abs(r[v]).max())
        d = np.abs(g[v] - r[v])
        big = np.abs(r[v]) >= tau
        if tau == 0.0:  # zero everywhere in the reference: the scale of all variables
            if d.max() > 0.0:
                small = max(small, float(d.max() / tau_all) if tau_all > 0.0 else float("inf"))
            continue
        if big.any():
            rel = max(rel, float((d[big] / np.abs(r[v][big])).max()))
        if (~big).any():
            small = max(small, float(d[~big].max() / tau))
    return rel, small


def percell_err(got: np.ndarray, ref: np.ndarray, var_axis: int = 1, floor: float = FLOOR) -> float:
    rel, small = percell_parts(got, ref, var_axis, floor)
    return max(rel, small)


def one_ulp_noise(blocks: np.ndarray, seed: int = 1) -> np.ndarray:
    """Every value times (1 +/- 2^-52), random signs: one ulp of input noise.

    Running the oracle on this input measures how far the reference formula
    itself moves on the same data when its input changes in the last place;
    that self-noise is the parity bar where it exceeds the fixed one."""
    rng = np.random.default_rng(seed)
    return blocks * (1.0 + 2.0 ** -52 * rng.choice([-1.0, 1.0], blocks.shape))
