"""Static AMR hierarchies for tests and benchmarks (test infrastructure).

``build_leaves`` refines the blocks whose centre satisfies a predicate, level
by level, and then enforces 2:1 balance over all 3^d neighbour directions
(periodic domain), as the reference's tree keeps it.  ``fill_blocks``
evaluates a primitive-field function at the cell centres of every leaf
(ghost cells included), giving ghosted block arrays.
"""
from __future__ import annotations

import itertools

import numpy as np

from tests import _problems as P


def build_leaves(nd, nbase, levels, refine_fn, xmin=None, xmax=None):
    xmin = np.zeros(nd) if xmin is None else np.asarray(xmin, float)
    xmax = np.ones(nd) if xmax is None else np.asarray(xmax, float)
    nbase = list(nbase)[:nd]
    leaves = {(1,) + ig for ig in itertools.product(*[range(n) for n in nbase])}

    def centre(lv, ig):
        w = (xmax - xmin) / (np.array(nbase) * (1 << (lv - 1)))
        return xmin + (np.array(ig) + 0.5) * w

    def wrap(lv, ig):
        return tuple(int(i % (nbase[d] << (lv - 1))) for d, i in enumerate(ig))

    for lv in range(1, levels):
        for leaf in sorted(leaves):
            if leaf[0] == lv and refine_fn(centre(lv, leaf[1:]), lv):
                leaves.discard(leaf)
                for c in itertools.product(*[(0, 1)] * nd):
                    leaves.add((lv + 1,) + tuple(2 * i + ci for i, ci in zip(leaf[1:], c)))
    # 2:1 balance: refine any leaf with a neighbour two levels finer
    changed = True
    while changed:
        changed = False
        fine_at = {}
        for leaf in leaves:
            fine_at.setdefault(leaf[0], set()).add(leaf[1:])
        for leaf in sorted(leaves):
            lv, ig = leaf[0], leaf[1:]
            too_fine = False
            for dd in itertools.product(*[(-1, 0, 1)] * nd):
                if not any(dd):
                    continue
                jg = wrap(lv, tuple(i + d for i, d in zip(ig, dd)))
                # any leaf at level >= lv+2 inside the neighbour region?
                for l2 in range(lv + 2, levels + 1):
                    f = 1 << (l2 - lv)
                    for c in itertools.product(*[range(f)] * nd):
                        if tuple(j * f + ci for j, ci in zip(jg, c)) in fine_at.get(l2, ()):
                            too_fine = True
                            break
                    if too_fine:
                        break
                if too_fine:
                    break
            if too_fine:
                leaves.discard(leaf)
                for c in itertools.product(*[(0, 1)] * nd):
                    leaves.add((lv + 1,) + tuple(2 * i + ci for i, ci in zip(ig, c)))
                changed = True
                break
    return sorted(leaves)


def fill_blocks(leaves, nd, nbase, prim_fn, physics, ndir, gamma, xmin=None, xmax=None, nghost=2, bn=16,
                conserved=False):
    """prim_fn(x, y, z) -> primitive array [nw][...] at cell centres (or the
    conserved array if conserved=True)."""
    xmin = np.zeros(nd) if xmin is None else np.asarray(xmin, float)
    xmax = np.ones(nd) if xmax is None else np.asarray(xmax, float)
    out = []
    for leaf in leaves:
        lv, ig = leaf[0], leaf[1:]
        dx = (xmax - xmin) / (np.array(nbase[:nd]) * bn * (1 << (lv - 1)))
        coords = []
        for d in range(3):
            if d < nd:
                x0 = xmin[d] + ig[d] * bn * dx[d]
                coords.append(x0 + (np.arange(-nghost, bn + nghost) + 0.5) * dx[d])
            else:
                coords.append(np.zeros(1))
        Z, Y, X = np.meshgrid(coords[2], coords[1], coords[0], indexing="ij")
        prim = prim_fn(X, Y, Z)
        out.append(prim if conserved else P.prim_to_cons(prim, physics, ndir, gamma))
    return np.array(out)


def block_volume(leaf, nd, nbase, xmin=None, xmax=None, bn=16):
    xmin = np.zeros(nd) if xmin is None else np.asarray(xmin, float)
    xmax = np.ones(nd) if xmax is None else np.asarray(xmax, float)
    dx = (xmax - xmin) / (np.array(nbase[:nd]) * bn * (1 << (leaf[0] - 1)))
    return float(np.prod(dx))
