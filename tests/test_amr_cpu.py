"""The oracle's multi-level grid (restated multi-level getbc and flux fix).

* Linear conserved fields: every ghost cell of every block away from the
  periodic wrap equals the field at its centre after getbc — same-level
  copies, restriction (averages of fine cells) and prolongation (psc with
  monotonized-central slopes) are all exact for linear data.
* The flux correction makes the multi-level update conservative: totals of
  every conserved variable stay constant to rounding on a periodic domain.
* A hierarchy refined everywhere is the uniform finer grid, bit for bit.

Each holds for blocks of 16 and of 8 cells per edge (block_nx; the
reference's 3-D blast test runs 8^3 blocks).
"""
import numpy as np
import pytest

from tests import _amr as A


def _cfg(O, nd, **kw):
    base = dict(physics="hd", ndim=nd, gamma=1.4, flux_scheme="hllc", limiter="vanleer", courantpar=0.8)
    # (block_nx passes through **kw)
    base.update(kw)
    return O.make_cfg(**base)


def _nbase(nd):
    return [8] * nd if nd == 2 else [4] * nd


def _leaves(nd, levels=3):
    def ref(c, lv):
        r = np.linalg.norm(c - 0.5)
        return r < (0.3 if lv == 1 else 0.15)
    return A.build_leaves(nd, _nbase(nd), levels, ref)


def _lin(nd):
    def f(X, Y, Z):
        out = np.zeros((nd + 2,) + X.shape)
        out[0] = 1.0 + 0.1 * X + 0.2 * Y + (0.05 * Z if nd > 2 else 0)
        out[1] = 0.1 + 0.05 * X - 0.02 * Y
        out[2] = -0.1 * Y + 0.03 * X
        if nd > 2:
            out[3] = 0.02 * Z - 0.01 * X
        out[nd + 1] = 3.0 + 0.2 * X - 0.1 * Y + (0.04 * Z if nd > 2 else 0)
        return out
    return f


@pytest.mark.parametrize("nd", [2, 3])
@pytest.mark.parametrize("bn", [16, 8])
def test_ghost_cells_exact_for_linear_data(oracle_lib, nd, bn):
    O = oracle_lib
    leaves = _leaves(nd, levels=3 if nd == 2 else 2)
    assert len({l[0] for l in leaves}) == (3 if nd == 2 else 2)
    c = _cfg(O, nd, block_nx=bn)
    nb = _nbase(nd)
    g = O.AmrGrid(c, nb, [0.0] * nd, [1.0] * nd, leaves)
    blocks = A.fill_blocks(leaves, nd, nb, _lin(nd), "hd", nd, 1.4, conserved=True, bn=bn)
    for b in range(len(leaves)):
        g.set_block(b, blocks[b])
    # scramble the ghost cells so that only getbc can make them right
    for b in range(len(leaves)):
        w = blocks[b].copy()
        sl = (slice(None),) + tuple(slice(2, 2 + bn) if d < nd else slice(None) for d in (2, 1, 0))
        z = np.full_like(w, -7.0)
        z[sl] = w[sl]
        g.set_block(b, z)
    g.getbc()
    checked = 0
    for b, leaf in enumerate(leaves):
        lv, ig = leaf[0], leaf[1:]
        n = nb[0] << (lv - 1)
        if any(i == 0 or i == n - 1 for i in ig):
            continue  # the periodic wrap breaks a linear field
        got = g.get_block(b)
        assert np.allclose(got, blocks[b], rtol=0, atol=1e-13), (leaf, np.abs(got - blocks[b]).max())
        checked += 1
    assert checked > 0


def _periodic(nd):
    def f(X, Y, Z):
        out = np.zeros((nd + 2,) + X.shape)
        s = np.sin(2 * np.pi * X) * np.cos(2 * np.pi * Y) * (np.cos(2 * np.pi * Z) if nd > 2 else 1)
        out[0] = 1.0 + 0.3 * s
        out[1] = 0.5 + 0.2 * np.cos(2 * np.pi * Y)
        out[2] = -0.3 + 0.2 * np.sin(2 * np.pi * X)
        if nd > 2:
            out[3] = 0.1 * np.sin(2 * np.pi * Y)
        out[nd + 1] = 1.0 + 0.2 * s
        return out
    return f


@pytest.mark.parametrize("nd", [2, 3])
@pytest.mark.parametrize("bn", [16, 8])
def test_flux_fix_conserves(oracle_lib, nd, bn):
    O = oracle_lib
    leaves = _leaves(nd, levels=3 if nd == 2 else 2)
    c = _cfg(O, nd, block_nx=bn)
    nb = _nbase(nd)
    g = O.AmrGrid(c, nb, [0.0] * nd, [1.0] * nd, leaves)
    blocks = A.fill_blocks(leaves, nd, nb, _periodic(nd), "hd", nd, 1.4, bn=bn)
    for b in range(len(leaves)):
        g.set_block(b, blocks[b])
    g.getbc()
    sl = (slice(None),) + tuple(slice(2, 2 + bn) if d < nd else slice(None) for d in (2, 1, 0))

    def totals():
        return sum(g.get_block(b)[sl].reshape(nd + 2, -1).sum(axis=1) * A.block_volume(l, nd, nb, bn=bn)
                   for b, l in enumerate(leaves))
    t0 = totals()
    for _ in range(4 if nd == 2 else 2):
        dt, _ = g.getdt()
        g.advance(dt)
    t1 = totals()
    assert np.all(np.abs(t1 - t0) <= 1e-13 * np.abs(t0).max()), (t0, t1)


@pytest.mark.parametrize("bn", [16, 8])
def test_refined_everywhere_is_the_uniform_grid(oracle_lib, bn):
    O = oracle_lib
    nd = 2
    leaves = A.build_leaves(nd, [2, 2], 2, lambda c, lv: True)
    assert all(l[0] == 2 for l in leaves) and len(leaves) == 16
    c = _cfg(O, nd, block_nx=bn)
    g = O.AmrGrid(c, [2, 2], [0.0, 0.0], [1.0, 1.0], leaves)
    blocks = A.fill_blocks(leaves, nd, [2, 2], _periodic(nd), "hd", nd, 1.4, bn=bn)
    u = O.Grid(c, [4 * bn, 4 * bn], [0.0, 0.0], [1.0, 1.0], ["periodic"] * 4)
    order = {}
    for b, l in enumerate(leaves):
        g.set_block(b, blocks[b])
        order[b] = l[1] + 4 * l[2]
        u.set_block(order[b], blocks[b])
    g.getbc()
    u.getbc()
    for _ in range(3):
        dt, _ = u.getdt()
        dta, _ = g.getdt()
        assert dt == dta
        g.advance(dt)
        u.advance(dt)
    for b in range(len(leaves)):
        assert np.array_equal(g.get_block(b), u.get_block(order[b]))


def test_regrid_remap_is_exact_and_conservative(oracle_lib):
    """prolong_2nd is exact for linear data, coarsen_grid conserves every
    total, and refining then coarsening a block gives it back (to rounding)."""
    from amrvac_b200.amr import Tree, ops
    O = oracle_lib
    nd, nb = 2, [4, 4]
    c = _cfg(O, nd)
    T = Tree(nd, nb, 3)
    T, _ = T.regrid([t[1:3] in ((1, 1), (3, 3)) for t in T.leaves])
    blocks = A.fill_blocks(T.leaves, nd, nb, _lin(nd), "hd", nd, 1.4, conserved=True)
    g = O.AmrGrid(c, nb, [0.0] * nd, [1.0] * nd, T.leaves)
    for b in range(len(T.leaves)):
        g.set_block(b, blocks[b])
    g.getbc()
    sl = (slice(None), 0, slice(2, 18), slice(2, 18))

    def totals(grid, tree):
        return sum(grid.get_block(b)[sl].reshape(nd + 2, -1).sum(axis=1) * A.block_volume(l, nd, nb)
                   for b, l in enumerate(tree.leaves))
    t0 = totals(g, T)
    # refine one level-2 block away from the wrap (proper nesting refines the
    # level-1 leaves next to it as well), coarsen the children of root (3, 3)
    ref = [t == (2, 3, 3, 0) for t in T.leaves]
    coa = [t[0] == 2 and t[1] in (6, 7) and t[2] in (6, 7) for t in T.leaves]
    T2, origin = T.regrid(ref, coa)
    kinds = {o[0] for o in origin}
    assert kinds == {"same", "child", "parent"}
    g2 = g.remap(T2.leaves, ops(origin))
    exact = A.fill_blocks(T2.leaves, nd, nb, _lin(nd), "hd", nd, 1.4, conserved=True)
    for b, o in enumerate(origin):
        if o[0] == "child":
            got = g2.get_block(b)[sl]
            assert np.allclose(got, exact[b][sl], rtol=0, atol=1e-14), np.abs(got - exact[b][sl]).max()
    t1 = totals(g2, T2)
    assert np.all(np.abs(t1 - t0) <= 1e-14 * np.abs(t0).max()), (t0, t1)
    # refine then coarsen back: the parent's interior returns
    assert (2, 3, 3, 0) not in T2.set and (1, 3, 3, 0) in T2.set
    T3, o3 = T2.regrid([False] * len(T2.leaves), [t[0] == 3 for t in T2.leaves])
    g3 = g2.remap(T3.leaves, ops(o3))
    b3 = T3.leaves.index((2, 3, 3, 0))
    b0 = T.leaves.index((2, 3, 3, 0))
    assert np.allclose(g3.get_block(b3)[sl], g.get_block(b0)[sl], rtol=1e-15, atol=0)


@pytest.mark.parametrize("bc", ["cont", "symm"])
def test_refined_everywhere_with_physical_boundaries_is_the_uniform_grid(oracle_lib, bc):
    """Physical boundaries on a multi-level grid (fill_boundary_after_gc per
    block): a tree refined everywhere reproduces the uniform finer grid with
    the same boundaries, bit for bit."""
    O = oracle_lib
    nd = 2
    leaves = A.build_leaves(nd, [2, 2], 2, lambda c, lv: True)
    c = _cfg(O, nd)
    bcs = [bc] * 4
    g = O.AmrGrid(c, [2, 2], [0.0, 0.0], [1.0, 1.0], leaves, bc=bcs)
    blocks = A.fill_blocks(leaves, nd, [2, 2], _periodic(nd), "hd", nd, 1.4)
    u = O.Grid(c, [64, 64], [0.0, 0.0], [1.0, 1.0], bcs)
    order = {}
    for b, l in enumerate(leaves):
        g.set_block(b, blocks[b])
        order[b] = l[1] + 4 * l[2]
        u.set_block(order[b], blocks[b])
    g.getbc()
    u.getbc()
    for b in range(len(leaves)):
        assert np.array_equal(g.get_block(b), u.get_block(order[b]))
    for _ in range(3):
        dt, _ = u.getdt()
        assert g.getdt()[0] == dt
        g.advance(dt)
        u.advance(dt)
    for b in range(len(leaves)):
        assert np.array_equal(g.get_block(b), u.get_block(order[b]))
