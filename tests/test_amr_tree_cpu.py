"""Host tree logic of multi-level grids (amrvac_b200.amr): refinement with
proper nesting, coarsening of whole sibling groups, the coarse average and
settree's initial hierarchy.  No GPU needed."""
import itertools

import numpy as np
import pytest

from amrvac_b200.amr import Tree, coarsen_average, initial_hierarchy


def _volume(tree):
    return sum(1.0 / (np.prod(tree.nbase[:tree.nd]) * (1 << (tree.nd * (t[0] - 1)))) for t in tree.leaves)


def _flags(tree, pred):
    return [bool(pred(t)) for t in tree.leaves]


def test_refine_keeps_nesting_2d():
    T = Tree(2, [4, 4], 4)
    T, _ = T.regrid(_flags(T, lambda t: t[1:3] == (1, 1)))
    assert T.counts() == {1: 15, 2: 4}
    # refine the level-2 child at the corner of its parent: the level-1
    # leaves next to that corner must refine with it
    T, _ = T.regrid(_flags(T, lambda t: t == (2, 2, 2, 0)))
    assert T.balanced()
    assert T.counts()[3] == 4
    assert (1, 0, 0, 0) not in T.set and (1, 1, 0, 0) not in T.set and (1, 0, 1, 0) not in T.set
    assert abs(_volume(T) - 1.0) < 1e-14


@pytest.mark.parametrize("nd,nbase", [(2, [4, 4]), (3, [2, 2, 2])])
def test_random_regrids_stay_balanced(nd, nbase):
    rng = np.random.default_rng(11)
    T = Tree(nd, nbase, 4)
    for it in range(12):
        ref = rng.random(len(T.leaves)) < 0.15
        coa = rng.random(len(T.leaves)) < 0.6
        T, origin = T.regrid(ref, coa)
        assert T.balanced(), it
        assert abs(_volume(T) - 1.0) < 1e-12
        assert len(origin) == len(T.leaves)
    assert max(T.level_of()) >= 3


def test_coarsen_needs_the_whole_group():
    T = Tree(2, [2, 2], 3)
    T, _ = T.regrid(_flags(T, lambda t: t[1:3] == (0, 0)))
    kids = [t for t in T.leaves if t[0] == 2]
    # three of four flagged: nothing happens
    T2, _ = T.regrid([False] * len(T.leaves), _flags(T, lambda t: t in kids[:3]))
    assert T2.leaves == T.leaves
    # all four: the parent comes back, built from its children in x-fastest order
    T3, origin = T.regrid([False] * len(T.leaves), _flags(T, lambda t: t in kids))
    assert T3.leaves == Tree(2, [2, 2], 3).leaves
    o = origin[T3.leaves.index((1, 0, 0, 0))]
    assert o[0] == "parent"
    assert [T.leaves[k] for k in o[1]] == [(2, 0, 0, 0), (2, 1, 0, 0), (2, 0, 1, 0), (2, 1, 1, 0)]
    # a same-level neighbour that refines cancels the coarsening (a coarser
    # one does not: the result is nested either way)
    T4, _ = T.regrid(_flags(T, lambda t: t == (1, 1, 0, 0)), _flags(T, lambda t: t in kids))
    assert (1, 0, 0, 0) in T4.set and T4.balanced()
    U = Tree(2, [4, 4], 3)
    U, _ = U.regrid(_flags(U, lambda t: t[1:3] in ((0, 0), (1, 0))))
    ukids = [t for t in U.leaves if t[0] == 2 and t[1] < 2]
    U2, _ = U.regrid(_flags(U, lambda t: t == (2, 2, 0, 0)), _flags(U, lambda t: t in ukids))
    assert (2, 0, 0, 0) in U2.set and U2.balanced()


@pytest.mark.parametrize("nd", [2, 3])
def test_coarsen_average(nd):
    rng = np.random.default_rng(2)
    g = [20 if d < nd else 1 for d in range(3)]
    kids = [rng.random((3, g[2], g[1], g[0])) for _ in range(1 << nd)]
    out = coarsen_average(kids, nd)
    for cb, w in enumerate(kids):
        c = [(cb >> d) & 1 for d in range(3)]
        for idx in itertools.product(*[range(8) if d < nd else range(1) for d in (2, 1, 0)]):
            k, j, i = idx
            fine = [w[:, 2 + 2 * k + kk if nd > 2 else 0, 2 + 2 * j + jj, 2 + 2 * i + ii]
                    for kk in range(2 if nd > 2 else 1) for jj in range(2) for ii in range(2)]
            ref = fine[0]
            for f in fine[1:]:
                ref = ref + f
            ref = ref * (1.0 / (1 << nd))
            got = out[:, 2 + 8 * c[2] + k if nd > 2 else 0, 2 + 8 * c[1] + j, 2 + 8 * c[0] + i]
            assert np.array_equal(got, ref)


def test_initial_hierarchy_reaches_the_finest_level():
    def init(tree):
        return np.zeros((len(tree.leaves), 1, 1, 20, 20))

    def err(tree, blocks):  # refine every block whose centre is within 0.2 of (0.5, 0.5)
        ref = []
        for t in tree.leaves:
            n = 4 << (t[0] - 1)
            c = (np.array(t[1:3]) + 0.5) / n
            ref.append(np.linalg.norm(c - 0.5) < 0.2)
        return ref, [not r for r in ref]

    T, blocks = initial_hierarchy(Tree(2, [4, 4], 4), init, err)
    assert max(T.level_of()) == 4 and T.balanced()
    assert blocks.shape[0] == len(T.leaves)


@pytest.mark.parametrize("nd,nbase,periodic", [(2, [4, 4], None), (3, [2, 2, 2], None), (2, [3, 2], None),
                                                (2, [4, 4], [False, False]), (3, [2, 2, 2], [True, False, False])])
def test_native_plan_matches_python(nd, nbase, periodic):
    """The library's C++ tree decision (amrvac_amr_plan) equals Tree.regrid:
    same leaves in the same order, same ops, over random regrid sequences,
    on periodic domains and with physical boundaries."""
    from amrvac_b200.amr import ops, plan_native
    rng = np.random.default_rng(7 + nd + (0 if periodic is None else 3))
    T = Tree(nd, nbase, 4, periodic=periodic)
    for it in range(10):
        ref = rng.random(len(T.leaves)) < 0.2
        coa = rng.random(len(T.leaves)) < 0.5
        nt, origin = T.regrid(ref, coa)
        leaves, op = plan_native(T, ref, coa)
        assert leaves == nt.leaves, it
        assert np.array_equal(op, ops(origin)), it
        T = nt
    assert max(T.level_of()) >= 3
