"""Host side of multi-level grids: the block tree, its refinement and
coarsening with 2:1 nesting, and the initial hierarchy.

A tree is a set of leaves (level, ig0, ig1, ig2) over nbase root blocks per
direction of a periodic domain; level 1 is the root level and block indices
are per level (a block of level l+1 with index 2*ig + c is a child of block
ig of level l).  The device holds the leaves' states and computes everything
per cell (ghost cells across level jumps, flux fix, Löhner error estimate);
this module decides which leaves exist:

* ``Tree.regrid(refine, coarsen)`` restates amr_coarsen_refine
  (src/amr/mod_coarsen_refine.t:20-182) with proper_nesting (186-319): a
  leaf flagged for refinement also flags the leaves of its parent's level
  next to it (so that refined blocks keep 2:1 nesting, walking the levels
  from fine to coarse); a coarsening happens only when all 2^d siblings are
  leaves flagged for it and no neighbour across the siblings' outer sides is
  flagged for refinement or refined further; refinement wins over
  coarsening.
* ``initial_hierarchy`` restates settree (src/amr/mod_amr_grid.t:13-43): on
  the initial condition, repeat errest (Löhner, refine_criterion 3) and
  amr_coarsen_refine once per new level, filling refined children with the
  initial condition (refine_grids, src/amr/mod_refine.t:12-40, before the
  time loop) and coarsened parents with the 2^d-average of their children
  (coarsen_grid, src/amr/mod_coarsen.t), until refine_max_level or until no
  finer level appears.
"""
from __future__ import annotations

import itertools

import numpy as np


class Tree:
    def __init__(self, ndim, nbase, max_level, leaves=None, periodic=None):
        self.nd = int(ndim)
        self.nbase = [int(n) for n in list(nbase)[:self.nd]] + [1] * (3 - self.nd)
        self.max_level = int(max_level)
        self.periodic = [True] * self.nd if periodic is None else [bool(p) for p in periodic][:self.nd]
        if leaves is None:
            leaves = [(1,) + ig for ig in itertools.product(*[range(n) for n in self.nbase[:self.nd]])]
        self.leaves = [self._key(t) for t in leaves]
        self._index()

    # ---------------------------------------------------------------- helpers
    def _key(self, t):
        t = tuple(int(x) for x in t)
        return t + (0,) * (4 - len(t))

    def _index(self):
        self.leaves.sort()
        self.set = set(self.leaves)
        self.refined = set()  # (level, ig) of every non-leaf ancestor
        for L, *ig in self.leaves:
            for L2 in range(L - 1, 0, -1):
                self.refined.add((L2,) + tuple(i >> (L - L2) for i in ig))

    def _wrap(self, L, ig):
        """ig inside the domain (wrapped across periodic sides), or None
        across a physical boundary."""
        out = []
        for d in range(3):
            if d >= self.nd:
                out.append(0)
                continue
            n = self.nbase[d] << (L - 1)
            if not (0 <= ig[d] < n) and not self.periodic[d]:
                return None
            out.append(ig[d] % n)
        return tuple(out)

    def _dirs(self):
        return [dd + (0,) * (3 - self.nd) for dd in itertools.product((-1, 0, 1), repeat=self.nd) if any(dd)]

    def level_of(self):
        return np.array([t[0] for t in self.leaves], np.int32)

    def counts(self):
        out = {}
        for t in self.leaves:
            out[t[0]] = out.get(t[0], 0) + 1
        return dict(sorted(out.items()))

    def cells(self, bn=16):
        return len(self.leaves) * bn ** self.nd

    # ---------------------------------------------------------------- regrid
    def regrid(self, refine, coarsen=None):
        """refine/coarsen: boolean per leaf (current order).  Returns
        (new Tree, origin) where origin[b] for every new leaf is ("same", old),
        ("child", old parent leaf, child bits) or ("parent", [old children])."""
        pos = {t: b for b, t in enumerate(self.leaves)}
        ref = {t for t, f in zip(self.leaves, refine) if f and t[0] < self.max_level}
        coa = set() if coarsen is None else {t for t, f in zip(self.leaves, coarsen) if f and t[0] > 1}
        # proper_nesting, refinement part: levels from fine to coarse
        levmax = max(t[0] for t in self.leaves)
        for L in range(min(levmax, self.max_level - 1), 1, -1):
            for t in sorted(x for x in ref if x[0] == L):
                ig = t[1:]
                pg = tuple(i >> 1 for i in ig)
                ic = [ig[d] & 1 for d in range(3)]
                rng = [((-1, 0) if ic[d] == 0 else (0, 1)) if d < self.nd else (0,) for d in range(3)]
                for inp in itertools.product(*rng):
                    if not any(inp):
                        continue
                    w = self._wrap(L - 1, tuple(pg[d] + inp[d] for d in range(3)))
                    if w is not None and (L - 1,) + w in self.set:
                        ref.add((L - 1,) + w)
        coa -= ref
        # proper_nesting, coarsening part: whole sibling groups whose outer
        # neighbours neither refine nor are refined further (unless those
        # children coarsen too)
        groups = {}
        for t in coa:
            groups.setdefault((t[0] - 1,) + tuple(i >> 1 for i in t[1:]), []).append(t)
        nchild = 1 << self.nd
        coarsen_parents = []
        # finer levels first, a group that fails is unflagged before the
        # coarser levels look at it (unflag_coarsen_siblings)
        for par, kids in sorted(groups.items(), key=lambda kv: (-kv[0][0], kv[0][1:])):
            kids = sorted(kids, key=lambda t: sum((t[1 + d] & 1) << d for d in range(3)))
            if len(kids) != nchild:
                coa -= set(kids)
                continue
            ok = True
            for t in kids:
                ig = t[1:]
                ic = [ig[d] & 1 for d in range(3)]
                rng = [((-1, 0) if ic[d] == 0 else (0, 1)) if d < self.nd else (0,) for d in range(3)]
                for i in itertools.product(*rng):
                    if not any(i):
                        continue
                    w = self._wrap(t[0], tuple(ig[d] + i[d] for d in range(3)))
                    if w is None:  # a physical boundary: no neighbour
                        continue
                    nb = (t[0],) + w
                    if nb in self.set:
                        if nb in ref:
                            ok = False
                    elif nb in self.refined:
                        ch = (t[0] + 1,) + tuple(2 * nb[1 + d] if d < self.nd else 0 for d in range(3))
                        if not (ch in self.set and ch in coa):
                            ok = False
                    if not ok:
                        break
                if not ok:
                    break
            if ok:
                coarsen_parents.append((par, kids))
            else:
                coa -= set(kids)
        gone = set()
        new = []
        origin = {}
        for par, kids in coarsen_parents:
            gone.update(kids)
            new.append(par)
            origin[par] = ("parent", [pos[k] for k in kids])
        for t in self.leaves:
            if t in gone:
                continue
            if t in ref:
                for c in itertools.product(*[(0, 1) if d < self.nd else (0,) for d in range(3)]):
                    ch = (t[0] + 1,) + tuple(2 * t[1 + d] + c[d] if d < self.nd else 0 for d in range(3))
                    new.append(ch)
                    origin[ch] = ("child", pos[t], c[0] + 2 * c[1] + 4 * c[2])
            else:
                new.append(t)
                origin[t] = ("same", pos[t])
        T = Tree(self.nd, self.nbase, self.max_level, new, self.periodic)
        return T, [origin[t] for t in T.leaves]

    def balanced(self):
        """True if no two leaves that share a face, edge or corner differ by
        more than one level."""
        for t in self.leaves:
            L, ig = t[0], t[1:]
            for dd in self._dirs():
                g = self._wrap(L, tuple(ig[d] + dd[d] for d in range(3)))
                if g is None:
                    continue
                # the leaf covering g at level L, or a refined region
                if (L,) + g in self.set or (L,) + g in self.refined:
                    if (L,) + g in self.refined:
                        for c in itertools.product(*[(0, 1) if d < self.nd else (0,) for d in range(3)]):
                            adj = all(d >= self.nd or dd[d] == 0 or c[d] == (0 if dd[d] > 0 else 1) for d in range(3))
                            ch = (L + 1,) + tuple(2 * g[d] + c[d] if d < self.nd else 0 for d in range(3))
                            if adj and ch not in self.set:
                                return False
                    continue
                p = (L - 1,) + tuple(i >> 1 for i in g)
                if p not in self.set:
                    return False
        return True


def coarsen_average(children, ndim, ng=2, bn=None):
    """Parent block (ghosted, ghost cells zero) from its 2^d children
    (ghosted), child bits x fastest: the average of every 2^d fine cells
    (coarsen_grid on conserved variables), summed x fastest.  bn: cells per
    block edge (default: from the children's shape)."""
    nw = children[0].shape[0]
    bn = children[0].shape[-1] - 2 * ng if bn is None else bn
    g = [bn + 2 * ng if d < ndim else 1 for d in range(3)]
    out = np.zeros((nw, g[2], g[1], g[0]))
    h = bn // 2
    for cb, w in enumerate(children):
        c = [(cb >> d) & 1 for d in range(3)]
        inner = w[(slice(None),) + tuple(slice(ng, ng + bn) if d < ndim else slice(0, 1) for d in (2, 1, 0))]
        acc = None
        for kk in range(2 if ndim > 2 else 1):
            for jj in range(2 if ndim > 1 else 1):
                for ii in range(2):
                    s = inner[:, kk::2 if ndim > 2 else 1, jj::2 if ndim > 1 else 1, ii::2]
                    acc = s.copy() if acc is None else acc + s
        acc = acc * (1.0 / (1 << ndim))
        sl = (slice(None),) + tuple(slice(ng + c[d] * h, ng + c[d] * h + h) if d < ndim else slice(0, 1)
                                    for d in (2, 1, 0))
        out[sl] = acc
    return out


def initial_hierarchy(tree, init_fn, error_fn, max_iter=None):
    """settree: tree (level-1 leaves), init_fn(tree) -> ghosted conserved
    blocks of every leaf from the initial condition, error_fn(tree, blocks)
    -> (refine, coarsen) per leaf.  Returns the final tree and its blocks."""
    blocks = init_fn(tree)
    for levnew in range(2, tree.max_level + 1):
        refine, coarsen = error_fn(tree, blocks)
        nt, origin = tree.regrid(refine, coarsen)
        fresh = init_fn(nt)
        out = np.empty_like(fresh)
        for b, o in enumerate(origin):
            if o[0] == "same":
                out[b] = blocks[o[1]]
            elif o[0] == "child":
                out[b] = fresh[b]
            else:
                out[b] = coarsen_average([blocks[k] for k in o[1]], tree.nd)
        tree, blocks = nt, out
        if max(t[0] for t in tree.leaves) != levnew:
            break
    return tree, blocks


def lohner_flags(ctx, tree, blocks, xprobmin, xprobmax, weight, logflag=None, refine_threshold=0.1,
                 derefine_ratio=0.125, amr_wavefilter=1.0e-2):
    """errest on the device: puts tree and blocks into ctx and runs the
    Löhner estimator (ghost cells across level jumps included).  Returns
    (refine, coarsen, errmax) per leaf."""
    ctx.set_amr_grid(tree.leaves, tree.nbase[:tree.nd], xprobmin, xprobmax)
    ctx.upload(blocks)
    L = tree.max_level

    def per_level(x):
        return [float(x)] * L if np.isscalar(x) else list(x)
    flags, errmax = ctx.lohner(weight, logflag, refine_max_level=L, refine_threshold=per_level(refine_threshold),
                               derefine_ratio=per_level(derefine_ratio), amr_wavefilter=per_level(amr_wavefilter),
                               block_level=tree.level_of())
    flags = np.asarray(flags)
    return (flags & 1).astype(bool), (flags & 2).astype(bool), errmax


def ops(origin):
    """The op table of amrvac_gpu_amr_regrid from Tree.regrid's origin list."""
    out = np.zeros((len(origin), 9), np.int32)
    for b, o in enumerate(origin):
        if o[0] == "same":
            out[b, :2] = (0, o[1])
        elif o[0] == "child":
            out[b, :3] = (1, o[1], o[2])
        else:
            out[b, 0] = 2
            out[b, 1:1 + len(o[1])] = o[1]
    return out


def regrid(ctx, tree, weight, logflag=None, refine_threshold=0.1, derefine_ratio=0.125, amr_wavefilter=1.0e-2):
    """resettree on the resident state in one library call
    (amrvac_gpu_amr_resettree: device Löhner on register ps, the C++ tree
    decision, the device remap).  Returns the new Tree (the same object if
    nothing changed)."""
    changed = ctx.amr_resettree(weight, logflag, refine_max_level=tree.max_level, refine_threshold=refine_threshold,
                                derefine_ratio=derefine_ratio, amr_wavefilter=amr_wavefilter)
    if not changed:
        return tree
    return Tree(tree.nd, tree.nbase[:tree.nd], tree.max_level, ctx.amr_leaves(), tree.periodic)


def regrid_python(ctx, tree, weight, logflag=None, refine_threshold=0.1, derefine_ratio=0.125,
                  amr_wavefilter=1.0e-2):
    """The same resettree with the tree decision made here (Tree.regrid) and
    the remap through amrvac_gpu_amr_regrid."""
    L = tree.max_level

    def per_level(x):
        return [float(x)] * L if np.isscalar(x) else list(x)
    flags, _ = ctx.lohner(weight, logflag, refine_max_level=L, refine_threshold=per_level(refine_threshold),
                          derefine_ratio=per_level(derefine_ratio), amr_wavefilter=per_level(amr_wavefilter),
                          block_level=tree.level_of())
    flags = np.asarray(flags)
    nt, origin = tree.regrid((flags & 1).astype(bool), (flags & 2).astype(bool))
    if nt.leaves == tree.leaves:
        return tree
    ctx.amr_regrid(nt.leaves, ops(origin))
    return nt


def plan_native(tree, refine, coarsen):
    """Tree.regrid's decision computed by the library (amrvac_amr_plan, C++,
    host only): (new leaves, op table)."""
    import ctypes
    from . import _lib
    L = _lib.load()
    nd = tree.nd
    lv = np.ascontiguousarray(np.array(tree.leaves, np.int32).reshape(-1))
    nb = np.ascontiguousarray(tree.nbase[:nd], np.int32)
    r = np.ascontiguousarray(np.asarray(refine, np.uint8))
    c = np.ascontiguousarray(np.asarray(coarsen, np.uint8))
    cap = len(tree.leaves) << nd
    out_l = np.zeros(4 * cap, np.int32)
    out_o = np.zeros(9 * cap, np.int32)
    n = ctypes.c_int(0)
    ip, up = ctypes.POINTER(ctypes.c_int), ctypes.POINTER(ctypes.c_ubyte)
    per = np.ascontiguousarray([1 if p else 0 for p in tree.periodic], np.int32)
    _lib.check(L.amrvac_amr_plan(nd, nb.ctypes.data_as(ip), per.ctypes.data_as(ip), tree.max_level,
                                 len(tree.leaves), lv.ctypes.data_as(ip),
                                 r.ctypes.data_as(up), c.ctypes.data_as(up), cap, ctypes.byref(n),
                                 out_l.ctypes.data_as(ip), out_o.ctypes.data_as(ip)), "amrvac_amr_plan")
    k = n.value
    return [tuple(int(x) for x in out_l[4 * b:4 * b + 4]) for b in range(k)], out_o[:9 * k].reshape(k, 9)
