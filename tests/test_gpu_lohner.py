"""Löhner error estimator on the GPU against the oracle's lohner_grid.

Per block: the refine/coarsen decision exactly, and the largest cell error to
1e-12 relative; with per-level thresholds, log10 flags, several weighted
variables and physical boundaries.
"""
import numpy as np
import pytest

from tests import _problems as P

pytestmark = pytest.mark.gpu


def _cuda():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")


CASES = [
    ("hd2", dict(physics="hd", ndim=2, gamma=1.4), 64, ["periodic"] * 4),
    ("hd2_cont_symm", dict(physics="hd", ndim=2, gamma=1.4), 48, ["cont", "cont", "symm", "symm"]),
    ("mhd3_glm", dict(physics="mhd", ndim=3, typedivbfix="glm"), 32, ["periodic"] * 6),
]


def _state(kind, physics, ndim, ndir, n, glm):
    prim = P.random_smooth(physics, ndim, ndir, n, seed=7, glm=glm)
    if kind == "step":  # a density jump so that some blocks refine
        x = (np.arange(n) + 0.5) / n
        prim[0][..., x > 0.55] *= 3.0
    return prim


@pytest.mark.parametrize("name,kw,n,bc", CASES, ids=[c[0] for c in CASES])
@pytest.mark.parametrize("kind", ["smooth", "step"])
def test_lohner_matches_oracle(oracle_lib, name, kw, n, bc, kind):
    _cuda()
    from amrvac_b200 import Context, make_cfg
    O = oracle_lib
    ndim = kw["ndim"]
    ndir = kw.get("ndir", ndim)
    glm = kw.get("typedivbfix") == "glm"
    gcfg = make_cfg(typeboundary=bc, **kw)
    okw = dict(kw)
    okw["divb"] = okw.pop("typedivbfix", "none")
    ocfg = O.make_cfg(**okw)
    prim = _state(kind, kw["physics"], ndim, ndir, n, glm)
    cons = P.prim_to_cons(prim, kw["physics"], ndir, ocfg.gamma)
    blocks = P.to_blocks(cons, ndim)
    og = O.Grid(ocfg, [n] * ndim, [0.0] * ndim, [1.0] * ndim, bc)
    for ib in range(og.nblocks):
        og.set_block(ib, blocks[ib])
    og.getbc()
    ctx = Context(gcfg)
    ctx.set_uniform_grid([n] * ndim, [0.0] * ndim, [1.0] * ndim)
    ctx.upload(blocks)
    nw = ctx.nw
    rng = np.random.default_rng(3)
    levels = rng.integers(1, 4, size=ctx.nblocks)
    thr = [0.05, 0.1, 0.2]
    der = [0.125, 0.2, 0.3]
    wf = [1e-2, 2e-2, 5e-3]
    for weight, logflag in (([1.0] + [0.0] * (nw - 1), [1] + [0] * (nw - 1)),
                            ([0.5] + [0.0] * (nw - 3) + [0.5, 0.0] if nw > 4 else [0.5, 0.0, 0.0, 0.5], None)):
        weight = np.array(weight[:nw] + [0.0] * (nw - len(weight[:nw])))
        flags, errmax = ctx.lohner(weight, logflag, refine_max_level=3, refine_threshold=thr, derefine_ratio=der,
                                   amr_wavefilter=wf, block_level=levels)
        lf = np.zeros(nw, np.int32) if logflag is None else np.array(logflag[:nw], np.int32)
        for ib in range(og.nblocks):
            lv = int(levels[ib])
            err, r, c = O.lohner_block(ocfg, og.get_block(ib), weight, lf, wf[lv - 1], thr[lv - 1], der[lv - 1], lv, 3)
            assert abs(errmax[ib] - err.max()) <= 1e-12 * err.max(), (ib, errmax[ib], err.max())
            assert flags[ib] == (1 if r else 0) | (2 if c else 0), (ib, flags[ib], r, c)
    if kind == "step":
        assert (flags & 1).any()
