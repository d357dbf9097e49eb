"""Stage-kernel variants of the 3-D MHD HLLD + GLM schemes (cada3, and
vanleer on 'cont' sides) against the oracle: threads per CTA, CTAs per SM, and asynchronous bulk-copy staging
of the next conserved plane (FP64).  Each variant runs one stage with every
work distribution (persistent plane ranges, z-chunks of 16, 8 and 4 planes)
on a 48^3 grid of 27 blocks — z neighbours inside the domain take the bulk
copies, planes behind a 'cont' boundary the gathered loads — and must give
the oracle's stage cell by cell (tests/_parity.py; bar 1e-12).  The mixed
variants are checked against the FP64 kernel (FP32 faces).  The autotuner
picks one of them and reports it.
"""
import numpy as np
import pytest

from tests import _problems as P
from tests._parity import percell_err

pytestmark = pytest.mark.gpu

RTOL = 1e-12
KW = dict(physics="mhd", ndim=3, ndir=3, flux_scheme="hlld", limiter="cada3", typedivbfix="glm")
N = 48


def _cuda():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")


def _setup(O, bc, precision="fp64", lim="cada3"):
    from amrvac_b200 import Context, make_cfg
    kw = dict(KW, limiter=lim)
    ok = dict(kw)
    ok["divb"] = ok.pop("typedivbfix")
    ocfg = O.make_cfg(**ok)
    prim = P.random_smooth("mhd", 3, 3, N, glm=True)
    blocks = P.to_blocks(P.prim_to_cons(prim, "mhd", 3, ocfg.gamma), 3)
    og = O.Grid(ocfg, [N] * 3, [0.0] * 3, [1.0] * 3, [bc] * 6)
    for ib in range(og.nblocks):
        og.set_block(ib, blocks[ib])
    og.getbc()
    ctx = Context(make_cfg(precision=precision, typeboundary=[bc] * 6, **kw))
    ctx.set_uniform_grid([N] * 3, [0.0] * 3, [1.0] * 3)
    ctx.upload(blocks)
    return og, ocfg, ctx


def _oracle_stage(O, og, ocfg):
    dt, cg = og.getdt()
    dt *= 0.5
    ref = []
    for ib in range(og.nblocks):
        w = og.get_block(ib)
        wn = w.copy()
        O.finite_volume(ocfg, w, wn, dt, og.dx(), cg)
        ref.append(wn)
    return dt, cg, P.interior(np.array(ref), 3)


@pytest.mark.parametrize("bc,lim", [("periodic", "cada3"), ("cont", "cada3"), ("cont", "vanleer")])
def test_fp64_variants_match_oracle(oracle_lib, bc, lim):
    _cuda()
    O = oracle_lib
    og, ocfg, ctx = _setup(O, bc, lim=lim)
    dt, cg, ref = _oracle_stage(O, og, ocfg)
    ctx.set_cmax_global(cg)
    info = ctx.stage_variant()
    assert info["nvariants"] == 4 and info["variant"] == 0
    seen_async = False
    for var in range(info["nvariants"]):
        ctx.set_stage_variant(var)
        vi = ctx.stage_variant()
        seen_async |= vi["async_staging"]
        for z in (0, 16, 8, 4):
            ctx.set_zchunk(z)
            assert ctx.advect1("ps", "ps1", 1.0, dt) == 0
            err = percell_err(P.interior(ctx.download("ps1"), 3), ref)
            assert err <= RTOL, (vi, z, err)
    assert seen_async
    assert ctx.status() == 0


def test_mixed_variants_match_fp64(oracle_lib):
    """Every mixed variant's stage is within FP32 round-off of the FP64
    kernel's (L1 of the density 1e-6, no cell off by more than 1e-4 of its
    variable's scale)."""
    _cuda()
    O = oracle_lib
    og, ocfg, c64 = _setup(O, "periodic")
    _, _, cmx = _setup(O, "periodic", precision="mixed")
    dt, cg = og.getdt()
    dt *= 0.5
    c64.set_cmax_global(cg)
    c64.advect1("ps", "ps1", 1.0, dt)
    ref = P.interior(c64.download("ps1"), 3)
    cmx.set_cmax_global(cg)
    scale = np.abs(ref).max(axis=(0, 2, 3, 4))
    for var in range(cmx.stage_variant()["nvariants"]):
        cmx.set_stage_variant(var)
        for z in (0, 8):
            cmx.set_zchunk(z)
            assert cmx.advect1("ps", "ps1", 1.0, dt) == 0
            got = P.interior(cmx.download("ps1"), 3)
            rel = np.abs(got[:, 0] - ref[:, 0]).sum() / np.abs(ref[:, 0]).sum()
            dev = (np.abs(got - ref).max(axis=(0, 2, 3, 4)) / scale).max()
            assert rel <= 1e-6 and dev <= 1e-4, (var, z, rel, dev)
    assert cmx.status() == 0


def test_autotune_reports_the_chosen_variant(oracle_lib, tmp_path, monkeypatch):
    _cuda()
    O = oracle_lib
    monkeypatch.setenv("AMRVAC_TUNE_CACHE", str(tmp_path / "tune.json"))
    og, ocfg, ctx = _setup(O, "periodic")
    ctx.set_time(0.0, 1.0e99, 0.0)
    z, ms = ctx.autotune(reps=2)
    info = ctx.stage_variant()
    assert z in (0, 16, 8, 4) and 0 <= info["variant"] < info["nvariants"] and ms > 0
    # the cache restores both knobs
    ctx.set_zchunk(0)
    ctx.set_stage_variant(0)
    z2, ms2 = ctx.autotune(reps=2)
    assert z2 == z and ms2 is None and ctx.stage_variant()["variant"] == info["variant"]
    # a step with the tuned kernel still matches the oracle
    ctx.set_time(0.0, 1.0e99, 0.0)
    ctx.step()
    dt, cg = og.getdt()
    og.advance(dt, cg)
    got = P.interior(ctx.download(), 3)
    ref = P.interior(np.array([og.get_block(ib) for ib in range(og.nblocks)]), 3)
    assert percell_err(got, ref) <= RTOL


def test_bounded_wait_gives_up_with_timeout_status(oracle_lib):
    """The asynchronous variant's mbarrier wait is bounded: a wait on a
    phase that nothing completes gives up after its poll limit and reports
    AMRVAC_ST_TIMEOUT (16) instead of hanging; the device stays usable — a
    stage of the asynchronous variant right after still matches the oracle."""
    _cuda()
    import ctypes
    from amrvac_b200 import _lib
    L = _lib.load()
    f = ctypes.c_uint32(0)
    assert L.amrvac_gpu_wait_probe(1000, ctypes.byref(f)) == 0
    assert f.value == 16
    O = oracle_lib
    og, ocfg, ctx = _setup(O, "periodic")
    dt, cg, ref = _oracle_stage(O, og, ocfg)
    ctx.set_cmax_global(cg)
    ctx.set_stage_variant(1)
    assert ctx.stage_variant()["async_staging"]
    assert ctx.advect1("ps", "ps1", 1.0, dt) == 0
    assert percell_err(P.interior(ctx.download("ps1"), 3), ref) <= RTOL
    assert ctx.status() == 0
