"""Dimensional splitting and TVD-MUSCL on the GPU against the oracle.

dimsplit (src/mod_advance.t:23-45) runs the whole time stepper once per
direction, each sweep advancing one direction (fluxes, Hancock predictor,
divB sources with qdt/ndim, fix_conserve of that direction only), in
increasing order on even steps and decreasing order on odd steps ('xyyx') or
always increasing ('xy').  TVD-MUSCL (tvdmu: central flux plus tvdlimit2's
Roe-characteristic limiter, src/mod_tvd.t:38-112) is run split, as the
reference's tests run it.  Three steps cover both sweep orders; the bar is
the path's 1e-12 per cell.
"""
import numpy as np
import pytest

from tests._parity import percell_err

from tests import _problems as P
from tests import _amr as A

pytestmark = pytest.mark.gpu

RTOL = 1e-12
# MHD TVD-MUSCL is ill-conditioned in the Roe normalisation of its fast and
# slow eigenvectors (cslow = (cf - sqrt(cf^2 - 4 cs^2 bn^2 / rho)) / 2 and
# the weights af, as where the two speeds approach each other): the oracle
# alone turns a 1-ulp relative perturbation of its input into 3.5e-11 after
# three split steps of the 2-D case (MHD HLL: 8e-14, HD TVD-MUSCL: 7e-14), so
# the FMA-contraction differences between device and oracle get the bar of
# that self-noise rather than 1e-12.
RTOL_MHD_TVDMU = 1e-10

CASES = {
    "hd2_hll_minmod_xyyx": dict(physics="hd", ndim=2, gamma=1.4, flux_scheme="hll", limiter="minmod"),
    "hd3_hllc_vanleer_xy": dict(physics="hd", ndim=3, gamma=1.4, flux_scheme="hllc", limiter="vanleer",
                                typedimsplit="xy"),
    "hd2_tvdlf_koren_pc": dict(physics="hd", ndim=2, gamma=1.4, flux_scheme="tvdlf", limiter="koren",
                               time_stepper="twostep"),
    "mhd25_hlld_cada3_glm": dict(physics="mhd", ndim=2, ndir=3, flux_scheme="hlld", limiter="cada3",
                                 typedivbfix="glm"),
    "mhd2_hll_minmod_linde_fourstep": dict(physics="mhd", ndim=2, flux_scheme="hll", limiter="minmod",
                                           typedivbfix="linde", time_stepper="fourstep"),
    "hd2_tvdmu_albada_pc": dict(physics="hd", ndim=2, gamma=1.4, flux_scheme="tvdmu", limiter="albada",
                                time_stepper="twostep", typeboundspeed="cmaxmean"),
    "hd3_tvdmu_minmod_pc": dict(physics="hd", ndim=3, gamma=1.4, flux_scheme="tvdmu", limiter="minmod",
                                time_stepper="twostep"),
    "hd2_tvdmu_woodward_ssprk3": dict(physics="hd", ndim=2, gamma=1.4, flux_scheme="tvdmu", limiter="woodward"),
    # MHD TVD-MUSCL (the Roe system of src/mhd/mod_mhd_roe.t)
    "mhd2_tvdmu_albada_linde_pc": dict(physics="mhd", ndim=2, flux_scheme="tvdmu", limiter="albada",
                                       typedivbfix="linde", time_stepper="twostep", typeboundspeed="cmaxmean"),
    "mhd25_tvdmu_minmod_none": dict(physics="mhd", ndim=2, ndir=3, flux_scheme="tvdmu", limiter="minmod",
                                    typedivbfix="none", time_stepper="twostep"),
    "mhd3_tvdmu_vanleer_none": dict(physics="mhd", ndim=3, flux_scheme="tvdmu", limiter="vanleer",
                                    typedivbfix="none"),
}


def _cuda():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")


def _maxrel(a, b):
    """Per-cell parity measure (tests/_parity.py): relative error for cells
    >= 1e-3 of the variable's maximum, absolute at that scale below it."""
    return percell_err(a, b, var_axis=1)


def _cfgs(O, name, bc):
    from amrvac_b200 import make_cfg
    kw = dict(CASES[name])
    tds = kw.pop("typedimsplit", "xyyx")
    gcfg = make_cfg(typeboundary=bc, dimsplit=True, typedimsplit=tds, **kw)
    ok = dict(kw)
    div = ok.pop("typedivbfix", "none")
    ocfg = O.make_cfg(divb=div, dimsplit=True, typedimsplit=tds, **ok)
    return kw, gcfg, ocfg


@pytest.mark.parametrize("name", sorted(CASES))
def test_split_steps_match_oracle(oracle_lib, name):
    _cuda()
    from amrvac_b200 import Context
    O = oracle_lib
    ndim = CASES[name]["ndim"]
    bc = ["periodic"] * (2 * ndim)
    kw, gcfg, ocfg = _cfgs(O, name, bc)
    ndir = kw.get("ndir", ndim)
    n = 32
    prim = P.random_smooth(kw["physics"], ndim, ndir, n, seed=P.SEED, glm=kw.get("typedivbfix") == "glm")
    blocks = P.to_blocks(P.prim_to_cons(prim, kw["physics"], ndir, ocfg.gamma), ndim)
    og = O.Grid(ocfg, [n] * ndim, [0.0] * ndim, [1.0] * ndim, bc)
    for ib in range(og.nblocks):
        og.set_block(ib, blocks[ib])
    og.getbc()
    ctx = Context(gcfg)
    ctx.set_uniform_grid([n] * ndim, [0.0] * ndim, [1.0] * ndim)
    ctx.upload(blocks)
    ctx.set_time(0.0, 1.0e99, 0.0)
    for _ in range(3):
        dt_ref, cg_ref = og.getdt()
        ctx.step()
        assert abs(ctx.get_time()[0] - dt_ref) <= 1e-12 * dt_ref
        og.advance(dt_ref, cg_ref)
    got = P.interior(ctx.download("ps"), ndim)
    ref = P.interior(np.array([og.get_block(ib) for ib in range(og.nblocks)]), ndim)
    err = _maxrel(got, ref)
    tol = RTOL_MHD_TVDMU if (kw["physics"] == "mhd" and kw["flux_scheme"] == "tvdmu") else RTOL
    assert err <= tol, f"{name}: max rel err {err:.3e}"
    assert ctx.status() == 0


def test_split_is_not_unsplit(oracle_lib):
    """The split scheme differs from the unsplit one (the sweeps really are
    one-directional), and 'xy' differs from 'xyyx' from the second step on."""
    _cuda()
    from amrvac_b200 import Context, make_cfg
    n = 32
    prim = P.random_smooth("hd", 2, 2, n, seed=P.SEED)
    blocks = P.to_blocks(P.prim_to_cons(prim, "hd", 2, 1.4), 2)
    outs = []
    for kw in (dict(), dict(dimsplit=True), dict(dimsplit=True, typedimsplit="xy")):
        ctx = Context(make_cfg(physics="hd", ndim=2, gamma=1.4, flux_scheme="hll", **kw))
        ctx.set_uniform_grid([n, n], [0.0, 0.0], [1.0, 1.0])
        ctx.upload(blocks)
        ctx.set_time(0.0, 1.0e99, 0.0)
        ctx.step()
        ctx.step()
        outs.append(ctx.download())
        ctx.close()
    assert np.abs(outs[0] - outs[1]).max() > 1e-8
    assert np.abs(outs[1] - outs[2]).max() > 1e-10


AMR_CASES = [
    ("hd2_tvdmu_albada_pc_cont", dict(physics="hd", flux_scheme="tvdmu", limiter="albada", time_stepper="twostep",
                                      typeboundspeed="cmaxmean"), ["cont"] * 4),
    ("hd2_hllc_vanleer_split", dict(physics="hd", flux_scheme="hllc", limiter="vanleer"), ["periodic"] * 4),
    ("mhd2_hlld_linde_split", dict(physics="mhd", flux_scheme="hlld", limiter="minmod", typedivbfix="linde"),
     ["periodic"] * 4),
    ("mhd2_tvdmu_albada_linde_pc", dict(physics="mhd", flux_scheme="tvdmu", limiter="albada", typedivbfix="linde",
                                        time_stepper="twostep"), ["periodic"] * 4),
]


@pytest.mark.parametrize("name,kw,bc", AMR_CASES, ids=[c[0] for c in AMR_CASES])
def test_split_amr_steps_match_oracle(oracle_lib, name, kw, bc):
    """Multi-level grids: split sweeps with the flux fix of the sweep's
    direction only."""
    _cuda()
    from amrvac_b200 import Context, make_cfg
    from tests.test_gpu_amr import _field, _nbase
    O = oracle_lib
    nd, levels = 2, 3
    nb = _nbase(nd)

    def ref(c, lv):
        return np.linalg.norm(c - (0.1 if bc[0] == "cont" else 0.45)) < (0.3 if lv == 1 else 0.15)
    leaves = A.build_leaves(nd, nb, levels, ref)
    physics = kw["physics"]
    base = dict(ndim=nd, gamma=5.0 / 3.0 if physics == "mhd" else 1.4, courantpar=0.6)
    base.update(kw)
    ok = dict(base)
    if "typedivbfix" in ok:
        ok["divb"] = ok.pop("typedivbfix")
    og = O.AmrGrid(O.make_cfg(dimsplit=True, **ok), nb, [0.0] * nd, [1.0] * nd, leaves, bc=bc)
    blocks = A.fill_blocks(leaves, nd, nb, _field(nd, physics), physics, nd, base["gamma"])
    for b in range(len(leaves)):
        og.set_block(b, blocks[b])
    og.getbc()
    ctx = Context(make_cfg(typeboundary=bc, dimsplit=True, **base))
    ctx.set_amr_grid(leaves, nb, [0.0] * nd, [1.0] * nd)
    ctx.upload(blocks)
    ctx.set_time(0.0, 1.0e99, 0.0)
    sl = (slice(None), slice(None), slice(2, 18), slice(2, 18))
    for n in range(3):
        dt, cg = og.getdt()
        ctx.step()
        og.advance(dt, cg)
        got = ctx.download()
        worst = max(_maxrel(got[b][sl][None], og.get_block(b)[sl][None]) for b in range(len(leaves)))
        tol = RTOL_MHD_TVDMU if (physics == "mhd" and kw["flux_scheme"] == "tvdmu") else RTOL
        assert worst <= tol, (name, n, worst)
    assert ctx.status() == 0


def test_advect1_dim_reproduces_a_split_step(oracle_lib):
    """The C ABI's one-direction stage (amrvac_gpu_advect1_dim): a split
    onestep step equals the x stage then the y stage through the ABI, bit for
    bit (same kernels, same dt)."""
    _cuda()
    from amrvac_b200 import Context, make_cfg
    n = 32
    prim = P.random_smooth("mhd", 2, 2, n, seed=P.SEED)
    blocks = P.to_blocks(P.prim_to_cons(prim, "mhd", 2, 5.0 / 3.0), 2)
    kw = dict(physics="mhd", ndim=2, flux_scheme="hlld", limiter="vanleer", typedivbfix="linde",
              time_stepper="onestep", dimsplit=True)
    a = Context(make_cfg(**kw))
    a.set_uniform_grid([n, n], [0.0, 0.0], [1.0, 1.0])
    a.upload(blocks)
    _, cg, _ = a.getdt("ps")
    a.set_time(0.0, 1.0e99, 0.0)
    a.step()
    dt = a.get_time()[0]
    b = Context(make_cfg(**kw))
    b.set_uniform_grid([n, n], [0.0, 0.0], [1.0, 1.0])
    b.upload(blocks)
    b.set_cmax_global(cg)
    b.advect1("ps", "ps1", 1.0, dt, idim=1)
    b.advect1("ps1", "ps", 1.0, dt, reg_base="ps1", idim=2)
    assert np.array_equal(a.download("ps"), b.download("ps"))
    a.close()
    b.close()
