"""fix_small_values on the GPU against the oracle, on fields with planted
small densities and pressures.

The reference fixes small values at three places of a stage: the conversion
of the ghosted block to primitives (hd_to_primitive / mhd_to_primitive_origin
calling phys_handle_small_values, src/hd/mod_hd_phys.t:703-734,
src/mhd/mod_mhd_phys.t:1741-1765), the reconstructed left and right face
states (src/mod_finite_volume.t:1212-1216) and the updated state on exit
(src/mod_finite_volume.t:326-333); the sound speeds clamp the thermal
pressure at small_pressure (src/hd/mod_hd_phys.t:1040-1045,
src/mhd/mod_mhd_phys.t:3573).  Method 'replace' (src/hd/mod_hd_phys.t:
1440-1466, src/mhd/mod_mhd_phys.t:2207-2225) sets density and pressure to
their floors and zeroes the momentum where the density is small; it raises
no error.  Each case plants a cell below small_density, one with negative
pressure and one on a block edge, and compares setdt and a full step cell by
cell (tests/_parity.py; bar 1e-12 or the oracle's own one-ulp noise).
"""
import numpy as np
import pytest

from tests import _problems as P
from tests._parity import one_ulp_noise, percell_err

pytestmark = pytest.mark.gpu

RTOL = 1e-12
SMALL = dict(fix_small_values=True, small_values_method="replace", small_density=1e-8, small_pressure=1e-8)

CASES = {
    "hd2_hll_minmod": dict(physics="hd", ndim=2, gamma=1.4, flux_scheme="hll", limiter="minmod"),
    "hd3_hllc_vanleer": dict(physics="hd", ndim=3, gamma=1.4, flux_scheme="hllc", limiter="vanleer"),
    "hd2_tvdlf_koren_twostep": dict(physics="hd", ndim=2, gamma=1.4, flux_scheme="tvdlf", limiter="koren",
                                    time_stepper="twostep"),
    "mhd3_hlld_cada3_glm": dict(physics="mhd", ndim=3, flux_scheme="hlld", limiter="cada3", typedivbfix="glm"),
    "mhd25_hll_vanleer_linde": dict(physics="mhd", ndim=2, ndir=3, flux_scheme="hll", limiter="vanleer",
                                    typedivbfix="linde"),
    "mhd2_hllc_minmod_none": dict(physics="mhd", ndim=2, flux_scheme="hllc", limiter="minmod", typedivbfix="none"),
}


def _cuda():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")


def _planted(physics, ndim, ndir, n, glm, gamma):
    """Conserved field with three planted cells: density 1e-10 (below the
    1e-8 floor, with pressure 1e-10), pressure -1e-3, and density 1e-10 on
    the last cell row of the first block along y (x in 1-D)."""
    prim = P.random_smooth(physics, ndim, ndir, n, glm=glm)
    ip = ndir + 1
    mid = tuple([n // 2 + 3] * ndim)[::-1]
    other = tuple([5] * ndim)[::-1]
    edge = tuple([7] * (ndim - 1) + [15])[::-1] if ndim > 1 else (15,)
    pad = (0,) * (3 - ndim)
    for cell, (rho, p) in ((mid, (1e-10, 1e-10)), (other, (None, -1e-3)), (edge, (1e-10, 1e-10))):
        ix = pad + cell
        if rho is not None:
            prim[(0,) + ix] = rho
        prim[(ip,) + ix] = p
    return P.prim_to_cons(prim, physics, ndir, gamma)


def _setup(O, name, noisy=False):
    from amrvac_b200 import Context, make_cfg
    kw = dict(CASES[name], **SMALL)
    nd = kw["ndim"]
    ndir = kw.get("ndir", nd)
    ok = dict(kw)
    ok["divb"] = ok.pop("typedivbfix", "none")
    ocfg = O.make_cfg(**ok)
    n = 32
    cons = _planted(kw["physics"], nd, ndir, n, ok["divb"] == "glm", ocfg.gamma)
    blocks = P.to_blocks(cons, nd)
    if noisy:
        blocks = one_ulp_noise(blocks)
    og = O.Grid(ocfg, [n] * nd, [0.0] * nd, [1.0] * nd, ["periodic"] * (2 * nd))
    for ib in range(og.nblocks):
        og.set_block(ib, blocks[ib])
    og.getbc()
    ctx = None
    if not noisy:
        ctx = Context(make_cfg(**kw))
        ctx.set_uniform_grid([n] * nd, [0.0] * nd, [1.0] * nd)
        ctx.upload(blocks)
    return og, ctx, nd


@pytest.mark.parametrize("name", sorted(CASES))
def test_replace_step_matches_oracle(oracle_lib, name):
    _cuda()
    O = oracle_lib
    og, ctx, nd = _setup(O, name)
    dt_ref, cg_ref = og.getdt()
    ctx.set_time(0.0, 1.0e99, 0.0)
    ctx.step()
    dt, cg, _ = ctx.get_time()
    assert abs(dt - dt_ref) <= 1e-13 * dt_ref and abs(cg - cg_ref) <= 1e-13 * cg_ref
    st = og.advance(dt_ref, cg_ref)
    gn = _setup(O, name, noisy=True)[0]
    gn.getdt()
    gn.advance(dt_ref, cg_ref)
    got = P.interior(ctx.download(), nd)
    ref = P.interior(np.array([og.get_block(ib) for ib in range(og.nblocks)]), nd)
    noise = percell_err(P.interior(np.array([gn.get_block(ib) for ib in range(gn.nblocks)]), nd), ref)
    err = percell_err(got, ref)
    assert np.isfinite(got).all()
    assert err <= max(RTOL, noise), f"{name}: {err:.3e} (oracle self-noise {noise:.3e})"
    # 'replace' repairs and carries on: no error status on either side
    assert ctx.status() == 0
    assert not (st or 0) & 1


def test_replace_floors_the_planted_cells(oracle_lib):
    """The planted cells stay at or above the floors after the step: the
    exit fix of the updated state ran (src/mod_finite_volume.t:326-333)."""
    _cuda()
    og, ctx, nd = _setup(oracle_lib, "hd2_hll_minmod")
    ctx.set_time(0.0, 1.0e99, 0.0)
    ctx.step()
    got = P.interior(ctx.download(), nd)
    assert got[:, 0].min() >= 1e-8


@pytest.mark.parametrize("name", ["hd2_hll_minmod", "hd3_hllc_vanleer", "mhd3_hlld_cada3_glm",
                                  "mhd25_hll_vanleer_linde"])
def test_mixed_form_takes_the_fp64_decisions(oracle_lib, name):
    """Mixed form (FP32 faces) with 'replace': the faces whose states come
    near a floor are recomputed from the FP64 state, so the replace
    decisions are the FP64 kernel's and no cell moves by more than FP32
    round-off against it (a different decision would move a cell by O(1):
    the momentum is zeroed)."""
    _cuda()
    from amrvac_b200 import Context, make_cfg
    og, ctx, nd = _setup(oracle_lib, name)
    kw = dict(CASES[name], **SMALL)
    blocks = ctx.download()
    ctx.set_time(0.0, 1.0e99, 0.0)
    ctx.step()
    ref = P.interior(ctx.download(), nd)
    mx = Context(make_cfg(precision="mixed", **kw))
    mx.set_uniform_grid([32] * nd, [0.0] * nd, [1.0] * nd)
    mx.upload(blocks)
    mx.set_time(0.0, 1.0e99, 0.0)
    mx.step()
    got = P.interior(mx.download(), nd)
    assert mx.status() == 0
    scale = np.abs(ref).reshape(ref.shape[0], ref.shape[1], -1).max(axis=(0, 2))
    dev = np.abs(got - ref).max(axis=(0, 2, 3, 4)) / scale
    assert dev.max() <= 1e-4, dev


# ---------------------------------------------------------------- 'average'
# small_values_average (src/mod_small_values.t:89-144): a flagged density or
# pressure becomes the mean of the unflagged values of the surrounding cube
# (half-width 1 .. small_values_daverage, clipped to the ghosted block) —
# on the ghosted block's conserved cells before the conversion to
# primitives, on the reconstructed face-state arrays, on the updated state
# (whose cube reaches the output register's ghost values) and after the
# GLM source; and on getdt's primitives.  The device detects the blocks
# where a check fires and recomputes them whole (csrc/smallavg.cu).
AVG_CASES = {
    "hd2_hll_minmod": dict(CASES["hd2_hll_minmod"]),
    "hd3_hllc_vanleer": dict(CASES["hd3_hllc_vanleer"]),
    "hd2_hllc_koren_ssprk2": dict(physics="hd", ndim=2, gamma=1.4, flux_scheme="hllc", limiter="koren",
                                  time_stepper="twostep", time_integrator="ssprk2"),
    "hd2_tvdlf_woodward_dav2": dict(physics="hd", ndim=2, gamma=1.4, flux_scheme="tvdlf", limiter="woodward",
                                    small_values_daverage=2),
    "mhd3_hlld_cada3_glm": dict(CASES["mhd3_hlld_cada3_glm"]),
    "mhd2_hllc_minmod_none": dict(CASES["mhd2_hllc_minmod_none"]),
    "mhd25_hll_vanleer_glm_fourstep": dict(physics="mhd", ndim=2, ndir=3, flux_scheme="hll", limiter="vanleer",
                                           typedivbfix="glm", time_stepper="fourstep"),
    # a smooth density minimum just above the floor: cada3 (not TVD at
    # extrema) reconstructs face densities below it, so the face-state fix
    # fires on many faces of a row
    "hd2_hllc_cada3_dip": dict(physics="hd", ndim=2, gamma=1.4, flux_scheme="hllc", limiter="cada3", dip=1e-8),
    # (at a 1e-8 floor the field's B ~ 0.4 makes HLLD non-finite in the
    # oracle too: Alfven speeds of 4e3)
    "mhd3_hlld_cada3_glm_dip": dict(physics="mhd", ndim=3, flux_scheme="hlld", limiter="cada3", typedivbfix="glm",
                                    dip=1e-3),
}


def _dip(physics, ndim, ndir, n, glm, gamma, floor):
    """Conserved field whose density has a smooth minimum of 1.02 floor
    across x = 10.3 cells, 0.1 floor (x - 10.3)^2 within four cells."""
    prim = P.random_smooth(physics, ndim, ndir, n, glm=glm)
    x = np.arange(n) + 0.5
    X = np.broadcast_to(x, prim.shape[1:])
    mask = np.abs(X - 10.3) < 4
    prim[0][mask] = (1.02 * floor + 0.1 * floor * (X - 10.3) ** 2)[mask]
    return P.prim_to_cons(prim, physics, ndir, gamma)


def _setup_avg(O, name, noisy=False):
    from amrvac_b200 import Context, make_cfg
    kw = dict(AVG_CASES[name], fix_small_values=True, small_values_method="average", small_density=1e-8,
              small_pressure=1e-8)
    dip = kw.pop("dip", None)
    if dip:
        kw["small_density"] = dip
    nd = kw["ndim"]
    ndir = kw.get("ndir", nd)
    ok = dict(kw)
    ok["divb"] = ok.pop("typedivbfix", "none")
    ocfg = O.make_cfg(**ok)
    n = 32
    if dip:
        cons = _dip(kw["physics"], nd, ndir, n, ok["divb"] == "glm", ocfg.gamma, dip)
    else:
        cons = _planted(kw["physics"], nd, ndir, n, ok["divb"] == "glm", ocfg.gamma)
    blocks = P.to_blocks(cons, nd)
    if noisy:
        blocks = one_ulp_noise(blocks)
    og = O.Grid(ocfg, [n] * nd, [0.0] * nd, [1.0] * nd, ["periodic"] * (2 * nd))
    for ib in range(og.nblocks):
        og.set_block(ib, blocks[ib])
    og.getbc()
    ctx = None
    if not noisy:
        ctx = Context(make_cfg(**kw))
        ctx.set_uniform_grid([n] * nd, [0.0] * nd, [1.0] * nd)
        ctx.upload(blocks)
    return og, ctx, nd


@pytest.mark.parametrize("name", sorted(AVG_CASES))
def test_average_steps_match_oracle(oracle_lib, name):
    """setdt and two full steps with 'average' on the planted field."""
    _cuda()
    O = oracle_lib
    og, ctx, nd = _setup_avg(O, name)
    gn = _setup_avg(O, name, noisy=True)[0]
    ctx.set_time(0.0, 1.0e99, 0.0)
    for step in range(2):
        dt_ref, cg_ref = og.getdt()
        gn.getdt()
        ctx.step()
        dt, cg, _ = ctx.get_time()
        assert abs(dt - dt_ref) <= 1e-13 * dt_ref and abs(cg - cg_ref) <= 1e-13 * cg_ref, (step, dt, dt_ref)
        og.advance(dt_ref, cg_ref)
        gn.advance(dt_ref, cg_ref)
        got = P.interior(ctx.download(), nd)
        ref = P.interior(np.array([og.get_block(ib) for ib in range(og.nblocks)]), nd)
        noise = percell_err(P.interior(np.array([gn.get_block(ib) for ib in range(gn.nblocks)]), nd), ref)
        err = percell_err(got, ref)
        assert np.isfinite(got).all()
        assert err <= max(RTOL, noise), f"{name} step {step}: {err:.3e} (oracle self-noise {noise:.3e})"
    assert ctx.status() == 0


def test_average_graph_replay_matches_direct_steps(oracle_lib):
    """The captured step graph (amrvac_gpu_run) holds the detection, the
    register copy and the whole-block recomputation: three replayed steps
    give the directly launched steps bit for bit."""
    _cuda()
    O = oracle_lib
    _, a, nd = _setup_avg(O, "mhd3_hlld_cada3_glm_dip")
    _, b, _ = _setup_avg(O, "mhd3_hlld_cada3_glm_dip")
    a.set_time(0.0, 1.0e99, 0.0)
    b.set_time(0.0, 1.0e99, 0.0)
    for _ in range(3):
        a.step()
    b.run(3)
    assert np.array_equal(a.download(), b.download())
    assert a.status() == 0 and b.status() == 0


@pytest.mark.parametrize("bn,bc", [(8, "cont"), (16, "symm")])
def test_average_block_edges_and_physical_sides(oracle_lib, bn, bc):
    """'average' on 8^3 blocks with 'cont' sides and on 16^3 blocks with
    'symm' sides: the cubes of cells next to the domain boundary reach the
    physical ghost cells, which the device gathers as the reference's
    boundary fill leaves them; two full steps against the oracle."""
    _cuda()
    from amrvac_b200 import Context, make_cfg
    O = oracle_lib
    kw = dict(physics="hd", ndim=3, gamma=1.4, flux_scheme="hllc", limiter="cada3", fix_small_values=True,
              small_values_method="average", small_density=1e-3, small_pressure=1e-8)
    n = 2 * bn
    ocfg = O.make_cfg(block_nx=bn, **kw)

    def grid(noisy):
        cons = _dip("hd", 3, 3, n, False, ocfg.gamma, 1e-3)
        blocks = P.to_blocks(cons, 3, bn=bn)
        if noisy:
            blocks = one_ulp_noise(blocks)
        g = O.Grid(ocfg, [n] * 3, [0.0] * 3, [1.0] * 3, [bc] * 6)
        for ib in range(g.nblocks):
            g.set_block(ib, blocks[ib])
        g.getbc()
        return g, blocks
    og, blocks = grid(False)
    gn, _ = grid(True)
    ctx = Context(make_cfg(block_nx=bn, typeboundary=[bc] * 6, **kw))
    ctx.set_uniform_grid([n] * 3, [0.0] * 3, [1.0] * 3)
    ctx.upload(blocks)
    ctx.set_time(0.0, 1.0e99, 0.0)
    for step in range(2):
        dt_ref, cg_ref = og.getdt()
        gn.getdt()
        ctx.step()
        dt = ctx.get_time()[0]
        assert abs(dt - dt_ref) <= 1e-13 * dt_ref
        og.advance(dt_ref, cg_ref)
        gn.advance(dt_ref, cg_ref)
        got = P.interior(ctx.download(), 3)
        ref = P.interior(np.array([og.get_block(ib) for ib in range(og.nblocks)]), 3)
        noise = percell_err(P.interior(np.array([gn.get_block(ib) for ib in range(gn.nblocks)]), 3), ref)
        err = percell_err(got, ref)
        assert err <= max(RTOL, noise), (bn, bc, step, err, noise)
    assert ctx.status() == 0


@pytest.mark.parametrize("name", ["hd2_hll_minmod", "hd2_hllc_cada3_dip", "mhd3_hlld_cada3_glm",
                                  "mhd3_hlld_cada3_glm_dip"])
def test_average_mixed_form_takes_the_fp64_decisions(oracle_lib, name):
    """Mixed form (FP32 faces) with 'average': a face state near a floor is
    recomputed in FP64, so the blocks the whole-block path recomputes (in
    FP64) are the FP64 kernel's, and after two steps no cell is further from
    the FP64 run than FP32 round-off (a missed average would leave a cell at
    the floor or below it: an O(1) difference)."""
    _cuda()
    from amrvac_b200 import Context, make_cfg
    _, c64, nd = _setup_avg(oracle_lib, name)
    kw = dict(AVG_CASES[name], fix_small_values=True, small_values_method="average", small_density=1e-8,
              small_pressure=1e-8)
    dip = kw.pop("dip", None)
    if dip:
        kw["small_density"] = dip
    blocks = c64.download()
    mx = Context(make_cfg(precision="mixed", **kw))
    mx.set_uniform_grid([32] * nd, [0.0] * nd, [1.0] * nd)
    mx.upload(blocks)
    for c in (c64, mx):
        c.set_time(0.0, 1.0e99, 0.0)
        c.step()
        c.step()
    ref = P.interior(c64.download(), nd)
    got = P.interior(mx.download(), nd)
    assert c64.status() == 0 and mx.status() == 0
    assert np.isfinite(got).all() and got[:, 0].min() >= kw["small_density"] * (1 - 1e-6)
    scale = np.abs(ref).reshape(ref.shape[0], ref.shape[1], -1).max(axis=(0, 2))
    dev = np.abs(got - ref).reshape(ref.shape[0], ref.shape[1], -1).max(axis=(0, 2)) / scale
    assert dev.max() <= 1e-4, dev


@pytest.mark.parametrize("name,presteps", [("hd2_hll_minmod", 0), ("hd2_hllc_cada3_dip", 1),
                                           ("mhd3_hlld_cada3_glm_dip", 1)])
def test_average_mixed_form_recomputes_the_fp64_blocks(oracle_lib, name, presteps):
    """One stage from the same state (the planted field, or the dip after one
    FP64 step, when cada3 first reconstructs face densities below the
    floor): every block where a small-value fix fires — the oracle's
    'average' and 'replace' stages differ there — is recomputed in FP64 by
    the whole-block path in the mixed form too, so it is bit-identical to the
    FP64 run's; the other blocks differ from it by FP32 round-off only."""
    _cuda()
    from amrvac_b200 import Context, make_cfg
    O = oracle_lib
    og, c64, nd = _setup_avg(O, name)
    kw = dict(AVG_CASES[name], fix_small_values=True, small_values_method="average", small_density=1e-8,
              small_pressure=1e-8)
    dip = kw.pop("dip", None)
    if dip:
        kw["small_density"] = dip
    ok = dict(kw)
    ok["divb"] = ok.pop("typedivbfix", "none")
    rep = O.make_cfg(**dict(ok, small_values_method="replace"))
    avg = O.make_cfg(**ok)
    c64.set_time(0.0, 1.0e99, 0.0)
    for _ in range(presteps):
        c64.step()
    state = c64.download()
    for ib in range(og.nblocks):
        og.set_block(ib, state[ib])
    og.getbc()
    dt, cg = og.getdt()
    dt *= 0.5
    fired = []
    for ib in range(og.nblocks):
        w = og.get_block(ib)
        wa, wr = w.copy(), w.copy()
        O.finite_volume(avg, w, wa, dt, og.dx(), cg)
        O.finite_volume(rep, w, wr, dt, og.dx(), cg)
        fired.append(not np.array_equal(wa, wr))
    assert any(fired) and not all(fired), fired
    mx = Context(make_cfg(precision="mixed", **kw))
    mx.set_uniform_grid([32] * nd, [0.0] * nd, [1.0] * nd)
    for c in (c64, mx):
        c.upload(state)
        c.set_cmax_global(cg)
        assert c.advect1("ps", "ps1", 1.0, dt) == 0
    ref = P.interior(c64.download("ps1"), nd)
    got = P.interior(mx.download("ps1"), nd)
    scale = np.abs(ref).reshape(ref.shape[0], ref.shape[1], -1).max(axis=(0, 2))
    for ib, f in enumerate(fired):
        if f:
            assert np.array_equal(got[ib], ref[ib]), ib
        else:
            dev = np.abs(got[ib] - ref[ib]).reshape(ref.shape[1], -1).max(axis=1) / scale
            assert dev.max() <= 1e-4, (ib, dev)
    assert c64.status() == 0 and mx.status() == 0
