"""Fifth-order reconstructions (three ghost cells) on the GPU against the
oracle: MP5 and the WENO5 family.

The stage kernel stages a three-cell halo (a six-plane z ring in 3-D) and
reconstructs each face from six cells with MP5limiter's formulas, then
fix_limiter1's fallback; the oracle restates MP5limiter
(src/limiter/mod_mp5.t:16-201).  Bars as for the other limiters: ghost
fill bit-exact (now three layers), one stage and full steps <= 1e-12.
"""
import numpy as np
import pytest

from tests._parity import percell_err

from tests import _problems as P

pytestmark = pytest.mark.gpu

RTOL = 1e-12

CASES = {
    "hd2_hllc_mp5": dict(physics="hd", ndim=2, gamma=1.4, flux_scheme="hllc"),
    "hd2_hll_mp5_cont": dict(physics="hd", ndim=2, gamma=1.4, flux_scheme="hll", bc=["cont"] * 4),
    "hd3_hll_mp5": dict(physics="hd", ndim=3, gamma=1.4, flux_scheme="hll"),
    "hd3_hllc_mp5_symm": dict(physics="hd", ndim=3, gamma=1.4, flux_scheme="hllc",
                              bc=["symm", "symm", "periodic", "periodic", "cont", "cont"]),
    "mhd2_hll_mp5_linde": dict(physics="mhd", ndim=2, flux_scheme="hll", typedivbfix="linde"),
    "mhd2_hlld_mp5_none": dict(physics="mhd", ndim=2, flux_scheme="hlld", typedivbfix="none"),
    "mhd25_hlld_mp5_glm": dict(physics="mhd", ndim=2, ndir=3, flux_scheme="hlld", typedivbfix="glm"),
    "mhd3_hlld_mp5_glm": dict(physics="mhd", ndim=3, flux_scheme="hlld", typedivbfix="glm"),
    "mhd3_hll_mp5_glm_pc": dict(physics="mhd", ndim=3, flux_scheme="hll", typedivbfix="glm",
                                time_stepper="twostep"),
    "hd2_hll_mp5_ssprk54": dict(physics="hd", ndim=2, gamma=1.4, flux_scheme="hll", time_stepper="fivestep"),
    # the WENO5 family (WENO5limiter: JS, Z, Z+)
    "hd2_hllc_weno5": dict(physics="hd", ndim=2, gamma=1.4, flux_scheme="hllc", limiter="weno5"),
    "hd2_hll_wenozp5_cont": dict(physics="hd", ndim=2, gamma=1.4, flux_scheme="hll", limiter="wenozp5",
                                 bc=["cont"] * 4),
    "hd3_hll_wenoz5": dict(physics="hd", ndim=3, gamma=1.4, flux_scheme="hll", limiter="wenoz5"),
    "mhd2_hll_weno5_linde": dict(physics="mhd", ndim=2, flux_scheme="hll", limiter="weno5", typedivbfix="linde"),
    "mhd25_hlld_wenozp5_glm": dict(physics="mhd", ndim=2, ndir=3, flux_scheme="hlld", limiter="wenozp5",
                                   typedivbfix="glm"),
    "mhd3_hlld_wenoz5_glm": dict(physics="mhd", ndim=3, flux_scheme="hlld", limiter="wenoz5", typedivbfix="glm"),
}


def _cuda():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")


def _setup(oracle_lib, name, n=32):
    from amrvac_b200 import Context, make_cfg
    O = oracle_lib
    kw = dict(CASES[name])
    bc = kw.pop("bc", None)
    limiter = kw.pop("limiter", "mp5")
    ndim = kw["ndim"]
    ndir = kw.get("ndir", ndim)
    bc = bc or ["periodic"] * (2 * ndim)
    gcfg = make_cfg(typeboundary=bc, limiter=limiter, **kw)
    assert gcfg.nghostcells == 3
    ok = dict(kw)
    div = ok.pop("typedivbfix", "none")
    ocfg = O.make_cfg(divb=div, limiter=limiter, nghost=3, **ok)
    glm = kw.get("typedivbfix") == "glm"
    prim = P.random_smooth(kw["physics"], ndim, ndir, n, seed=P.SEED, glm=glm)
    cons = P.prim_to_cons(prim, kw["physics"], ndir, ocfg.gamma)
    blocks = P.to_blocks(cons, ndim, nghost=3)
    dom = [n] * ndim
    og = O.Grid(ocfg, dom, [0.0] * ndim, [1.0] * ndim, bc)
    for ib in range(og.nblocks):
        og.set_block(ib, blocks[ib])
    og.getbc()
    ctx = Context(gcfg)
    ctx.set_uniform_grid(dom, [0.0] * ndim, [1.0] * ndim)
    ctx.upload(blocks)
    return O, ocfg, og, ctx


def _maxrel(a, b):
    """Per-cell parity measure (tests/_parity.py): relative error for cells
    >= 1e-3 of the variable's maximum, absolute at that scale below it."""
    return percell_err(a, b, var_axis=1)


@pytest.mark.parametrize("name", sorted(CASES))
def test_mp5_ghost_fill_three_layers(oracle_lib, name):
    _cuda()
    O, ocfg, og, ctx = _setup(oracle_lib, name)
    ref = np.array([og.get_block(ib) for ib in range(og.nblocks)])
    got = ctx.download()
    assert got.shape == ref.shape and got.shape[-1] == 22
    assert np.array_equal(got, ref)


@pytest.mark.parametrize("name", sorted(CASES))
def test_mp5_stage_matches_oracle(oracle_lib, name):
    _cuda()
    O, ocfg, og, ctx = _setup(oracle_lib, name)
    dt, cg = og.getdt()
    dt *= 0.5
    ctx.set_cmax_global(cg)
    assert ctx.advect1("ps", "ps1", 1.0, dt) == 0
    got = P.interior(ctx.download("ps1"), ocfg.ndim, nghost=3)
    dx = og.dx()
    ref = []
    for ib in range(og.nblocks):
        w = og.get_block(ib)
        wn = w.copy()
        O.finite_volume(ocfg, w, wn, dt, dx, cg)
        ref.append(wn)
    ref = P.interior(np.array(ref), ocfg.ndim, nghost=3)
    err = _maxrel(got, ref)
    assert err <= RTOL, f"{name}: max rel err {err:.3e}"
    assert ctx.status() == 0


@pytest.mark.parametrize("name", sorted(CASES))
def test_mp5_steps_match_oracle(oracle_lib, name):
    _cuda()
    O, ocfg, og, ctx = _setup(oracle_lib, name)
    ctx.set_time(0.0, 1.0e99, 0.0)
    for _ in range(3):
        dt_ref, cg_ref = og.getdt()
        ctx.step()
        dt, cg, _t = ctx.get_time()
        assert abs(dt - dt_ref) <= 1e-12 * dt_ref
        og.advance(dt_ref, cg_ref)
    got = P.interior(ctx.download("ps"), ocfg.ndim, nghost=3)
    ref = P.interior(np.array([og.get_block(ib) for ib in range(og.nblocks)]), ocfg.ndim, nghost=3)
    err = _maxrel(got, ref)
    assert err <= RTOL, f"{name}: max rel err {err:.3e}"
    assert ctx.status() == 0


def test_mp5_conserves_on_periodic_domain(oracle_lib):
    _cuda()
    O, ocfg, og, ctx = _setup(oracle_lib, "hd3_hll_mp5")
    before = P.interior(ctx.download(), 3, nghost=3).sum(axis=(0, 2, 3, 4))
    ctx.set_time(0.0, 1.0e99, 0.0)
    ctx.run(4)
    blocks = P.interior(ctx.download(), 3, nghost=3)
    after = blocks.sum(axis=(0, 2, 3, 4))
    scale = np.abs(blocks).sum(axis=(0, 2, 3, 4))
    assert np.all(np.abs(after - before) <= 1e-13 * scale)


def _device_l1_error(n, limiter="mp5", tend=0.1):
    """The oracle-side accuracy pin (tests/test_oracle_mp5_cpu.py) on the
    device: a smooth density wave advected at v = (1, 0)."""
    from amrvac_b200 import Context, make_cfg
    cfg = make_cfg(physics="hd", ndim=2, gamma=1.4, flux_scheme="hll", limiter=limiter, courantpar=0.1)
    x = (np.arange(n) + 0.5) / n
    X, _ = np.meshgrid(x, x, indexing="xy")
    k, h = 2.0 * np.pi, 1.0 / n
    sinc = np.sin(k * h / 2) / (k * h / 2)

    def cons_of(rho_avg):
        prim = np.zeros((4, 1, n, n))
        prim[0, 0] = rho_avg
        prim[1], prim[3] = 1.0, 1.0
        return P.prim_to_cons(prim, "hd", 2, 1.4)
    ctx = Context(cfg)
    ctx.set_uniform_grid([n, n], [0.0, 0.0], [1.0, 1.0])
    ctx.upload(P.to_blocks(cons_of(1.0 + 0.2 * np.sin(k * X) * sinc), 2, nghost=3))
    ctx.set_time(0.0, tend, 0.0)
    for _ in range(100000):
        ctx.step()
        if ctx.get_time()[2] >= tend - 1e-12:
            break
    got = P.interior(ctx.download(), 2, nghost=3)
    ex = P.interior(P.to_blocks(cons_of(1.0 + 0.2 * np.sin(k * (X - tend)) * sinc), 2, nghost=3), 2, nghost=3)
    ctx.close()
    return float(np.abs(got[:, 0] - ex[:, 0]).mean())


@pytest.mark.parametrize("limiter", ["mp5", "weno5", "wenoz5", "wenozp5"])
def test_fifth_order_on_smooth_wave(limiter):
    _cuda()
    e32, e64 = _device_l1_error(32, limiter), _device_l1_error(64, limiter)
    assert 24.0 < e32 / e64 < 40.0, (e32, e64)
