"""The reference's golden regression logs reproduced on the GPU path.

Field loop 2.5D (tests/mhd/field_loop_2.5D, reference): the whole time loop
(setdt with dtsave/time_max clipping, SSP-RK3, getbc) runs on the device; the
host downloads the state at each log time and forms the regression-log row
(printlog_regression_test, src/io/mod_input_output.t:2653-2729).  Accepted with
the reference's compare_logs rule, rtol=1e-5, atol=1e-8.
"""
import os

import numpy as np
import pytest

from tests import _problems as P

pytestmark = pytest.mark.gpu
GOLD = os.path.join(os.path.dirname(__file__), "golden")


def _run_field_loop_gpu(kw, nwflux, time_max=0.5, dtsave=0.01):
    from amrvac_b200 import Context, make_cfg
    cfg = make_cfg(physics="mhd", ndim=2, ndir=3, courantpar=0.9, **kw)
    ctx = Context(cfg)
    ctx.set_uniform_grid(P.FL["domain_nx"], P.FL["xprobmin"], P.FL["xprobmax"])
    ctx.upload(P.field_loop_blocks()[:, :nwflux])
    ctx.set_time(0.0, time_max, dtsave)
    rows = []
    t, tsavelast = 0.0, 0.0
    for _ in range(100000):
        ctx.step()
        dt, cg, t = ctx.get_time()
        if t >= tsavelast + dtsave - 1e-12:
            tsavelast = t
            rows.append(P.field_loop_log_row(ctx.download(), t, nwflux))
        if t >= time_max - 1e-10:
            break
    assert ctx.status() == 0
    return np.array(rows)


@pytest.mark.parametrize("name,kw,nw", [
    ("hlld", dict(flux_scheme="hlld", limiter="cada3", typedivbfix="glm"), 9),
    ("hll", dict(flux_scheme="hll", limiter="cada3", typedivbfix="linde", typeboundspeed="cmaxmean"), 8),
])
def test_field_loop_golden_log_gpu(oracle_lib, name, kw, nw):
    rows = _run_field_loop_gpu(kw, nw)
    gold = oracle_lib.read_log(os.path.join(GOLD, f"fl_2d_3step_{name}_cada.log"))
    assert rows.shape == gold.shape
    assert oracle_lib.compare_logs(rows, gold, rtol=1e-5, atol=1e-8)
    ib = 1 + nw + 2
    rel = np.abs(rows[:, ib] - gold[:, ib]) / np.abs(gold[:, ib])
    assert rel.max() < 1e-5


# ---------------------------------------------------------------- multi-level
# Orszag-Tang 2-D (tests/mhd/Orszag_Tang_2D, reference): 64^2 level-1 cells in
# 16^2 blocks on [0,1]^2, periodic, refine_max_level 3, Löhner on rho and e
# (w_refine_weight 0.5 each, refine_threshold 0.4), the initial tree by
# settree on the initial condition and a resettree after every step
# (ditregrid = 1), log every 1e-3 to t = 0.1.


def _ot2d_prim(nw):
    rho0, p0, b0 = 25.0 / 36.0 / np.pi, 5.0 / 12.0 / np.pi, 1.0 / np.sqrt(4.0 * np.pi)

    def f(X, Y, Z):
        out = np.zeros((nw,) + X.shape)
        out[0] = rho0
        out[1] = -np.sin(2.0 * np.pi * Y)
        out[2] = np.sin(2.0 * np.pi * X)
        out[3] = p0
        out[4] = -b0 * np.sin(2.0 * np.pi * Y)
        out[5] = b0 * np.sin(4.0 * np.pi * X)
        return out
    return f


def _amr_log_row(blocks, leaves, nbase, t, nw, nd=2, bn=16, xlen=1.0):
    """printlog_regression_test: volume averages of w and w**2 over the leaves
    (xlen: the domain length, one value or one per dimension)."""
    s1, s2, vol = np.zeros(nw), np.zeros(nw), 0.0
    sl = (slice(None, nw),) + tuple(slice(2, 2 + bn) if d < nd else slice(None) for d in (2, 1, 0))
    xl = np.broadcast_to(np.asarray(xlen, float), (nd,))
    for b, lf in enumerate(leaves):
        dv = 1.0
        for d in range(nd):
            dv *= xl[d] / (nbase[d] * bn * (1 << (lf[0] - 1)))
        w = blocks[b][sl].reshape(nw, -1)
        s1 += w.sum(axis=1) * dv
        s2 += (w * w).sum(axis=1) * dv
        vol += bn ** nd * dv
    return np.concatenate([[t], s1 / vol, s2 / vol])


def _run_amr_golden(physics, nb, prim_fn, weight, threshold, kw, time_max, dtsave=1.0e-3, levels=3, xmax=1.0,
                    bc="periodic", nd=2, bn=16, xmin=0.0):
    """The reference's time loop on a multi-level grid over [xmin, xmax]^nd
    (one value or one per dimension) with blocks of bn^nd cells: settree,
    then setdt + advance + resettree every step, a log row at every dtsave.
    bc: one boundary for every side, or one per side (min1, max1, ...)."""
    from tests import _amr as A
    from amrvac_b200 import Context, make_cfg
    from amrvac_b200.amr import Tree, initial_hierarchy, lohner_flags
    nw = len(weight)
    xmin = list(np.broadcast_to(np.asarray(xmin, float), (nd,)))
    xmax = list(np.broadcast_to(np.asarray(xmax, float), (nd,)))
    xlen = [b - a for a, b in zip(xmin, xmax)]
    bcs = [bc] * (2 * nd) if isinstance(bc, str) else list(bc)
    cfg = make_cfg(physics=physics, ndim=nd, ndir=nd, typeboundary=bcs, block_nx=bn, **kw)
    ctx = Context(cfg)
    lkw = dict(refine_threshold=threshold, derefine_ratio=0.125, amr_wavefilter=1.0e-2)

    def init(tree):
        return A.fill_blocks(tree.leaves, nd, nb, prim_fn, physics, nd, cfg.gamma, xmin, xmax, bn=bn)

    def err(tree, blocks):
        r, c, _ = lohner_flags(ctx, tree, blocks, xmin, xmax, weight, **lkw)
        return r, c
    tree, blocks = initial_hierarchy(Tree(nd, nb, levels, periodic=[bcs[2 * d] == "periodic" for d in range(nd)]),
                                     init, err)
    ctx.set_amr_grid(tree.leaves, nb, xmin, xmax)
    ctx.upload(blocks)
    ctx.set_time(0.0, time_max, dtsave)
    rows = []
    tsavelast = 0.0
    for _ in range(100000):
        ctx.step()
        ctx.amr_resettree(weight, refine_max_level=levels, **lkw)
        dt, cg, t = ctx.get_time()
        if t >= tsavelast + dtsave - 1e-12:
            tsavelast = t
            rows.append(_amr_log_row(ctx.download(), ctx.amr_leaves(), nb, t, nw, nd, bn, xlen))
        if t >= time_max - 1e-10:
            break
    assert ctx.status() == 0
    ctx.close()
    return np.array(rows)


@pytest.mark.parametrize("name,kw,nw", [
    ("3step_hlld_cada", dict(flux_scheme="hlld", limiter="cada3", typedivbfix="glm", courantpar=0.9), 7),
    ("3step_hll_cada", dict(flux_scheme="hll", limiter="cada3", typedivbfix="linde", typeboundspeed="cmaxmean",
                            courantpar=0.9), 6),
    ("4step_hll_mc", dict(flux_scheme="hll", limiter="woodward", typedivbfix="linde", typeboundspeed="cmaxmean",
                          courantpar=0.9, time_stepper="fourstep", time_integrator="rk4"), 6),
    ("rk4_tvdlf_cada", dict(flux_scheme="tvdlf", limiter="cada3", typedivbfix="linde", typeboundspeed="cmaxmean",
                            courantpar=0.9, time_stepper="fourstep", time_integrator="rk4"), 6),
    ("2step_tvdlf_mm", dict(flux_scheme="tvdlf", limiter="minmod", typedivbfix="linde", typeboundspeed="cmaxmean",
                            courantpar=0.9, time_stepper="twostep"), 6),
    ("4step_hllc_ko", dict(flux_scheme="hllc", limiter="koren", typedivbfix="linde", typeboundspeed="cmaxmean",
                           courantpar=0.9, time_stepper="fourstep"), 6),
    ("2step_tvdmu_al", dict(flux_scheme="tvdmu", limiter="albada", typedivbfix="linde", typeboundspeed="cmaxmean",
                            courantpar=0.9, time_stepper="twostep", dimsplit=True), 6),
])
def test_orszag_tang_2d_amr_golden_log_gpu(oracle_lib, name, kw, nw):
    weight = np.zeros(nw)
    weight[0] = weight[3] = 0.5  # w_refine_weight(1) = w_refine_weight(4) = 0.5
    rows = _run_amr_golden("mhd", [4, 4], _ot2d_prim(nw), weight, 0.4, kw, time_max=0.1)
    gold = oracle_lib.read_log(os.path.join(GOLD, f"ot_2d_{name}.log"))
    assert rows.shape == gold.shape, (rows.shape, gold.shape)
    bad = np.abs(rows - gold) > 1e-8 + 1e-5 * np.abs(gold)
    assert oracle_lib.compare_logs(rows, gold, rtol=1e-5, atol=1e-8), (
        np.argwhere(bad)[:10].tolist(), rows[bad][:10].tolist(), gold[bad][:10].tolist())


# Kelvin-Helmholtz 2-D (tests/hd/Kelvin_Helmholtz_2D, reference, iprob 1):
# 32^2 level-1 cells in 16^2 blocks, periodic, refine_max_level 3 with the
# default estimator settings (w_refine_weight(1) = 1, refine_threshold 0.1),
# slowsteps 10; schemes 3step_hll_cada (SSP-RK3, HLL, cada3), 4step_hll_mc
# (RK4, HLL, woodward) and 4step_hllc_ko (SSPRK(4,3), HLLC, koren), all with
# cmaxmean and CFL 0.9.


def _kh2d_prim(X, Y, Z):
    rhodens, rholight, kx, pint, dlin, sigma, vextra = 10.0, 1.0, 4.0 * np.pi, 2.5, 0.025, 0.00125, 0.0
    out = np.zeros((4,) + X.shape)
    out[0] = np.where((Y < 0.25) | (Y > 0.75), rholight, rhodens)
    out[3] = pint
    vx = np.zeros_like(X)
    vx = np.where((Y <= 0.25 - dlin) | (Y >= 0.75 + dlin), vextra - 0.5, vx)
    vx = np.where((Y >= 0.25 + dlin) & (Y <= 0.75 - dlin), vextra + 0.5, vx)
    low = (Y > 0.25 - dlin) & (Y < 0.25 + dlin)
    vx = np.where(low, (Y - (0.25 - dlin)) * ((vextra + 0.5) - (vextra - 0.5)) / (2.0 * dlin) + (vextra - 0.5), vx)
    high = (Y > 0.75 - dlin) & (Y < 0.75 + dlin)
    vx = np.where(high, (Y - (0.75 - dlin)) * ((vextra - 0.5) - (vextra + 0.5)) / (2.0 * dlin) + (vextra + 0.5), vx)
    out[1] = vx
    out[2] = 0.01 * np.sin(kx * X) * (np.exp(-0.5 * (Y - 0.25) ** 2 / sigma) + np.exp(-0.5 * (Y - 0.75) ** 2 / sigma))
    return out


@pytest.mark.parametrize("name,kw", [
    ("3step_hll_cada", dict(flux_scheme="hll", limiter="cada3", typeboundspeed="cmaxmean")),
    ("4step_hll_mc", dict(flux_scheme="hll", limiter="woodward", typeboundspeed="cmaxmean", time_stepper="fourstep",
                          time_integrator="rk4")),
    ("4step_hllc_ko", dict(flux_scheme="hllc", limiter="koren", typeboundspeed="cmaxmean", time_stepper="fourstep")),
    ("rk4_tvdlf_cada", dict(flux_scheme="tvdlf", limiter="cada3", typeboundspeed="cmaxmean", time_stepper="fourstep",
                            time_integrator="rk4")),
])
def test_kelvin_helmholtz_2d_amr_golden_log_gpu(oracle_lib, name, kw):
    kw = dict(kw, courantpar=0.9, slowsteps=10)
    rows = _run_amr_golden("hd", [2, 2], _kh2d_prim, np.array([1.0, 0.0, 0.0, 0.0]), 0.1, kw, time_max=0.05)
    gold = oracle_lib.read_log(os.path.join(GOLD, f"kh_2d_{name}.log"))
    assert rows.shape == gold.shape, (rows.shape, gold.shape)
    bad = np.abs(rows - gold) > 1e-8 + 1e-5 * np.abs(gold)
    assert oracle_lib.compare_logs(rows, gold, rtol=1e-5, atol=1e-8), (
        np.argwhere(bad)[:10].tolist(), rows[bad][:10].tolist(), gold[bad][:10].tolist())


# Blast wave 2-D (tests/hd/blast_wave_Cartesian_2D, reference): [0,2]^2,
# 32^2 level-1 cells in 16^2 blocks, cont boundaries, refine_max_level 3 with
# w_refine_weight(1) = w_refine_weight(4) = 0.5, p = 100 for r < 0.2 around
# the centre, rho = 1, p = 1, v = 0; log every 1e-3 to t = 0.05.


def _bw2d_prim(X, Y, Z):
    out = np.zeros((4,) + X.shape)
    out[0] = 1.0
    out[3] = np.where((X - 1.0) ** 2 + (Y - 1.0) ** 2 < 0.2 ** 2, 100.0, 1.0)
    return out


@pytest.mark.parametrize("name,kw", [
    ("3step_hll_cada", dict(flux_scheme="hll", limiter="cada3", typeboundspeed="cmaxmean")),
    ("4step_hll_mc", dict(flux_scheme="hll", limiter="woodward", typeboundspeed="cmaxmean", time_stepper="fourstep",
                          time_integrator="rk4")),
    ("4step_hllc_ko", dict(flux_scheme="hllc", limiter="koren", typeboundspeed="cmaxmean", time_stepper="fourstep")),
    ("rk4_tvdlf_cada", dict(flux_scheme="tvdlf", limiter="cada3", typeboundspeed="cmaxmean", time_stepper="fourstep",
                            time_integrator="rk4")),
    ("2step_tvdlf_mm", dict(flux_scheme="tvdlf", limiter="minmod", typeboundspeed="cmaxmean", time_stepper="twostep")),
    ("2step_tvdmu_al", dict(flux_scheme="tvdmu", limiter="albada", typeboundspeed="cmaxmean", time_stepper="twostep",
                            dimsplit=True)),
])
def test_blast_wave_2d_amr_golden_log_gpu(oracle_lib, name, kw):
    kw = dict(kw, courantpar=0.9)
    weight = np.array([0.5, 0.0, 0.0, 0.5])
    rows = _run_amr_golden("hd", [2, 2], _bw2d_prim, weight, 0.1, kw, time_max=0.05, xmax=2.0, bc="cont")
    gold = oracle_lib.read_log(os.path.join(GOLD, f"bw_2d_{name}.log"))
    assert rows.shape == gold.shape, (rows.shape, gold.shape)
    bad = np.abs(rows - gold) > 1e-8 + 1e-5 * np.abs(gold)
    assert oracle_lib.compare_logs(rows, gold, rtol=1e-5, atol=1e-8), (
        np.argwhere(bad)[:10].tolist(), rows[bad][:10].tolist(), gold[bad][:10].tolist())


# Blast wave 3-D MHD (tests/mhd/blast_wave_Cartesian_3D, reference): [0,2]^3,
# 16^3 level-1 cells in 8^3 blocks (block_nx 8), cont boundaries,
# refine_max_level 3 with w_refine_weight(1) = w_refine_weight(5) = 0.5 and
# refine_threshold 0.2, rho = 1, p = 1 with p = 100 for r < 0.2 around the
# centre, v = 0, B = (1, 1, 1) (Busr = 1), psi = 0; small_density =
# small_pressure = 1e-14 with fix_small_values; log every 1e-3 to t = 0.02.
# The first golden logs of the 3-D path and of a block edge other than 16.


def _bw3d_prim(nw):
    def f(X, Y, Z):
        out = np.zeros((nw,) + X.shape)
        out[0] = 1.0
        out[4] = np.where((X - 1.0) ** 2 + (Y - 1.0) ** 2 + (Z - 1.0) ** 2 < 0.2 ** 2, 100.0, 1.0)
        out[5] = out[6] = out[7] = 1.0
        return out
    return f


@pytest.mark.parametrize("name,kw,nw", [
    ("3step_hlld_cada", dict(flux_scheme="hlld", limiter="cada3", typedivbfix="glm"), 9),
    ("3step_hll_cada", dict(flux_scheme="hll", limiter="cada3", typedivbfix="linde", typeboundspeed="cmaxmean"), 8),
    ("3step_hll_ko", dict(flux_scheme="hll", limiter="koren", typedivbfix="linde", typeboundspeed="cmaxmean"), 8),
    ("4step_hll_mc", dict(flux_scheme="hll", limiter="woodward", typedivbfix="linde", typeboundspeed="cmaxmean",
                          time_stepper="fourstep", time_integrator="rk4"), 8),
    ("4step_hllc_ko", dict(flux_scheme="hllc", limiter="koren", typedivbfix="linde", typeboundspeed="cmaxmean",
                           time_stepper="fourstep"), 8),
    ("rk4_tvdlf_cada", dict(flux_scheme="tvdlf", limiter="cada3", typedivbfix="linde", typeboundspeed="cmaxmean",
                            time_stepper="fourstep", time_integrator="rk4"), 8),
    ("2step_tvdlf_mm", dict(flux_scheme="tvdlf", limiter="minmod", typedivbfix="linde", typeboundspeed="cmaxmean",
                            time_stepper="twostep"), 8),
])
def test_blast_wave_3d_amr_golden_log_gpu(oracle_lib, name, kw, nw):
    kw = dict(kw, courantpar=0.9, fix_small_values=True, small_density=1.0e-14, small_pressure=1.0e-14)
    weight = np.zeros(nw)
    weight[0] = weight[4] = 0.5
    rows = _run_amr_golden("mhd", [2, 2, 2], _bw3d_prim(nw), weight, 0.2, kw, time_max=0.02, xmax=2.0, bc="cont",
                           nd=3, bn=8)
    gold = oracle_lib.read_log(os.path.join(GOLD, f"bw_3d_{name}.log"))
    assert rows.shape == gold.shape, (rows.shape, gold.shape)
    bad = np.abs(rows - gold) > 1e-8 + 1e-5 * np.abs(gold)
    assert oracle_lib.compare_logs(rows, gold, rtol=1e-5, atol=1e-8), (
        np.argwhere(bad)[:10].tolist(), rows[bad][:10].tolist(), gold[bad][:10].tolist())


# Riemann problem 2-D (tests/hd/Riemann_2D, reference, rm_2d.par): [0,1]^2,
# 24^2 level-1 cells in 12^2 blocks (block_nx 12), cont boundaries,
# refine_max_level 3 with the default estimator settings (w_refine_weight(1)
# = 1, refine_threshold 0.1), gamma 1.4, four quadrants about (0.5, 0.5);
# log every 1e-2 to t = 0.5.


def _rm2d_prim(X, Y, Z):
    out = np.zeros((4,) + X.shape)
    ul = (np.abs(X) < 0.5) & (Y > 0.5) & (Y < 1.0)
    ur = (np.abs(X) > 0.5) & (X < 1.0) & (Y > 0.5) & (Y < 1.0)
    ll = (np.abs(X) < 0.5) & (Y < 0.5)
    lr = (np.abs(X) > 0.5) & (X < 1.0) & (Y < 0.5)
    out[3] = np.where(ul | lr, 0.3, np.where(ur | ll, 1.5, 0.0))
    out[0] = np.where(ul | lr, 0.5323, np.where(ur | ll, 1.5, 0.0))
    out[1] = np.where(ul, 1.206, 0.0)
    out[2] = np.where(lr, 1.206, 0.0)
    return out


@pytest.mark.parametrize("name,kw", [
    ("3step_hll_cada", dict(flux_scheme="hll", limiter="cada3", typeboundspeed="cmaxmean")),
    ("4step_hll_mc", dict(flux_scheme="hll", limiter="woodward", typeboundspeed="cmaxmean", time_stepper="fourstep",
                          time_integrator="rk4")),
    ("4step_hllc_ko", dict(flux_scheme="hllc", limiter="koren", typeboundspeed="cmaxmean", time_stepper="fourstep")),
    ("rk4_tvdlf_cada", dict(flux_scheme="tvdlf", limiter="cada3", typeboundspeed="cmaxmean", time_stepper="fourstep",
                            time_integrator="rk4")),
    ("2step_tvdlf_mm", dict(flux_scheme="tvdlf", limiter="minmod", typeboundspeed="cmaxmean", time_stepper="twostep")),
    ("2step_tvdmu_al", dict(flux_scheme="tvdmu", limiter="albada", typeboundspeed="cmaxmean", time_stepper="twostep",
                            dimsplit=True)),
])
def test_riemann_2d_amr_golden_log_gpu(oracle_lib, name, kw):
    kw = dict(kw, courantpar=0.9, gamma=1.4, dtmin=1.0e-6)
    rows = _run_amr_golden("hd", [2, 2], _rm2d_prim, np.array([1.0, 0.0, 0.0, 0.0]), 0.1, kw, time_max=0.5,
                           dtsave=1.0e-2, bc="cont", bn=12)
    gold = oracle_lib.read_log(os.path.join(GOLD, f"rm_2d_{name}.log"))
    assert rows.shape == gold.shape, (rows.shape, gold.shape)
    bad = np.abs(rows - gold) > 1e-8 + 1e-5 * np.abs(gold)
    assert oracle_lib.compare_logs(rows, gold, rtol=1e-5, atol=1e-8), (
        np.argwhere(bad)[:10].tolist(), rows[bad][:10].tolist(), gold[bad][:10].tolist())


# Kelvin-Helmholtz 3-D MHD jet (tests/mhd/Kelvin_Helmholtz_3D, reference):
# [0,1] x [-1,1]^2, 20 x 40 x 40 level-1 cells in 10^3 blocks (block_nx 10),
# periodic in x, cont in y and z, refine_max_level 3 with w_refine_weight
# 0.4 (rho) and 0.2 (m1, m2, m3), refine_threshold 0.2, slowsteps 10; rho = 1,
# p = 1, B = (0.129, 0, 0), v_x = 0.645 tanh((r - 0.5)/0.05) with an m = 1
# perturbation of 0.01 in v_y, v_z; log every 1e-3 to t = 0.01.


def _kh3d_prim(nw):
    def f(X, Y, Z):
        out = np.zeros((nw,) + X.shape)
        r = np.sqrt(Y * Y + Z * Z)
        phi = np.arctan2(Z, Y)
        k1 = 2.0 * np.pi / 1.0
        rjet, width, qv, b0, dv = 0.5, 0.05, 0.645, 0.129, 0.01
        out[0] = 1.0
        out[4] = 1.0
        out[5] = b0
        out[1] = qv * np.tanh((r - rjet) / width)
        env = dv * np.exp(-((r - rjet) / (4.0 * width)) ** 2) * np.cos(phi) * np.sin(k1 * X)
        out[2] = env * np.cos(phi)
        out[3] = env * np.sin(phi)
        return out
    return f


@pytest.mark.parametrize("name,kw,nw", [
    ("3step_hll_cada", dict(flux_scheme="hll", limiter="cada3", typedivbfix="linde", typeboundspeed="cmaxmean"), 8),
    ("3step_hlld_cada", dict(flux_scheme="hlld", limiter="cada3", typedivbfix="glm"), 9),
    ("4step_hll_mc", dict(flux_scheme="hll", limiter="woodward", typedivbfix="linde", typeboundspeed="cmaxmean",
                          time_stepper="fourstep", time_integrator="rk4"), 8),
    ("4step_hllc_ko", dict(flux_scheme="hllc", limiter="koren", typedivbfix="linde", typeboundspeed="cmaxmean",
                           time_stepper="fourstep"), 8),
    ("rk4_tvdlf_cada", dict(flux_scheme="tvdlf", limiter="cada3", typedivbfix="linde", typeboundspeed="cmaxmean",
                            time_stepper="fourstep", time_integrator="rk4"), 8),
    ("2step_tvdlf_mm", dict(flux_scheme="tvdlf", limiter="minmod", typedivbfix="linde", typeboundspeed="cmaxmean",
                            time_stepper="twostep"), 8),
    ("2step_tvdmu_al", dict(flux_scheme="tvdmu", limiter="albada", typedivbfix="linde", typeboundspeed="cmaxmean",
                            time_stepper="twostep", dimsplit=True), 8),
])
def test_kelvin_helmholtz_3d_amr_golden_log_gpu(oracle_lib, name, kw, nw):
    kw = dict(kw, courantpar=0.9, slowsteps=10)
    weight = np.zeros(nw)
    weight[0], weight[1], weight[2], weight[3] = 0.4, 0.2, 0.2, 0.2
    rows = _run_amr_golden("mhd", [2, 4, 4], _kh3d_prim(nw), weight, 0.2, kw, time_max=1.0e-2, nd=3, bn=10,
                           xmin=[0.0, -1.0, -1.0], xmax=[1.0, 1.0, 1.0],
                           bc=["periodic", "periodic", "cont", "cont", "cont", "cont"])
    gold = oracle_lib.read_log(os.path.join(GOLD, f"kh_3D_{name}.log"))
    assert rows.shape == gold.shape, (rows.shape, gold.shape)
    bad = np.abs(rows - gold) > 1e-8 + 1e-5 * np.abs(gold)
    assert oracle_lib.compare_logs(rows, gold, rtol=1e-5, atol=1e-8), (
        np.argwhere(bad)[:10].tolist(), rows[bad][:10].tolist(), gold[bad][:10].tolist())
