"""FP64 parity on the benchmark workloads themselves, at their full size.

The benchmark's own initial states (``bench.py`` builds them with the same
functions): 3-D ideal MHD Orszag-Tang at 128^3 (512 blocks of 16^3, HLLD +
cada3 + GLM, CFL 0.8) and 2-D Kelvin-Helmholtz at 256^2 (256 blocks of 16^2,
HLLC + vanleer).  For each: the CFL reduction (dt, cmax_global), one stage
(advect1, src/mod_advance.t:611-666 -> finite_volume) and one full SSP-RK3
step on the device against the oracle, cell by cell with the per-cell
measure of tests/_parity.py (relative error for cells >= 1e-3 of the
variable's maximum, |diff| against that floor below it).

The bar is 1e-12 for every variable, except where the reference formula
itself is worse conditioned on this data: each test also runs the oracle on
the same input with a relative perturbation of one unit in the last place
per value, and a variable's bar is the larger of 1e-12 and that self-noise.
Only the noise-only momentum components need it (z-momentum of Orszag-Tang,
which holds the seeded 1e-3 velocity noise, and y-momentum of
Kelvin-Helmholtz): there one ulp of input noise moves the oracle's own
result by up to 6e-8 (OT) and 1e-11 (KH) relative, far more than the device
differs from it.  The momentum vector is also checked per cell against its
magnitude at 1e-12 with no such allowance.
"""
import concurrent.futures as cf
import os

import numpy as np
import pytest

from tests import _problems as P
from tests._parity import one_ulp_noise, percell_parts

pytestmark = pytest.mark.gpu

RTOL = 1e-12


def _cuda():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")


def _workload(name):
    if name == "ot128":
        prim, geo = P.orszag_tang_3d(n=128)
        cons = P.prim_to_cons(prim, "mhd", 3, 5.0 / 3.0)
        kw = dict(physics="mhd", ndim=3, ndir=3, flux_scheme="hlld", limiter="cada3", courantpar=0.8)
        return P.to_blocks(cons, 3), geo, kw, dict(typedivbfix="glm"), dict(divb="glm")
    prim, geo = P.kh_2d(n=256)
    cons = P.prim_to_cons(prim, "hd", 2, 1.4)
    kw = dict(physics="hd", ndim=2, gamma=1.4, flux_scheme="hllc", limiter="vanleer", courantpar=0.8)
    return P.to_blocks(cons, 2), geo, kw, {}, {}


def _setup(O, name):
    from amrvac_b200 import Context, make_cfg
    blocks, geo, kw, gk, ok = _workload(name)
    nd = kw["ndim"]
    ocfg = O.make_cfg(**kw, **ok)
    og = O.Grid(ocfg, geo["domain_nx"], geo["xprobmin"], geo["xprobmax"], ["periodic"] * (2 * nd))
    for ib in range(og.nblocks):
        og.set_block(ib, blocks[ib])
    og.getbc()
    ctx = Context(make_cfg(**kw, **gk))
    ctx.set_uniform_grid(geo["domain_nx"], geo["xprobmin"], geo["xprobmax"])
    assert ctx.nblocks == og.nblocks
    ctx.upload(blocks)
    return ocfg, og, ctx, nd


def _perturbed(blocks, seed=1):
    """Every value times (1 +/- 2^-52): one ulp of input noise."""
    return one_ulp_noise(blocks, seed)


def _check(got, ref, noisy, nd, what):
    """Per variable: error <= max(RTOL, the oracle's own 1-ulp self-noise);
    momentum vector per cell <= RTOL of its magnitude."""
    report = []
    for v in range(got.shape[1]):
        if not np.any(ref[:, v]):  # zero everywhere (psi after one stage): absolute, on the scale of all variables
            assert np.abs(got[:, v]).max() <= RTOL * 1e-3 * np.abs(ref).max(), f"{what} var {v} not zero"
            continue
        rel, small = percell_parts(got[:, v:v + 1], ref[:, v:v + 1])
        nrel, nsmall = percell_parts(noisy[:, v:v + 1], ref[:, v:v + 1])
        bar = max(RTOL, nrel, nsmall) if np.isfinite(max(nrel, nsmall)) else RTOL
        report.append((v, rel, small, bar))
        assert rel <= bar and small <= bar, f"{what} var {v}: relative {rel:.3e}, small-cell {small:.3e} (bar {bar:.3e})"
    ndir = 3 if got.shape[1] >= 8 else nd
    m, mr = got[:, 1:1 + ndir], ref[:, 1:1 + ndir]
    mag = np.sqrt((mr * mr).sum(axis=1))
    big = mag >= 1e-3 * mag.max()
    dm = np.sqrt(((m - mr) ** 2).sum(axis=1))
    vec = float((dm[big] / mag[big]).max())
    assert vec <= RTOL, f"{what}: momentum vector {vec:.3e}"
    return report


def _stage_ref(O, ocfg, src, dt, dx, cg):
    def one(ib):  # the oracle releases the GIL inside its C++ code
        wn = src[ib].copy()
        O.finite_volume(ocfg, src[ib], wn, dt, dx, cg)
        return wn
    with cf.ThreadPoolExecutor(max_workers=os.cpu_count() or 1) as ex:
        return np.array(list(ex.map(one, range(len(src)))))


def _oracle_grid(O, ocfg, name, blocks):
    _, geo, kw, _, _ = _workload(name)
    nd = kw["ndim"]
    og = O.Grid(ocfg, geo["domain_nx"], geo["xprobmin"], geo["xprobmax"], ["periodic"] * (2 * nd))
    for ib in range(og.nblocks):
        og.set_block(ib, blocks[ib])
    og.getbc()
    return og


@pytest.mark.parametrize("name", ["ot128", "kh256"])
def test_config_getdt_and_stage(oracle_lib, name):
    """getdt, then one stage ps -> ps1 with the step's dt, on the full grid."""
    _cuda()
    O = oracle_lib
    ocfg, og, ctx, nd = _setup(O, name)
    dt_ref, cg_ref = og.getdt()
    dt, cg, st = ctx.getdt()
    assert st == 0
    assert abs(dt - dt_ref) <= 1e-13 * dt_ref and abs(cg - cg_ref) <= 1e-13 * max(cg_ref, 1e-300)
    ctx.set_cmax_global(cg_ref)
    assert ctx.advect1("ps", "ps1", 1.0, dt_ref) == 0
    got = P.interior(ctx.download("ps1"), nd)
    dx = og.dx()
    ref = P.interior(_stage_ref(O, ocfg, [og.get_block(ib) for ib in range(og.nblocks)], dt_ref, dx, cg_ref), nd)
    gp = _oracle_grid(O, ocfg, name, _perturbed(_workload(name)[0]))
    noisy = P.interior(_stage_ref(O, ocfg, [gp.get_block(ib) for ib in range(gp.nblocks)], dt_ref, dx, cg_ref), nd)
    _check(got, ref, noisy, nd, f"{name} stage")
    assert ctx.status() == 0
    ctx.close()


@pytest.mark.parametrize("name", ["ot128", "kh256"])
def test_config_full_step(oracle_lib, name):
    """setdt + the three SSP-RK3 stages + time update on the device against
    the oracle's advance, on the full grid."""
    _cuda()
    O = oracle_lib
    ocfg, og, ctx, nd = _setup(O, name)
    dt_ref, cg_ref = og.getdt()
    ctx.set_time(0.0, 1.0e99, 0.0)
    ctx.step()
    dt, cg, t = ctx.get_time()
    assert abs(dt - dt_ref) <= 1e-13 * dt_ref and abs(cg - cg_ref) <= 1e-13 * max(cg_ref, 1e-300)
    nth = os.cpu_count() or 1
    og.advance(dt_ref, cg_ref, nth)
    got = P.interior(ctx.download("ps"), nd)
    ref = P.interior(np.array([og.get_block(ib) for ib in range(og.nblocks)]), nd)
    gp = _oracle_grid(O, ocfg, name, _perturbed(_workload(name)[0]))
    gp.advance(dt_ref, cg_ref, nth)
    noisy = P.interior(np.array([gp.get_block(ib) for ib in range(gp.nblocks)]), nd)
    _check(got, ref, noisy, nd, f"{name} step")
    assert ctx.status() == 0
    ctx.close()
