"""Batched-ensemble host logic and its 1-D known answer, without a GPU.

* The exact Riemann solver (test infrastructure) reproduces the star states
  published for Toro's standard tests (Toro 2009, table 4.2).
* The oracle's 1-D runs converge to the exact solution of the Sod problem for
  the ensemble's schemes — the reference's analytic_test_1d check (RMSE of
  density), here on [0, 1] with the interface at 0.5 and t = 0.2.
* Invalid ensembles are refused by the C ABI before any CUDA call.
* The seeded ensemble inputs follow the stated distributions.
* Instance 20 of the seeded 512-instance ensemble is a strongly diverging
  Riemann problem whose rarefaction head the Einfeldt estimate (Roe averages,
  Toro eq. 10.52, src/hd/mod_hd_phys.t:911-932) does not bound: the oracle's
  state turns non-finite in the first step; with cmaxleftright it runs.
"""
import ctypes

import numpy as np
import pytest

from tests import _riemann as R


@pytest.fixture(scope="module")
def lib():
    from amrvac_b200 import build, _lib
    build.build()
    return _lib.load()


@pytest.mark.parametrize("left,right,pstar,ustar", [
    ((1.0, 0.0, 1.0), (0.125, 0.0, 0.1), 0.30313, 0.92745),        # Sod
    ((1.0, -2.0, 0.4), (1.0, 2.0, 0.4), 0.00189, 0.0),             # two rarefactions
    ((1.0, 0.0, 1000.0), (1.0, 0.0, 0.01), 460.894, 19.5975),      # strong shock
    ((5.99924, 19.5975, 460.894), (5.99242, -6.19633, 46.0950), 1691.64, 8.68975),  # colliding shocks
])
def test_exact_riemann_star_states(left, right, pstar, ustar):
    p, u = R.star_state(*left, *right, 1.4)
    assert abs(p - pstar) <= 1e-5 * max(1.0, pstar) + 5e-6
    assert abs(u - ustar) <= 1e-5 * max(1.0, abs(ustar)) + 5e-6


def _oracle_sod(oracle_lib, n, fs, lim, tmax=0.2, courantpar=0.8):
    O = oracle_lib
    c = O.make_cfg(physics="hd", ndim=1, gamma=1.4, flux_scheme=fs, limiter=lim, courantpar=courantpar)
    spec = dict(ndim=1, shape=(n,), rl=1.0, ul=0.0, pl=1.0, rr=0.125, ur=0.0, pr=0.1, x0=0.5, theta=0.0,
                flux_scheme=fs, limiter=lim, time_max=tmax)
    blocks = R.initial_blocks(spec, 1.4)
    g = O.Grid(c, [n], [0.0], [1.0], ["cont", "cont"])
    for ib in range(g.nblocks):
        g.set_block(ib, blocks[ib])
    g.getbc()
    t = 0.0
    while tmax - t > 1e-10:
        dt, _ = g.getdt()
        dt = min(dt, tmax - t)
        g.advance(dt)
        t += dt
    rho = np.concatenate([g.get_block(ib)[0, 0, 0, 2:18] for ib in range(g.nblocks)])
    x = (np.arange(n) + 0.5) / n
    ex = R.exact_riemann(1.0, 0.0, 1.0, 0.125, 0.0, 0.1, 1.4, (x - 0.5) / tmax)
    return float(np.sqrt(np.mean((rho - ex[0]) ** 2)))


@pytest.mark.parametrize("fs,lim", [("hll", "minmod"), ("hll", "vanleer"), ("hllc", "minmod"),
                                    ("hllc", "vanleer")])
def test_oracle_1d_sod_converges_to_exact(oracle_lib, fs, lim):
    errs = [_oracle_sod(oracle_lib, n, fs, lim) for n in (128, 256, 512)]
    assert errs[1] < 0.02
    assert errs[0] > errs[1] > errs[2]


def test_ensemble_refused_before_cuda(lib):
    from amrvac_b200 import _lib, make_cfg
    good = (_lib.AmrvacEnsInstance * 1)()
    good[0].ndim = 1
    good[0].domain_nx[0] = 64
    good[0].xprobmax[0] = 1.0
    good[0].flux_scheme = _lib.FS["hll"]
    good[0].limiter = _lib.LIMITER["minmod"]
    good[0].time_max = 0.1
    h = ctypes.c_void_p()
    # MHD ensembles are not offered
    rc = lib.amrvac_ens_create(ctypes.byref(make_cfg(physics="mhd", ndim=2)), 1, good, ctypes.byref(h))
    assert rc == _lib.E_UNSUPPORTED
    cfg = make_cfg(physics="hd", ndim=2, gamma=1.4, typeboundary=["cont"] * 4)
    for field, value, code in [("ndim", 3, _lib.E_UNSUPPORTED), ("flux_scheme", _lib.FS["hlld"], _lib.E_UNSUPPORTED),
                               ("limiter", 0, _lib.E_UNSUPPORTED)]:
        bad = (_lib.AmrvacEnsInstance * 1)()
        ctypes.memmove(ctypes.byref(bad), ctypes.byref(good), ctypes.sizeof(good))
        setattr(bad[0], field, value)
        assert lib.amrvac_ens_create(ctypes.byref(cfg), 1, bad, ctypes.byref(h)) == code
    bad = (_lib.AmrvacEnsInstance * 1)()
    ctypes.memmove(ctypes.byref(bad), ctypes.byref(good), ctypes.sizeof(good))
    bad[0].domain_nx[0] = 40
    assert lib.amrvac_ens_create(ctypes.byref(cfg), 1, bad, ctypes.byref(h)) == _lib.E_ARG
    sym = make_cfg(physics="hd", ndim=2, gamma=1.4, typeboundary=["symm"] * 4)
    assert lib.amrvac_ens_create(ctypes.byref(sym), 1, good, ctypes.byref(h)) == _lib.E_UNSUPPORTED
    assert lib.amrvac_ens_create(ctypes.byref(cfg), 0, good, ctypes.byref(h)) == _lib.E_ARG


def test_ensemble_specs_follow_the_distributions():
    specs = R.ensemble_specs(512)
    one = [s for s in specs if s["ndim"] == 1]
    two = [s for s in specs if s["ndim"] == 2]
    assert len(one) == 256 and len(two) == 256
    assert all(s["shape"][0] % 16 == 0 and 64 <= s["shape"][0] <= 4096 for s in one)
    assert all(s["shape"][0] == s["shape"][1] and 32 <= s["shape"][0] <= 512 for s in two)
    for s in specs:
        for k in ("rl", "pl", "rr", "pr"):
            assert 0.1 <= s[k] <= 10.0
        assert -2.0 <= s["ul"] <= 2.0 and 0.3 <= s["x0"] <= 0.7
        cl, cr = np.sqrt(1.4 * s["pl"] / s["rl"]), np.sqrt(1.4 * s["pr"] / s["rr"])
        assert 5.0 * (cl + cr) > 1.5 * (s["ur"] - s["ul"])
    assert {(s["flux_scheme"], s["limiter"]) for s in specs} == {("hll", "minmod"), ("hll", "vanleer"),
                                                                  ("hllc", "minmod"), ("hllc", "vanleer")}
    assert R.ensemble_specs(512) == specs  # seeded


def _oracle_steps(oracle_lib, spec, boundspeed, nsteps):
    O = oracle_lib
    nd = spec["ndim"]
    c = O.make_cfg(physics="hd", ndim=nd, gamma=1.4, flux_scheme=spec["flux_scheme"], limiter=spec["limiter"],
                   courantpar=0.8, typeboundspeed=boundspeed)
    g = O.Grid(c, list(spec["shape"]), [0.0] * nd, [1.0] * nd, ["cont"] * (2 * nd))
    b = R.initial_blocks(spec, 1.4)
    for ib in range(g.nblocks):
        g.set_block(ib, b[ib])
    g.getbc()
    pmin = []
    for _ in range(nsteps):
        dt, _ = g.getdt()
        g.advance(dt)
        w = np.concatenate([g.get_block(ib)[:, 0, 0, 2:18] for ib in range(g.nblocks)], axis=1)
        p = 0.4 * (w[2] - 0.5 * w[1] ** 2 / w[0])
        pmin.append(float(np.min(p)) if np.all(np.isfinite(p)) else float("nan"))
    return pmin


def test_einfeldt_crash_instance_in_the_oracle(oracle_lib):
    spec = R.ensemble_specs(512)[20]
    assert spec["ndim"] == 1
    pe = _oracle_steps(oracle_lib, spec, "Einfeldt", 1)
    assert not (pe[0] >= 0.0)  # negative pressure or NaN
    pl = _oracle_steps(oracle_lib, spec, "cmaxleftright", 20)
    assert all(p > 0.0 for p in pl)
