"""Discrete adjoint on the GPU.

Bars: the gradient of the blast-wave loss with respect to the initial density
field and gamma agrees with the oracle's forward-mode (dual-number) reference
gradient to 1e-6 relative; directional derivatives agree with central finite
differences of the GPU forward runs (frozen time steps); one adjoint step is
the transpose of one forward step (dot-product test); the checkpoint interval
does not change the gradient (bit-exact recomputation).
"""
import numpy as np
import pytest

from tests import _blast as B

pytestmark = pytest.mark.gpu


def _cuda():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")


def _setup(n, lim):
    import torch
    prim = B.blast_prim(n)
    rho0 = torch.tensor(prim[0, 0], dtype=torch.float64, device="cuda")
    p0 = torch.tensor(prim[3, 0], dtype=torch.float64, device="cuda")
    mask = torch.tensor(B.loss_mask(n), dtype=torch.float64, device="cuda")
    return prim, rho0, p0, mask


def _loss_fn(n, lim, dts, p0, mask, k=20, fs="hll"):
    import torch
    from amrvac_b200.adjoint import blocks_to_domain, domain_to_blocks, solve

    def f(rho0, gamma):
        z = torch.zeros_like(rho0)
        U0 = domain_to_blocks(torch.stack([rho0, z, z, p0 / (gamma - 1.0)]))
        UN = solve(U0, gamma, dts, (n, n), (0.0, 0.0), (1.0, 1.0), checkpoint_every=k, limiter=lim,
                   flux_scheme=fs, typeboundary=["cont"] * 4)
        rho = blocks_to_domain(UN, n, n)[0]
        return (mask * rho * rho).sum()
    return f


def _dts(n, rho0, p0, nsteps, lim, fs="hll"):
    import torch
    from amrvac_b200.adjoint import FrozenDtSolver, domain_to_blocks
    s = FrozenDtSolver((n, n), (0.0, 0.0), (1.0, 1.0), B.GAMMA, limiter=lim, flux_scheme=fs,
                       typeboundary=["cont"] * 4)
    z = torch.zeros_like(rho0)
    U0 = domain_to_blocks(torch.stack([rho0, z, z, p0 / (B.GAMMA - 1.0)]))
    dts = s.cfl_dts(U0, nsteps)
    s.close()
    return dts


SCHEMES = [("hll", "minmod"), ("hll", "vanleer"), ("hllc", "minmod"), ("hllc", "vanleer")]


@pytest.mark.parametrize("fs,lim", SCHEMES)
def test_gradient_matches_dual_number_reference(oracle_lib, fs, lim):
    _cuda()
    import torch
    O = oracle_lib
    n, nsteps = 32, 20
    prim, rho0, p0, mask = _setup(n, lim)
    dts = _dts(n, rho0, p0, nsteps, lim, fs)
    f = _loss_fn(n, lim, dts, p0, mask, fs=fs)
    r = rho0.clone().requires_grad_(True)
    g = torch.tensor(B.GAMMA, dtype=torch.float64, device="cuda", requires_grad=True)
    L = f(r, g)
    L.backward()
    grad_rho = r.grad.cpu().numpy()
    grad_gamma = float(g.grad)
    c = O.make_cfg(physics="hd", ndim=2, gamma=B.GAMMA, flux_scheme=fs, limiter=lim, courantpar=0.8)
    w0 = B.to_cons_blocks(prim)
    mb = B.mask_blocks(n)
    drho = np.random.default_rng(5).standard_normal((n, n))
    Lref, dref, st = O.dual_run(c, [n, n], [0.0, 0.0], [1.0, 1.0], ["cont"] * 4, w0, B.cons_direction(prim, drho, 0.0),
                                0.0, dts, mb)
    assert st == 0
    assert abs(float(L.detach()) - Lref) <= 1e-12 * abs(Lref)
    got = float((grad_rho * drho).sum())
    assert abs(got - dref) <= 1e-6 * abs(dref), (got, dref)
    _, dgref, _ = O.dual_run(c, [n, n], [0.0, 0.0], [1.0, 1.0], ["cont"] * 4, w0,
                             B.cons_direction(prim, np.zeros((n, n)), 1.0), 1.0, dts, mb)
    assert abs(grad_gamma - dgref) <= 1e-6 * abs(dgref), (grad_gamma, dgref)


def test_gradient_matches_central_differences():
    """16 seeded density directions and gamma, FD of the GPU forward at frozen dt."""
    _cuda()
    import torch
    n, nsteps, lim = 64, 40, "minmod"
    prim, rho0, p0, mask = _setup(n, lim)
    dts = _dts(n, rho0, p0, nsteps, lim)
    f = _loss_fn(n, lim, dts, p0, mask)
    r = rho0.clone().requires_grad_(True)
    g = torch.tensor(B.GAMMA, dtype=torch.float64, device="cuda", requires_grad=True)
    f(r, g).backward()
    rng = np.random.default_rng(17)
    # a step of 1e-8 stays below the limiter kinks that a random density
    # direction reaches at this size (1e-7 crosses some: errors ~3e-5) and
    # above roundoff of the loss (~200): measured errors <= 2e-6
    eps = 1e-8
    errs = []
    with torch.no_grad():
        for _ in range(16):
            d = torch.tensor(rng.standard_normal((n, n)), dtype=torch.float64, device="cuda")
            fd = (float(f(rho0 + eps * d, torch.tensor(B.GAMMA, dtype=torch.float64, device="cuda"))) -
                  float(f(rho0 - eps * d, torch.tensor(B.GAMMA, dtype=torch.float64, device="cuda")))) / (2 * eps)
            ad = float((r.grad * d).sum())
            errs.append(abs(fd - ad) / abs(ad))
        epg = 1e-7
        fdg = (float(f(rho0, torch.tensor(B.GAMMA + epg, dtype=torch.float64, device="cuda"))) -
               float(f(rho0, torch.tensor(B.GAMMA - epg, dtype=torch.float64, device="cuda")))) / (2 * epg)
    assert np.median(errs) <= 2e-6 and max(errs) <= 2e-5, errs
    assert abs(fdg - float(g.grad)) <= 2e-5 * abs(float(g.grad)), (fdg, float(g.grad))


@pytest.mark.parametrize("fs,lim", SCHEMES)
def test_adjoint_step_is_the_transpose_of_the_step(fs, lim):
    """<lam, J dU> == <J^T lam, dU> for one SSP-RK3 step (J by central
    differences), on a smooth state with flow everywhere: no limiter slope
    sits exactly at a kink (the blast's v = 0, uniform-pressure regions do)."""
    _cuda()
    import torch
    from amrvac_b200.adjoint import FrozenDtSolver, domain_to_blocks
    from tests import _problems as P
    n = 32
    cons = P.prim_to_cons(P.random_smooth("hd", 2, 2, n, seed=3), "hd", 2, B.GAMMA)[:, 0]
    U0 = domain_to_blocks(torch.tensor(cons, dtype=torch.float64, device="cuda")).contiguous()
    s = FrozenDtSolver((n, n), (0.0, 0.0), (1.0, 1.0), B.GAMMA, limiter=lim, flux_scheme=fs,
                       typeboundary=["cont"] * 4)
    dt = float(s.cfl_dts(U0, 1)[0])
    rng = np.random.default_rng(23)
    lam = torch.tensor(rng.standard_normal(s.shape), dtype=torch.float64, device="cuda")
    dU = torch.tensor(rng.standard_normal(s.shape), dtype=torch.float64, device="cuda")
    eps = 1e-7
    up, _ = s.forward(U0 + eps * dU, [dt])
    um, _ = s.forward(U0 - eps * dU, [dt])
    jdu = (up - um) / (2 * eps)
    _, ck = s.forward(U0, [dt])
    lt, _ = s.backward(lam, [dt], ck)
    a = float((lam * jdu).sum())
    b = float((lt * dU).sum())
    s.close()
    assert abs(a - b) <= 1e-7 * abs(b), (a, b)


def test_checkpoint_interval_does_not_change_the_gradient():
    _cuda()
    import torch
    n, nsteps, lim = 32, 12, "vanleer"
    prim, rho0, p0, mask = _setup(n, lim)
    dts = _dts(n, rho0, p0, nsteps, lim)
    grads = []
    for k in (1, 5, 20):
        r = rho0.clone().requires_grad_(True)
        g = torch.tensor(B.GAMMA, dtype=torch.float64, device="cuda", requires_grad=True)
        _loss_fn(n, lim, dts, p0, mask, k=k)(r, g).backward()
        grads.append((r.grad.clone(), float(g.grad)))
    for gr, gg in grads[1:]:
        assert torch.equal(gr, grads[0][0]) and gg == grads[0][1]


def test_recomputing_and_supplied_stage_states_agree():
    """amrvac_gpu_adjoint_step (recomputes the stages) and
    amrvac_gpu_adjoint_step_states (caller's stage inputs): bit-identical."""
    _cuda()
    import ctypes
    import torch
    from amrvac_b200 import _lib
    from amrvac_b200.adjoint import FrozenDtSolver, domain_to_blocks
    from tests import _problems as P
    n = 32
    cons = P.prim_to_cons(P.random_smooth("hd", 2, 2, n, seed=4), "hd", 2, B.GAMMA)[:, 0]
    U0 = domain_to_blocks(torch.tensor(cons, dtype=torch.float64, device="cuda")).contiguous()
    s = FrozenDtSolver((n, n), (0.0, 0.0), (1.0, 1.0), B.GAMMA, limiter="vanleer", typeboundary=["cont"] * 4)
    dt = float(s.cfl_dts(U0, 1)[0])
    lam0 = torch.tensor(np.random.default_rng(2).standard_normal(s.shape), dtype=torch.float64, device="cuda")
    p = lambda t: ctypes.c_void_p(t.data_ptr())  # noqa: E731
    la, ga = lam0.clone(), torch.zeros(s.ctx.nblocks, dtype=torch.float64, device="cuda")
    s._load(U0)
    _lib.check(s.L.amrvac_gpu_adjoint_step(s.ctx.h, p(la), dt, p(ga)), "adjoint_step")
    s.ctx.synchronize()
    st = [torch.empty(s.shape, dtype=torch.float64, device="cuda") for _ in range(3)]
    s._load(U0)
    s._store(st[0], 0)
    _lib.check(s.L.amrvac_gpu_step_dt(s.ctx.h, dt), "step_dt")
    s._store(st[1], 1)
    s._store(st[2], 2)
    lb, gb = lam0.clone(), torch.zeros(s.ctx.nblocks, dtype=torch.float64, device="cuda")
    _lib.check(s.L.amrvac_gpu_adjoint_step_states(s.ctx.h, p(st[0]), p(st[1]), p(st[2]), p(lb), dt, p(gb)),
               "adjoint_step_states")
    s.ctx.synchronize()
    s.close()
    assert torch.equal(la, lb) and torch.equal(ga, gb)


@pytest.mark.parametrize("stepper", [dict(), dict(time_stepper="twostep", time_integrator="ssprk2")])
def test_step_with_caller_stage_buffers_matches_the_registers(stepper):
    """amrvac_gpu_step_dt_states writes the same stage inputs and U^{n+1} as
    amrvac_gpu_step_dt leaves in the registers (bit-identical), also in place
    (unew = u0); without unew it leaves u0 untouched; aliased stage buffers
    are refused."""
    _cuda()
    import ctypes
    import torch
    from amrvac_b200 import _lib
    from amrvac_b200.adjoint import FrozenDtSolver, domain_to_blocks
    from tests import _problems as P
    n = 32
    cons = P.prim_to_cons(P.random_smooth("hd", 2, 2, n, seed=6), "hd", 2, B.GAMMA)[:, 0]
    U0 = domain_to_blocks(torch.tensor(cons, dtype=torch.float64, device="cuda")).contiguous()
    s = FrozenDtSolver((n, n), (0.0, 0.0), (1.0, 1.0), B.GAMMA, limiter="vanleer", typeboundary=["cont"] * 4,
                       **stepper)
    nst = s._nstages()
    dt = float(s.cfl_dts(U0, 1)[0])
    p = lambda t: ctypes.c_void_p(t.data_ptr())  # noqa: E731
    ref = [torch.empty(s.shape, dtype=torch.float64, device="cuda") for _ in range(3)]
    s._load(U0)
    _lib.check(s.L.amrvac_gpu_step_dt(s.ctx.h, dt), "step_dt")
    for r in range(3):
        s._store(ref[r], r)
    got = [U0.clone()] + [torch.full(s.shape, np.nan, dtype=torch.float64, device="cuda") for _ in range(3)]
    torch.cuda.synchronize()
    u2 = p(got[2]) if nst == 3 else None
    _lib.check(s.L.amrvac_gpu_step_dt_states(s.ctx.h, dt, p(got[0]), p(got[1]), u2, p(got[3])), "step_dt_states")
    s.ctx.synchronize()
    assert torch.equal(got[0], U0) and torch.equal(got[1], ref[1]) and torch.equal(got[3], ref[0])
    if nst == 3:
        assert torch.equal(got[2], ref[2])
    # in place: U^{n+1} over u0; no last stage: u0 untouched
    _lib.check(s.L.amrvac_gpu_step_dt_states(s.ctx.h, dt, p(got[0]), p(got[1]), u2, p(got[0])), "step_dt_states")
    s.ctx.synchronize()
    assert torch.equal(got[0], ref[0])
    got[0].copy_(U0)
    torch.cuda.synchronize()
    _lib.check(s.L.amrvac_gpu_step_dt_states(s.ctx.h, dt, p(got[0]), p(got[1]), u2, None), "step_dt_states")
    s.ctx.synchronize()
    assert torch.equal(got[0], U0) and torch.equal(got[1], ref[1])
    # a stage that would read and write one buffer
    last = got[2] if nst == 3 else got[1]
    assert s.L.amrvac_gpu_step_dt_states(s.ctx.h, dt, p(got[0]), p(got[0]), u2, None) == _lib.E_ARG
    assert s.L.amrvac_gpu_step_dt_states(s.ctx.h, dt, p(got[0]), p(got[1]), u2, p(last)) == _lib.E_ARG
    s.close()
