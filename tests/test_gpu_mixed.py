"""Mixed form: FP32 face arithmetic, FP64 state/accumulation/pressure recovery.

The north star bounds the L1 density error of the mixed form against the FP64
result at 1e-6 (relative); the per-variable L1 errors are reported by
bench.py for the benchmark workload.
"""
import numpy as np
import pytest

from tests import _problems as P

pytestmark = pytest.mark.gpu


def _cuda():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")


def _run(kw, blocks, geo, nsteps, precision):
    from amrvac_b200 import Context, make_cfg
    ctx = Context(make_cfg(precision=precision, **kw))
    ctx.set_uniform_grid(geo["domain_nx"], geo["xprobmin"], geo["xprobmax"])
    ctx.upload(blocks)
    ctx.set_time(0.0, 1.0e99, 0.0)
    ctx.run(nsteps)
    assert ctx.status() == 0
    out = P.interior(ctx.download(), kw["ndim"])
    ctx.close()
    return out


def _l1(a, b):
    return np.abs(a - b).sum() / np.abs(b).sum()


def test_mixed_orszag_tang_l1():
    _cuda()
    prim, geo = P.orszag_tang_3d(n=32)
    cons = P.prim_to_cons(prim, "mhd", 3, 5.0 / 3.0)
    blocks = P.to_blocks(cons, 3)
    kw = dict(physics="mhd", ndim=3, ndir=3, flux_scheme="hlld", limiter="cada3", typedivbfix="glm")
    ref = _run(kw, blocks, geo, 20, "fp64")
    got = _run(kw, blocks, geo, 20, "mixed")
    assert _l1(got[:, 0], ref[:, 0]) <= 1e-6
    for v in range(ref.shape[1] - 1):  # psi starts at zero; its error is relative to a tiny field
        assert _l1(got[:, v], ref[:, v]) <= 1e-4


def test_mixed_kelvin_helmholtz_l1():
    _cuda()
    prim, geo = P.kh_2d(n=64)
    cons = P.prim_to_cons(prim, "hd", 2, 1.4)
    blocks = P.to_blocks(cons, 2)
    kw = dict(physics="hd", ndim=2, gamma=1.4, flux_scheme="hllc", limiter="vanleer")
    ref = _run(kw, blocks, geo, 20, "fp64")
    got = _run(kw, blocks, geo, 20, "mixed")
    assert _l1(got[:, 0], ref[:, 0]) <= 1e-6


def test_mixed_conserves_mass():
    """FP64 accumulation of FP32 fluxes keeps the discrete conservation."""
    _cuda()
    prim, geo = P.kh_2d(n=64)
    cons = P.prim_to_cons(prim, "hd", 2, 1.4)
    blocks = P.to_blocks(cons, 2)
    kw = dict(physics="hd", ndim=2, gamma=1.4, flux_scheme="hllc", limiter="vanleer")
    got = _run(kw, blocks, geo, 10, "mixed")
    m0 = P.interior(blocks, 2)[:, 0].sum()
    assert abs(got[:, 0].sum() - m0) <= 1e-13 * abs(m0)
