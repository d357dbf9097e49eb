"""The FP64 reciprocal and quotient of the stage kernels against IEEE division.

Every stage kernel divides with ``div_`` / ``rcp_`` (csrc/physics.cuh):
Newton-Raphson from the hardware's approximate reciprocal, with an integer
guard that sends zero, subnormal, huge, infinite and NaN denominators (and
quotients that overflow) to the correctly rounded IEEE division.  The
reference divides with IEEE division everywhere, so the bar is one unit in
the last place over the whole double range of |y| (1e-300 .. 1e300), and
IEEE's own result bit for bit at the special values.
"""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

ULP = 2.0 ** -52


def _cuda():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")


def _div_points(x, y):
    from amrvac_b200 import _lib
    L = _lib.load()
    x = np.ascontiguousarray(x, np.float64)
    y = np.ascontiguousarray(y, np.float64)
    q, r, s = (np.empty_like(x) for _ in range(3))
    dp = lambda a: a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))  # noqa: E731
    _lib.check(L.amrvac_gpu_div_points(x.size, dp(x), dp(y), dp(q), dp(r), dp(s)), "div_points")
    return q, r, s


def _relerr(a, b):
    return np.abs(a - b) / np.abs(b)


def test_div_rcp_within_one_ulp_over_the_double_range():
    _cuda()
    rng = np.random.default_rng(20261203)
    n = 1 << 20
    y = 10.0 ** rng.uniform(-300.0, 300.0, n) * rng.choice([-1.0, 1.0], n)
    x = 10.0 ** rng.uniform(-5.0, 5.0, n) * rng.choice([-1.0, 1.0], n)
    # the denominators the stage kernels meet: densities, speeds, slopes
    y[: n // 4] = rng.uniform(1e-12, 1e3, n // 4)
    q, r, s = _div_points(x, y)
    eq, er, es = _relerr(q, x / y), _relerr(r, 1.0 / y), _relerr(s, 1.0 / y)
    assert eq.max() <= ULP, f"quotient: {eq.max() / ULP:.2f} ulp"
    assert er.max() <= ULP, f"reciprocal: {er.max() / ULP:.2f} ulp"
    # the Newton steps need a seed of about 20 correct bits
    assert es.max() <= 2.0 ** -19, f"seed: 2^{np.log2(es.max()):.1f}"
    # most quotients are the correctly rounded ones
    assert np.mean(q == x / y) >= 0.99


def test_div_rcp_special_values_are_ieee():
    _cuda()
    tiny = np.finfo(np.float64).tiny
    ys = np.array([0.0, -0.0, np.inf, -np.inf, np.nan, 1e-310, -1e-310, tiny, 1e308, -1e308, 2.0 ** 1021,
                   2.0 ** 1020, 2.0 ** -1021, 1e-300, 1.0, -3.0])
    xs = np.array([1.0, 1.0, 1.0, -2.0, 1.0, 1.0, 1.0, 1.0, 1.0, 1.0, 3.0, 3.0, 1e-300, 1e300, 0.0, -0.0])
    with np.errstate(all="ignore"):
        q_ref, r_ref = xs / ys, 1.0 / ys
    q, r, _ = _div_points(xs, ys)
    for got, ref, what in ((q, q_ref, "x/y"), (r, r_ref, "1/y")):
        for i in range(len(ys)):
            if np.isnan(ref[i]):
                assert np.isnan(got[i]), (what, xs[i], ys[i], got[i])
            elif np.isfinite(ref[i]) and ref[i] != 0.0 and abs(ref[i]) >= tiny:
                assert abs(got[i] - ref[i]) <= ULP * abs(ref[i]), (what, xs[i], ys[i], got[i], ref[i])
            else:  # infinities, zeros, subnormals: IEEE's value and sign, bit for bit
                assert got[i].tobytes() == ref[i].tobytes(), (what, xs[i], ys[i], got[i], ref[i])
