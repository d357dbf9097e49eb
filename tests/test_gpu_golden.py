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
