"""Pin the CPU oracle against the reference's own golden regression logs.

tests/mhd/field_loop_2.5D (reference): 128x64 periodic, 2.5D ideal MHD,
SSP-RK3, cada3, CFL 0.9, volume-averaged regression log every 0.01 to t=0.5.
Acceptance is the reference's compare_logs rule with rtol=1e-5, atol=1e-8
(tests/test_rules.make:45, tools/fortran/compare_logs.f:44-48).
"""
import os

import numpy as np
import pytest

GOLD = os.path.join(os.path.dirname(__file__), "golden")


@pytest.mark.parametrize("name,kw", [
    ("hlld", dict(flux_scheme="hlld", limiter="cada3", divb="glm")),
    ("hll", dict(flux_scheme="hll", limiter="cada3", divb="linde", typeboundspeed="cmaxmean")),
])
def test_field_loop_golden_log(oracle_lib, name, kw):
    O = oracle_lib
    c = O.make_cfg(ndim=2, ndir=3, physics="mhd", **kw)
    rows = O.run_field_loop(c, 0.9, time_max=0.5, dtsave=0.01)
    gold = O.read_log(os.path.join(GOLD, f"fl_2d_3step_{name}_cada.log"))
    assert rows.shape == gold.shape
    assert O.compare_logs(rows, gold, rtol=1e-5, atol=1e-8)
    # tighter: the B_err column (deviation from the analytic advected loop)
    ib = 1 + (c.nw + 2)
    rel = np.abs(rows[:, ib] - gold[:, ib]) / np.abs(gold[:, ib])
    assert rel.max() < 1e-5


def test_field_loop_golden_discriminates(oracle_lib):
    """A wrong limiter must fail the same comparison (the pin is not vacuous)."""
    O = oracle_lib
    c = O.make_cfg(ndim=2, ndir=3, physics="mhd", flux_scheme="hlld", limiter="vanleer", divb="glm")
    rows = O.run_field_loop(c, 0.9, time_max=0.5, dtsave=0.01)
    gold = O.read_log(os.path.join(GOLD, "fl_2d_3step_hlld_cada.log"))
    assert not O.compare_logs(rows, gold, rtol=1e-5, atol=1e-8)
