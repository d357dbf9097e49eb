"""Snapshots from and into the device: a run saved to a .dat file, read
back into a fresh context (blocks in file order) and continued, matches the
run that never stopped, bit for bit."""
import numpy as np
import pytest

from tests import _amr as A

pytestmark = pytest.mark.gpu


def _cuda():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")


@pytest.mark.parametrize("nd", [2, 3])
def test_restart_from_snapshot_is_bit_exact(tmp_path, nd):
    _cuda()
    from amrvac_b200 import Context, datio, make_cfg
    nb = [4, 4] if nd == 2 else [2, 2, 2]
    xmin, xmax = [0.0] * nd, [1.0] * nd

    def ref(c, lv):
        return np.linalg.norm(c - 0.5) < (0.3 if lv == 1 else 0.15)
    leaves = [tuple(t) + (0,) * (4 - len(t)) for t in A.build_leaves(nd, nb, 3 if nd == 2 else 2, ref)]

    def prim(X, Y, Z):
        out = np.zeros((nd + 2,) + X.shape)
        out[0] = 1.0 + 0.2 * np.sin(2 * np.pi * X) * np.cos(2 * np.pi * Y)
        out[1] = 0.4
        out[nd + 1] = 1.0 + 0.1 * np.cos(2 * np.pi * X)
        return out
    kw = dict(physics="hd", ndim=nd, gamma=1.4, flux_scheme="hllc", limiter="vanleer",
              typeboundary=["periodic"] * (2 * nd))
    a = Context(make_cfg(**kw))
    a.set_amr_grid(leaves, nb, xmin, xmax)
    a.upload(A.fill_blocks(leaves, nd, nb, prim, "hd", nd, 1.4))
    a.set_time(0.0, 1.0e99, 0.0)
    for _ in range(3):
        a.step()
    path = str(tmp_path / "run0003.dat")
    datio.save(a, path, nbase=nb, xprobmin=xmin, xprobmax=xmax, it=3)
    for _ in range(2):
        a.step()
    wa = a.download()
    h, lv, blocks = datio.read_snapshot(path)
    assert h["it"] == 3 and h["time"] > 0 and h["nleafs"] == len(leaves)
    b = Context(make_cfg(**kw))
    b.set_amr_grid(lv, nb, h["xprobmin"], h["xprobmax"])
    b.upload(datio.ghosted(blocks, nd))
    b.set_time(h["time"], 1.0e99, 0.0)
    for _ in range(2):
        b.step()
    wb = b.download()
    sl = (slice(None),) + tuple(slice(2, 18) if d < nd else slice(None) for d in (2, 1, 0))
    for q, t in enumerate(lv):
        assert np.array_equal(wb[q][sl], wa[leaves.index(t)][sl]), t
    assert abs(b.get_time()[2] - a.get_time()[2]) == 0.0
    a.close()
    b.close()
