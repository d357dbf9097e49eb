""".dat snapshots (amrvac_b200.datio) against the reference's reader.

tests/golden/dat_golden.json holds what the reference's own Python reader
(datfile_utilities: get_header, get_tree_info, get_single_block_data) saw in
snapshots of two deterministic hierarchies; the writer must reproduce it
field by field, offset by offset and block by block.  Round trips are exact,
the forest's leaf flags describe the leaves in file order, and root blocks of
non-power-of-two grids follow the reference's Morton order.
"""
import hashlib
import importlib.util
import json
import os
import struct

import numpy as np
import pytest

from amrvac_b200 import datio

HERE = os.path.dirname(os.path.abspath(__file__))


def _golden_cases():
    spec = importlib.util.spec_from_file_location("make_dat_golden", os.path.join(HERE, "golden", "make_dat_golden.py"))
    m = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(m)
    return m.cases()


def _tree_info(path, h):
    with open(path, "rb") as f:
        data = f.read()
    n, nd = h["nleafs"], h["ndim"]
    p = h["offset_tree"] + 4 * (n + h["nparents"])
    lv = struct.unpack_from(f"<{n}i", data, p)
    ix = np.array(struct.unpack_from(f"<{n * nd}i", data, p + 4 * n)).reshape(n, nd)
    off = struct.unpack_from(f"<{n}q", data, p + 4 * n * (1 + nd))
    flags = struct.unpack_from(f"<{n + h['nparents']}i", data, h["offset_tree"])
    return list(lv), ix.tolist(), list(off), flags


@pytest.mark.parametrize("idx", [0, 1], ids=["hd2d", "hd3d"])
def test_writer_matches_what_the_reference_reader_saw(tmp_path, idx):
    with open(os.path.join(HERE, "golden", "dat_golden.json")) as f:
        golden = json.load(f)
    name, leaves, nbase, blocks, kw = _golden_cases()[idx]
    g = golden[name]
    path = str(tmp_path / "s.dat")
    datio.write_snapshot(path, leaves, blocks, **kw)
    h, lv_read, data = datio.read_snapshot(path)
    gh = g["header"]
    for ours, theirs in (("version", "datfile_version"), ("offset_tree", "offset_tree"),
                         ("offset_blocks", "offset_blocks"), ("nw", "nw"), ("ndir", "ndir"), ("ndim", "ndim"),
                         ("levmax", "levmax"), ("nleafs", "nleafs"), ("nparents", "nparents"), ("it", "it"),
                         ("time", "time"), ("xprobmin", "xmin"), ("xprobmax", "xmax"), ("domain_nx", "domain_nx"),
                         ("block_nx", "block_nx"), ("periodic", "periodic"), ("geometry", "geometry"),
                         ("w_names", "w_names"), ("physics_type", "physics_type"), ("gamma", "gamma")):
        a, b = h[ours], gh[theirs]
        assert (list(a) if isinstance(a, (list, tuple)) else a) == (list(b) if isinstance(b, (list, tuple)) else b), ours
    lv, ix, off, _ = _tree_info(path, h)
    assert lv == g["block_lvls"] and ix == g["block_ixs"]
    bc = 8 * h["ndim"]  # the reference reader skips the ghost-count record
    assert [o + bc for o in off] == g["block_offsets"]
    sums = [hashlib.sha256(np.ascontiguousarray(data[b], "<f8").tobytes()).hexdigest()[:16] for b in range(len(data))]
    assert sums == g["block_sha256_16"]


@pytest.mark.parametrize("idx", [0, 1], ids=["hd2d", "hd3d"])
def test_round_trip_and_forest(tmp_path, idx):
    name, leaves, nbase, blocks, kw = _golden_cases()[idx]
    nd = kw["ndim"]
    path = str(tmp_path / "s.dat")
    datio.write_snapshot(path, leaves, blocks, **kw)
    h, lv_read, data = datio.read_snapshot(path)
    assert sorted(lv_read) == sorted(leaves)
    for b, t in enumerate(lv_read):
        assert np.array_equal(data[b], blocks[leaves.index(t)])
    # the depth-first leaf flags (level-1 Morton order, children x fastest)
    # enumerate exactly the leaves in file order
    _, _, _, flags = _tree_info(path, h)
    roots = sorted((tuple(reversed(r)) for r in np.ndindex(*[nbase[d] for d in reversed(range(nd))])),
                   key=lambda ig: datio._morton(ig, nd))
    it = iter(flags)
    walk = []

    def node(L, ig):
        if next(it):
            walk.append((L,) + ig + (0,) * (3 - nd))
            return
        for cb in range(1 << nd):
            node(L + 1, tuple(2 * ig[d] + ((cb >> d) & 1) for d in range(nd)))
    for r in roots:
        node(1, r)
    assert walk == lv_read


def test_root_order_of_non_power_of_two_grids():
    """level1_Morton_order: Morton numbers over the smallest power-of-two
    square holding the grid, out-of-domain blocks skipped."""
    nb = [3, 2]
    leaves = [(1, i, j, 0) for j in range(nb[1]) for i in range(nb[0])]
    order = [leaves[b][1:3] for b in datio.leaf_order(leaves, 2, nb)]
    # Z order over the 4x4 square, x in the lowest bit: (0,0) (1,0) (0,1) (1,1) (2,0) (2,1)
    assert order == [(0, 0), (1, 0), (0, 1), (1, 1), (2, 0), (2, 1)]
