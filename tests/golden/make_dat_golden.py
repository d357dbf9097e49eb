"""Golden views of `.dat` snapshots through the reference's own reader.

Run in a checkout that has the reference repository next to it:

    python tests/golden/make_dat_golden.py /path/to/amrvac

For two small deterministic hierarchies (2-D, three levels; 3-D, two
levels) this writes a snapshot with amrvac_b200.datio, reads it back with the
reference's Python reader (tools/python/amrvac_pytools/datfiles/reading/
datfile_utilities.py: get_header, get_tree_info, get_single_block_data),
checks every block against the data written (by level and index), and
stores what the reference reader saw — header fields, block levels, indices
and byte offsets, and a checksum of each block — in dat_golden.json.  The
CPU tests compare the writer's output against this file, so the format stays
the one the reference's tools read.
"""
import hashlib
import importlib.util
import json
import os
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

from amrvac_b200 import datio  # noqa: E402
from tests import _amr as A  # noqa: E402


def cases():
    """(name, leaves, nbase, interior blocks, writer keywords)."""
    out = []
    for nd, nbase, levels in ((2, [4, 2], 3), (3, [2, 2, 2], 2)):
        def ref(c, lv):
            return np.linalg.norm(c - 0.4) < (0.3 if lv == 1 else 0.15)
        leaves = [tuple(t) + (0,) * (4 - len(t)) for t in A.build_leaves(nd, nbase, levels, ref)]

        def field(X, Y, Z):
            out = np.zeros((nd + 2,) + X.shape)
            out[0] = 1.0 + 0.5 * np.sin(2 * np.pi * X) * np.cos(2 * np.pi * Y)
            for c in range(nd):
                out[1 + c] = 0.1 * (c + 1) * np.cos(2 * np.pi * (X + c * Y))
            out[nd + 1] = 2.0 + Z + 0.25 * X * Y
            return out
        blocks = A.fill_blocks(leaves, nd, nbase, field, "hd", nd, 1.4, conserved=True, nghost=0)
        kw = dict(ndim=nd, ndir=nd, physics="hd", gamma=1.4, xprobmin=[0.0] * nd, xprobmax=[1.0] * nd,
                  nbase=nbase, time=0.125, it=7, snapshotnext=3)
        out.append((f"hd{nd}d", leaves, nbase, blocks, kw))
    return out


def checksum(a):
    return hashlib.sha256(np.ascontiguousarray(a, "<f8").tobytes()).hexdigest()[:16]


def main(ref_root):
    path = os.path.join(ref_root, "tools/python/amrvac_pytools/datfiles/reading/datfile_utilities.py")
    spec = importlib.util.spec_from_file_location("ref_datfile_utilities", path)
    U = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(U)
    golden = {}
    for name, leaves, nbase, blocks, kw in cases():
        nd = kw["ndim"]
        with tempfile.TemporaryDirectory() as td:
            f = os.path.join(td, "snap.dat")
            datio.write_snapshot(f, leaves, blocks, **kw)
            with open(f, "rb") as s:
                h = U.get_header(s)
                lvls, ixs, offs = U.get_tree_info(s)
                shape = list(h["block_nx"]) + [h["nw"]]
                sums = []
                for b in range(h["nleafs"]):
                    w = U.get_single_block_data(s, offs[b], shape)  # Fortran (x, y, [z,] var)
                    leaf = (int(lvls[b]),) + tuple(int(i) - 1 for i in ixs[b]) + (0,) * (3 - nd)
                    mine = blocks[leaves.index(leaf)]
                    mine_f = np.transpose(mine.reshape((h["nw"],) + tuple(reversed(h["block_nx"]))),
                                          tuple(range(nd, 0, -1)) + (0,))
                    assert np.array_equal(w, mine_f), (name, leaf)
                    sums.append(checksum(w.transpose(tuple(range(nd, -1, -1)))))
        golden[name] = {
            "header": {k: (v.tolist() if isinstance(v, np.ndarray) else v) for k, v in h.items()},
            "block_lvls": [int(x) for x in lvls], "block_ixs": [[int(i) for i in r] for r in ixs],
            "block_offsets": [int(x) for x in offs], "block_sha256_16": sums,
        }
        print(name, "ok:", h["nleafs"], "leaves,", h["nparents"], "parents")
    with open(os.path.join(HERE, "dat_golden.json"), "w") as f:
        json.dump(golden, f, indent=1, sort_keys=True)
    print("wrote", os.path.join(HERE, "dat_golden.json"))


if __name__ == "__main__":
    ref = sys.argv[1] if len(sys.argv) > 1 else os.environ.get("AMRVAC_REFERENCE")
    if not ref:
        sys.exit(f"usage: python {os.path.basename(__file__)} <MPI-AMRVAC source root> "
                 "(or set AMRVAC_REFERENCE)")
    main(ref)
