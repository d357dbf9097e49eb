"""MPI-AMRVAC `.dat` snapshots (format version 5) from and into the device pool.

The file layout restated here (src/io/mod_input_output.t:2004-2379
write_snapshot / read_snapshot, header src/io/mod_input_output_helper.t:
128-200 snapshot_write_header1, forest src/amr/mod_functions_forest.t:300-333
write_forest), little-endian, no padding:

* header: int32 version (5), offset_tree, offset_blocks, nw, ndir, ndim,
  levmax, nleafs, nparents, it; float64 time; float64 xprobmin[ndim],
  xprobmax[ndim]; int32 domain_nx[ndim] (level-1 cells), block_nx[ndim];
  logical (int32) periodic[ndim]; char[16] geometry; logical staggered;
  char[16] x nw conserved-variable names; char[16] physics type; int32 n_par,
  float64 values[n_par], char[16] x n_par names (hd / mhd: "gamma");
  int32 snapshotnext, slicenext, collapsenext;
* tree (at offset_tree): one logical per tree node, depth first over the
  level-1 blocks in Morton order (level1_Morton_order,
  src/amr/mod_space_filling_curve.t:7-56: bits interleaved x lowest over the
  smallest power-of-two square or cube holding the level-1 grid, blocks
  outside the domain skipped), children x fastest; then per leaf in that
  order int32 level, int32 ig[ndim] (1-based), int64 byte offset of the
  block record;
* blocks (at offset_blocks): per leaf int32 n_ghost[2 ndim] (zero: no
  physical-boundary ghost cells) and float64 w(ixM^S, 1:nw) in Fortran order.

Blocks move between the file and a Context through `download` / `upload`
(the library's host transfer path); the files read with the reference's own
Python reader (tools/python/amrvac_pytools/datfiles/reading).
"""
from __future__ import annotations

import struct

import numpy as np

VERSION = 5
NAME_LEN = 16


def _names(nw, ndir, physics):
    names = ["rho"] + [f"m{c + 1}" for c in range(ndir)] + ["e"]
    if physics == "mhd":
        names += [f"b{c + 1}" for c in range(ndir)]
    names += ["psi"] * (nw - len(names))
    return names[:nw]


def _pad(s):
    b = s.encode()[:NAME_LEN]
    return b + b" " * (NAME_LEN - len(b))


def _morton(ig, nd):
    """mortonEncode of 0-based level-1 indices, x in the lowest bit."""
    out = 0
    for bit in range(21):
        for d in range(nd):
            out |= ((ig[d] >> bit) & 1) << (nd * bit + d)
    return out


def leaf_order(leaves, nd, nbase):
    """Positions of the leaves in the file order (amr_Morton_order): level-1
    Morton order, then depth first with children x fastest."""
    def key(t):
        L, ig = t[0], t[1:1 + nd]
        root = tuple(i >> (L - 1) for i in ig)
        path = tuple(sum(((ig[d] >> (L - 1 - s)) & 1) << d for d in range(nd)) for s in range(1, L))
        return (_morton(root, nd),) + path
    return sorted(range(len(leaves)), key=lambda b: key(leaves[b]))


def forest_flags(leaves, nd, nbase):
    """write_forest: leaf flags depth first (level-1 Morton order, children x
    fastest), and the number of parents."""
    leafset = {tuple(t[:1 + nd]) for t in leaves}
    roots = [tuple(reversed(r)) for r in np.ndindex(*[nbase[d] for d in reversed(range(nd))])]
    roots.sort(key=lambda ig: _morton(ig, nd))
    flags = []

    def node(L, ig):
        if (L,) + ig in leafset:
            flags.append(True)
            return
        flags.append(False)
        for cb in range(1 << nd):
            node(L + 1, tuple(2 * ig[d] + ((cb >> d) & 1) for d in range(nd)))
    for r in roots:
        node(1, r)
    return flags, sum(1 for f in flags if not f)


def write_snapshot(path, leaves, blocks, *, ndim, ndir, physics, gamma, xprobmin, xprobmax, nbase, time=0.0,
                   it=0, periodic=None, geometry=None, snapshotnext=0, slicenext=0, collapsenext=0, nghost=2,
                   block_nx=16):
    """leaves: (level, ig0, ig1, ig2) per block (0-based ig); blocks: ghosted
    block arrays (nblocks, nw, nz, ny, nx) as Context.download returns them,
    or interior arrays (nblocks, nw, nz', ny', nx') with block_nx cells per
    dimension."""
    nd = ndim
    bnx = int(block_nx)
    blocks = np.asarray(blocks, np.float64)
    nw = blocks.shape[1]
    sl = (slice(None), slice(None)) + tuple(
        slice(nghost, nghost + bnx) if (d < nd and blocks.shape[4 - d] == bnx + 2 * nghost) else slice(None)
        for d in (2, 1, 0))
    inner = blocks[sl]
    order = leaf_order(leaves, nd, nbase)
    flags, nparents = forest_flags(leaves, nd, nbase)
    levmax = max(t[0] for t in leaves)
    periodic = [True] * nd if periodic is None else list(periodic)
    geometry = geometry or (f"Cartesian_{nd}D" if ndir == nd else f"Cartesian_{nd}.5D")
    head = bytearray()

    def i32(*v):
        head.extend(struct.pack("<" + "i" * len(v), *v))

    def f64(*v):
        head.extend(struct.pack("<" + "d" * len(v), *v))
    nleafs = len(leaves)

    def header(offset_tree, offset_blocks):
        head.clear()
        i32(VERSION, offset_tree, offset_blocks, nw, ndir, nd, levmax, nleafs, nparents, it)
        f64(time)
        f64(*[float(x) for x in xprobmin[:nd]])
        f64(*[float(x) for x in xprobmax[:nd]])
        i32(*[int(n) * bnx for n in nbase[:nd]])
        i32(*([bnx] * nd))
        i32(*[1 if p else 0 for p in periodic])
        head.extend(_pad(geometry))
        i32(0)  # staggered
        for n in _names(nw, ndir, physics):
            head.extend(_pad(n))
        head.extend(_pad(physics))
        i32(1)
        f64(float(gamma))
        head.extend(_pad("gamma"))
        i32(snapshotnext + 1, slicenext, collapsenext)
        return bytes(head)
    h0 = header(-1, -1)
    offset_tree = len(h0)
    tree = bytearray()
    tree.extend(struct.pack("<" + "i" * len(flags), *[1 if f else 0 for f in flags]))
    tree.extend(struct.pack("<" + "i" * nleafs, *[leaves[b][0] for b in order]))
    tree.extend(struct.pack("<" + "i" * (nleafs * nd), *[leaves[b][1 + d] + 1 for b in order for d in range(nd)]))
    offset_offsets = offset_tree + len(tree)
    offset_blocks = offset_offsets + 8 * nleafs
    rec = 4 * 2 * nd + 8 * nw * bnx ** nd
    offsets = [offset_blocks + q * rec for q in range(nleafs)]
    with open(path, "wb") as f:
        f.write(header(offset_tree, offset_blocks))
        f.write(bytes(tree))
        f.write(struct.pack("<" + "q" * nleafs, *offsets))
        ghosts = struct.pack("<" + "i" * (2 * nd), *([0] * (2 * nd)))
        for b in order:
            f.write(ghosts)
            f.write(np.ascontiguousarray(inner[b], dtype="<f8").tobytes())


def read_snapshot(path):
    """(header dict, leaves (level, ig0, ig1, ig2) 0-based in file order,
    interior blocks (nleafs, nw, nz, ny, nx) in file order)."""
    with open(path, "rb") as f:
        data = f.read()
    p = 0

    def take(fmt):
        nonlocal p
        v = struct.unpack_from("<" + fmt, data, p)
        p += struct.calcsize("<" + fmt)
        return v
    h = {}
    (h["version"], h["offset_tree"], h["offset_blocks"], h["nw"], h["ndir"], h["ndim"], h["levmax"], h["nleafs"],
     h["nparents"], h["it"]) = take("10i")
    if h["version"] < 5:
        raise ValueError(f"{path}: .dat version {h['version']} (5 expected)")
    (h["time"],) = take("d")
    nd, nw = h["ndim"], h["nw"]
    h["xprobmin"] = list(take(f"{nd}d"))
    h["xprobmax"] = list(take(f"{nd}d"))
    h["domain_nx"] = list(take(f"{nd}i"))
    h["block_nx"] = list(take(f"{nd}i"))
    h["periodic"] = [bool(x) for x in take(f"{nd}i")]
    h["geometry"] = data[p:p + NAME_LEN].decode().strip()
    p += NAME_LEN
    (h["staggered"],) = take("i")
    h["w_names"] = []
    for _ in range(nw):
        h["w_names"].append(data[p:p + NAME_LEN].decode().strip())
        p += NAME_LEN
    h["physics_type"] = data[p:p + NAME_LEN].decode().strip()
    p += NAME_LEN
    (npar,) = take("i")
    vals = take(f"{npar}d")
    for k in range(npar):
        h[data[p:p + NAME_LEN].decode().strip()] = vals[k]
        p += NAME_LEN
    h["snapshotnext"], h["slicenext"], h["collapsenext"] = take("3i")
    nleafs = h["nleafs"]
    p = h["offset_tree"] + 4 * (nleafs + h["nparents"])
    lv = take(f"{nleafs}i")
    ig = np.array(take(f"{nleafs * nd}i")).reshape(nleafs, nd) - 1
    offs = take(f"{nleafs}q")
    bn = h["block_nx"]
    shape = (nw,) + tuple(bn[d] if d < nd else 1 for d in (2, 1, 0))
    blocks = np.empty((nleafs,) + shape)
    for b in range(nleafs):
        ng = struct.unpack_from("<" + "i" * (2 * nd), data, offs[b])
        if any(ng):
            raise ValueError(f"{path}: blocks with physical-boundary ghost cells are not supported")
        q = offs[b] + 8 * nd
        blocks[b] = np.frombuffer(data, "<f8", int(np.prod(shape)), q).reshape(shape)
    leaves = [(int(lv[b]),) + tuple(int(x) for x in ig[b]) + (0,) * (3 - nd) for b in range(nleafs)]
    return h, leaves, blocks


def save(ctx, path, *, nbase, xprobmin, xprobmax, leaves=None, it=0, time=None, **kw):
    """write_snapshot of a Context's register ps.  Leaves default to the
    multi-level grid's (Context.amr_leaves) or, on a grid set by
    set_uniform_grid, level-1 blocks x fastest."""
    cfg = ctx.cfg
    if leaves is None:
        try:
            leaves = ctx.amr_leaves()
        except RuntimeError:
            nb = list(nbase) + [1] * (3 - cfg.ndim)
            leaves = [(1, b % nb[0], (b // nb[0]) % nb[1], b // (nb[0] * nb[1])) for b in range(ctx.nblocks)]
    if time is None:
        time = ctx.get_time()[2]
    write_snapshot(path, leaves, ctx.download(), ndim=cfg.ndim, ndir=cfg.ndir,
                   physics="mhd" if cfg.physics == 1 else "hd", gamma=cfg.gamma, xprobmin=xprobmin,
                   xprobmax=xprobmax, nbase=nbase, it=it, time=time, block_nx=ctx.bn, **kw)


def ghosted(blocks, nd, nghost=2):
    """Interior blocks as ghosted arrays (zero ghosts) for Context.upload."""
    nb, nw = blocks.shape[:2]
    bnx = blocks.shape[-1]
    g = [bnx + 2 * nghost if d < nd else 1 for d in range(3)]
    out = np.zeros((nb, nw, g[2], g[1], g[0]))
    sl = (slice(None), slice(None)) + tuple(slice(nghost, nghost + bnx) if d < nd else slice(None) for d in (2, 1, 0))
    out[sl] = blocks
    return out
