#!/usr/bin/env python
"""Benchmark of the B200 finite-volume block update (one JSON line on rank 0).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                    [--workload ot128|ot256|kh256|ens512|blast512adj|amrblast3d]

A step is one full SSP-RK3 time step of the whole grid: setdt (CFL reduction
on the device), three fused finite-volume stages, time update.  The default
workload is 3-D ideal MHD Orszag-Tang at 128^3 (512 blocks of 16^3), HLLD,
cada3, GLM, FP64, periodic.  `value` is zone-updates/s (interior cells x full
steps / s) with the state resident in HBM, timed with CUDA events on the
library's stream; N>1 runs independent replicas, one per GPU (weak scaling),
with the max time over ranks.

--impl reference times the reference algorithm's CPU implementation (the C++
restatement in oracle/, all host threads) on a bounded sample of the same
workload (a 1/8 sub-box with the same per-cell work), rank 0 only.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "zone-updates/s on 1 B200, plain FP64 vs mixed/batched at fixed L1 err; adj/fwd"
UNIT = "zone-updates/s"

WORKLOADS = {
    "ot128": dict(desc="3D ideal MHD Orszag-Tang 128^3, 512 blocks of 16^3, HLLD + cada3 + GLM, SSP-RK3, FP64, "
                       "periodic", physics="mhd", n=128, ndim=3),
    "ot256": dict(desc="3D ideal MHD Orszag-Tang 256^3, 4096 blocks of 16^3, HLLD + cada3 + GLM, SSP-RK3, FP64, "
                       "periodic", physics="mhd", n=256, ndim=3),
    "kh256": dict(desc="2D Euler Kelvin-Helmholtz 256^2, 256 blocks of 16^2, HLLC + vanleer, SSP-RK3, FP64, "
                       "periodic", physics="hd", n=256, ndim=2),
    "ens512": dict(desc="Batched ensemble: 512 independent Euler Riemann problems (256 1-D of 64-4096 cells, "
                        "256 2-D of 32^2-512^2 in 16^2 blocks), HLL/HLLC x minmod/vanleer per instance, SSP-RK3 "
                        "to t=0.2 with per-instance CFL dt (0.8), cont boundaries, one persistent launch per stage",
                   physics="hd", ensemble=512),
    "blast512adj": dict(desc="Adjoint of the 2D Euler blast wave: 512^2 as 32x32 blocks of 16^2, gamma=1.4, "
                             "rho = 1 + 0.1 G (Gaussian random field, correlation length 0.05), p = 0.1 with "
                             "p = 10 for r < 0.1, v = 0, cont boundaries; HLL, minmod, SSP-RK3, 200 steps at the "
                             "CFL (0.8) dt sequence of the forward run; loss = sum rho^2 on 0.25 < r < 0.35; "
                             "gradient w.r.t. the initial rho field and gamma, checkpoint every 20 steps",
                        physics="hd", adjoint=dict(n=512, steps=200, every=20)),
    "amrblast3d": dict(desc="3D ideal MHD blast on a Löhner-refined hierarchy: [-0.5,0.5]^3, base 64^3 (4^3 root "
                            "blocks of 16^3), refine_max_level 4 (effective 512^3); initial tree by settree on the "
                            "initial state (Löhner, w_refine_weight 0.5 rho + 0.5 e, refine_threshold 0.1, "
                            "derefine_ratio 1/8, amr_wavefilter 1e-2), kept fixed over the timed steps; gamma 5/3, "
                            "rho 1, p 0.1 with p 100 for r < 0.1, B = (1,1,0)/sqrt 2, v = 0, psi = 0; HLLD, "
                            "vanleer, GLM, SSP-RK3, CFL 0.8, cont boundaries; every leaf block in one stage launch, "
                            "level-jump ghost pass and flux fix per stage",
                       physics="mhd", amr=dict(nbase=4, levels=4)),
}

# Signal-speed estimate of the ensemble workload (typeboundspeed).  With the
# default Einfeldt estimate (Roe averages only, Toro eq. 10.52) 34 of the 512
# seeded instances turn non-finite within ten steps (strongly diverging states
# whose rarefaction head it does not bound: negative pressure under a square
# root), in the oracle as on the GPU; cmaxleftright bounds both heads and
# every instance reaches t = 0.2.
ENS_BOUNDSPEED = "cmaxleftright"

# Algorithmic FP64 operations (+,-,*,/,sqrt,exp each 1) per cell for one
# stage and for one getdt, counted by the oracle's counting scalar on the same
# physics (tests/test_flop_counts.py recomputes and checks these numbers).
ALG_FLOPS = {
    "ot128": dict(stage=2047.0, getdt=86.5),
    "ot256": dict(stage=2047.0, getdt=86.5),
    "kh256": dict(stage=416.7, getdt=21.0),
    "amrblast3d": dict(stage=1696.5, getdt=86.5),
}
# Per-launch DRAM traffic of the stage kernel from one ncu capture, bytes per
# interior cell; None until captured.  ot128: the FP64 kernel's stage-1
# launch (variant 0, z-chunks of 8; ps -> ps1; algorithmic 2 * 8 * nw = 144 B
# per cell), dram__bytes_read.sum + dram__bytes_write.sum = 181.38 MB +
# 127.85 MB over 128^3 cells.
NCU_TRAFFIC_PER_CELL = {"ot128": (181.381888e6 + 127.851776e6) / 128 ** 3, "ot256": None, "kh256": None}


def _tile(ctx, zchunk):
    """The autotuned launch shape of the stage kernel: work distribution and
    kernel variant (threads per CTA, CTAs per SM, staging mode)."""
    v = ctx.stage_variant()
    return {"zchunk": zchunk, "distribution": "persistent plane ranges" if zchunk == 0 else f"z-chunks of {zchunk}",
            "variant": v["variant"], "variants_timed": v["nvariants"], "threads": v["threads"],
            "ctas_per_sm": v["ctas_per_sm"],
            "staging": "asynchronous bulk copies" if v["async_staging"] else "gathered loads"}


def _cfg_kwargs(wl: str):
    w = WORKLOADS[wl]
    if w["physics"] == "mhd":
        return dict(physics="mhd", ndim=3, ndir=3, flux_scheme="hlld", limiter="cada3", typedivbfix="glm",
                    courantpar=0.8)
    return dict(physics="hd", ndim=2, gamma=1.4, flux_scheme="hllc", limiter="vanleer", courantpar=0.8)


def _initial_blocks(wl: str, n: int | None = None):
    from tests import _problems as P
    w = WORKLOADS[wl]
    n = n or w["n"]
    if w["physics"] == "mhd":
        prim, geo = P.orszag_tang_3d(n=n)
        cons = P.prim_to_cons(prim, "mhd", 3, 5.0 / 3.0)
        return P.to_blocks(cons, 3), geo
    prim, geo = P.kh_2d(n=n)
    cons = P.prim_to_cons(prim, "hd", 2, 1.4)
    return P.to_blocks(cons, 2), geo


def _interior(blocks, ndim, ng=2):
    from tests import _problems as P
    return P.interior(blocks, ndim, ng)


def _measured_peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            return json.load(f), "measured"
    except OSError:
        return {"hbm_gbs": 6650.0, "bf16_tflops": 1590.0}, "fallback"


class ClockSampler:
    """Samples SM clock and throttle reasons of one GPU through NVML."""

    def __init__(self, device_index: int):
        self.samples = []
        self.reasons = set()
        self.max_mhz = None
        self._stop = threading.Event()
        self._t = None
        try:
            import pynvml
            pynvml.nvmlInit()
            self.nv = pynvml
            import torch
            uuid = str(torch.cuda.get_device_properties(device_index).uuid)
            try:
                self.h = pynvml.nvmlDeviceGetHandleByUUID(("GPU-" + uuid) if not uuid.startswith("GPU") else uuid)
            except Exception:
                self.h = pynvml.nvmlDeviceGetHandleByIndex(device_index)
            self.max_mhz = pynvml.nvmlDeviceGetMaxClockInfo(self.h, pynvml.NVML_CLOCK_SM)
        except Exception:
            self.nv = None

    def _run(self):
        nv = self.nv
        names = {
            "hw_slowdown": getattr(nv, "nvmlClocksEventReasonHwSlowdown", 0x8),
            "sw_thermal_slowdown": getattr(nv, "nvmlClocksEventReasonSwThermalSlowdown", 0x20),
            "hw_thermal_slowdown": getattr(nv, "nvmlClocksEventReasonHwThermalSlowdown", 0x40),
            "sw_power_cap": getattr(nv, "nvmlClocksEventReasonSwPowerCap", 0x4),
        }
        while not self._stop.is_set():
            try:
                self.samples.append(nv.nvmlDeviceGetClockInfo(self.h, nv.NVML_CLOCK_SM))
                r = nv.nvmlDeviceGetCurrentClocksEventReasons(self.h)
                for k, bit in names.items():
                    if r & bit:
                        self.reasons.add(k)
            except Exception:
                pass
            self._stop.wait(0.05)

    def __enter__(self):
        if self.nv is not None:
            self._t = threading.Thread(target=self._run, daemon=True)
            self._t.start()
        return self

    def __exit__(self, *a):
        self._stop.set()
        if self._t:
            self._t.join()

    def summary(self):
        return {"sm_mhz": statistics.median(self.samples) if self.samples else None,
                "sm_max_mhz": self.max_mhz, "reasons": sorted(self.reasons), "samples": len(self.samples)}


def _dist_init():
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if ws > 1:
        import torch.distributed as dist
        import datetime
        dist.init_process_group("gloo", timeout=datetime.timedelta(seconds=300))
    return ws, rank, local


def _allmax(x: float, ws: int) -> float:
    if ws == 1:
        return x
    import torch
    import torch.distributed as dist
    t = torch.tensor([x], dtype=torch.float64)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def _barrier(ws):
    if ws > 1:
        import torch.distributed as dist
        dist.barrier()


def _config(wl: str) -> dict:
    """The workload as both arms report it: identical in --impl ours and
    --impl reference (the run-dependent details go to other keys)."""
    w = WORKLOADS[wl]
    c = {"workload": w["desc"]}
    if "n" in w:
        cells = w["n"] ** w["ndim"]
        nw = 9 if w["physics"] == "mhd" else 4
        mb = 3 * cells * nw * 8 / 1e6
        c.update(cells=cells, blocks=cells // 16 ** w["ndim"], nw=nw,
                 step="one SSP-RK3 time step of the whole grid: setdt + 3 stages + time update",
                 l2=(f"no flush: working set {mb:.0f} MB (3 registers) > 126 MB L2" if mb > 126 else
                     f"L2 flushed (256 MB write) before every timed step: working set {mb:.1f} MB < 126 MB L2"))
    return c


def _oracle_cfg_uniform(wl: str):
    import oracle as O
    if WORKLOADS[wl]["physics"] == "mhd":
        return O.make_cfg(physics="mhd", ndim=3, ndir=3, flux_scheme="hlld", limiter="cada3", divb="glm",
                          courantpar=0.8)
    return O.make_cfg(physics="hd", ndim=2, gamma=1.4, flux_scheme="hllc", limiter="vanleer", courantpar=0.8)


def _oracle_grid_uniform(wl: str, blocks, geo):
    """The oracle's uniform grid of the workload (C++ restatement, OpenMP)."""
    import oracle as O
    O.build()
    g = O.Grid(_oracle_cfg_uniform(wl), geo["domain_nx"], geo["xprobmin"], geo["xprobmax"],
               ["periodic"] * (2 * WORKLOADS[wl]["ndim"]))
    for ib in range(g.nblocks):
        g.set_block(ib, blocks[ib])
    g.getbc()
    return g


def _oracle_step(g, nthreads):
    """One full step of the oracle (setdt + advance); returns its wall time (s)."""
    t0 = time.perf_counter()
    dt, cg = g.getdt()
    g.advance(dt, cg, nthreads)
    return time.perf_counter() - t0


def _parity_first_step(wl, blocks, geo, got, nthreads):
    """The device's first FP64 step from the initial state against the
    oracle's, per variable with the per-cell measure of tests/_parity.py.
    A variable's bar is max(1e-12, the oracle's own response to one ulp of
    input noise on the same data); returns (parity, cpu seconds of the step)."""
    from tests._parity import percell_parts
    nd = WORKLOADS[wl]["ndim"]
    g = _oracle_grid_uniform(wl, blocks, geo)
    t_cpu = _oracle_step(g, nthreads)
    ref = _interior(np.array([g.get_block(ib) for ib in range(g.nblocks)]), nd)
    rng = np.random.default_rng(1)
    gp = _oracle_grid_uniform(wl, blocks * (1.0 + 2.0 ** -52 * rng.choice([-1.0, 1.0], blocks.shape)), geo)
    _oracle_step(gp, nthreads)
    noisy = _interior(np.array([gp.get_block(ib) for ib in range(gp.nblocks)]), nd)
    got = _interior(got, nd)
    per, ok = [], True
    for v in range(ref.shape[1]):
        if not np.any(ref[:, v]):
            d = float(np.abs(got[:, v]).max() / (1e-3 * np.abs(ref).max()))
            per.append({"var": v, "zero_in_reference": True, "abs_over_floor": d})
            ok = ok and d <= 1e-12
            continue
        rel, small = percell_parts(got[:, v:v + 1], ref[:, v:v + 1])
        nrel, nsmall = percell_parts(noisy[:, v:v + 1], ref[:, v:v + 1])
        bar = max(1e-12, nrel, nsmall)
        per.append({"var": v, "rel": rel, "small_cell": small, "oracle_1ulp_self_noise": max(nrel, nsmall),
                    "bar": bar})
        ok = ok and rel <= bar and small <= bar
    ndir = 3 if ref.shape[1] >= 8 else nd
    mag = np.sqrt((ref[:, 1:1 + ndir] ** 2).sum(axis=1))
    big = mag >= 1e-3 * mag.max()
    dm = np.sqrt(((got[:, 1:1 + ndir] - ref[:, 1:1 + ndir]) ** 2).sum(axis=1))
    vec = float((dm[big] / mag[big]).max())
    ok = ok and vec <= 1e-12
    worst_rel = max(p.get("rel", 0.0) for p in per)
    return {"steps": 1, "ok": bool(ok), "tolerance": 1e-12, "max_rel_any_variable": worst_rel,
            "momentum_vector_rel": vec, "per_variable": per,
            "measure": "per cell: relative error where |ref| >= 1e-3 max|ref_v|, |diff| / (1e-3 max|ref_v|) "
                       "below; bar per variable max(1e-12, oracle self-noise under 1 ulp of input noise)"}, t_cpu


def run_reference(args, ws, rank):
    """The reference algorithm's CPU implementation (the oracle, all host
    threads) on the same workload, rank 0 only.  Uniform workloads: the full
    grid, built once outside the timing; W warm-up steps, then K timed steps
    of setdt + the three stages (each step times only itself)."""
    if rank != 0:
        return
    nthreads = os.cpu_count() or 1
    wl = args.workload
    w = WORKLOADS[wl]
    if "n" in w:
        blocks, geo = _initial_blocks(wl)
        g = _oracle_grid_uniform(wl, blocks, geo)
        cells = w["n"] ** w["ndim"]
        for _ in range(args.warmup):
            _oracle_step(g, nthreads)
        secs = [_oracle_step(g, nthreads) for _ in range(args.steps)]
        el = float(sum(secs))
        value = cells * args.steps / el
        sample = (f"{args.steps} full SSP-RK3 steps (setdt + 3 stages) of the whole {w['n']}^{w['ndim']} grid after "
                  f"{args.warmup} warm-up steps, oracle (C++ restatement, OpenMP)")
        ms = 1e3 * el / args.steps
    else:
        if "ensemble" in w:
            from tests import _riemann as R
            specs = R.ensemble_specs(w["ensemble"])
            init = [R.initial_blocks(sp, 1.4) for sp in specs]

            def sample_fn():  # a few seconds of whole instances per step
                v, _, smp = _ens_cpu_sample(specs, init, budget_s=3.0)
                return v, smp
        elif "adjoint" in w:
            from tests import _blast as B
            import oracle as O
            O.build()
            n = w["adjoint"]["n"]
            c = O.make_cfg(physics="hd", ndim=2, gamma=B.GAMMA, flux_scheme="hll", limiter="minmod", courantpar=0.8)
            w0 = B.to_cons_blocks(B.blast_prim(n))

            def sample_fn():  # the oracle's forward run of the blast, 10 steps (the reference has no adjoint)
                g = O.Grid(c, [n, n], [0.0, 0.0], [1.0, 1.0], ["cont"] * 4)
                for ib in range(g.nblocks):
                    g.set_block(ib, w0[ib])
                g.getbc()
                t0 = time.perf_counter()
                for _ in range(10):
                    dt, _ = g.getdt()
                    g.advance(dt, 0.0, nthreads)
                return n * n * 10 / (time.perf_counter() - t0), f"10 SSP-RK3 steps of the {n}^2 blast (forward only)"
        else:
            tree, blocks = _amr_tree_oracle(w)

            def sample_fn():  # one multi-level step of the whole hierarchy
                v, _ = _amr_cpu_sample(tree, blocks, nthreads, 1)
                return v, (f"1 SSP-RK3 step of the whole {len(tree.leaves)}-block hierarchy "
                           f"(levels {tree.counts()}), oracle multi-level advance")
        for _ in range(args.warmup):
            sample_fn()
        vals, sample = [], ""
        t0 = time.perf_counter()
        for _ in range(args.steps):
            v, sample = sample_fn()
            vals.append(v)
        value = float(np.mean(vals))
        ms = 1e3 * (time.perf_counter() - t0) / args.steps
    print(json.dumps({
        "impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic", "config": _config(wl), "execution": f"host threads ({nthreads})",
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": nthreads, "kind": "port", "sample": sample},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }))


def _ens_build(specs, precision, boundspeed=ENS_BOUNDSPEED):
    from amrvac_b200 import Ensemble, make_cfg
    from tests import _riemann as R
    cfg = make_cfg(physics="hd", ndim=2, gamma=1.4, courantpar=0.8, typeboundary=["cont"] * 4, precision=precision,
                   typeboundspeed=boundspeed)
    return Ensemble(cfg, [R.instance(s) for s in specs])


def _ens_cpu_sample(specs, init, budget_s=15.0):
    """Oracle (C++ restatement), one instance per host thread, on whole instances
    taken smallest first until about budget_s of CPU work; zone-updates/s."""
    import concurrent.futures as cf
    import oracle as O
    O.build()
    nthreads = os.cpu_count() or 1
    order = sorted(range(len(specs)), key=lambda i: int(np.prod(specs[i]["shape"])))

    def one(i):
        s = specs[i]
        nd = s["ndim"]
        c = O.make_cfg(physics="hd", ndim=nd, gamma=1.4, flux_scheme=s["flux_scheme"], limiter=s["limiter"],
                       courantpar=0.8, typeboundspeed=ENS_BOUNDSPEED)
        g = O.Grid(c, list(s["shape"]), [0.0] * nd, [1.0] * nd, ["cont"] * (2 * nd))
        for ib in range(g.nblocks):
            g.set_block(ib, init[i][ib])
        g.getbc()
        t, n = 0.0, 0
        while True:
            dt, _ = g.getdt()
            if s["time_max"] - t <= 1e-10:
                break
            g.advance(min(dt, s["time_max"] - t), 0.0, 1)
            t += min(dt, s["time_max"] - t)
            n += 1
        return int(np.prod(s["shape"])) * n

    done_zu, used = 0, []
    t0 = time.perf_counter()
    with cf.ThreadPoolExecutor(max_workers=nthreads) as ex:
        futs = []
        for i in order:
            futs.append(ex.submit(one, i))
            used.append(i)
            if len(futs) >= nthreads:
                done_zu += futs.pop(0).result()
            if time.perf_counter() - t0 > budget_s:
                break
        for f in futs:
            done_zu += f.result()
    el = time.perf_counter() - t0
    return done_zu / el, nthreads, (f"{len(used)} whole instances of the ensemble (smallest first) run to t=0.2 "
                                    f"by the oracle, one instance per host thread")


def run_ensemble(args, ws, rank, local):
    """Batched-ensemble workload: a step is one full run of all instances to t=0.2."""
    import torch
    from tests import _riemann as R
    if not torch.cuda.is_available():
        raise SystemExit("bench.py: no CUDA device")
    torch.cuda.set_device(local)
    w = WORKLOADS[args.workload]
    specs = R.ensemble_specs(w["ensemble"])
    init = [R.initial_blocks(sp, 1.4) for sp in specs]
    nw = np.array([sp["ndim"] + 2 for sp in specs], np.float64)
    cells = np.array([int(np.prod(sp["shape"])) for sp in specs], np.float64)
    runs = max(1, min(args.steps, 2))
    peaks, peak_kind = _measured_peaks()

    def load(ens):
        for i in range(len(specs)):
            ens.upload(i, init[i])
        ens.reset_time()

    def timed_run(ens, clocks=None):
        s = torch.cuda.ExternalStream(ens.stream_ptr())
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        l0 = ens.launch_count()
        e0.record(s)
        taken, active = ens.run(max_steps=args.it_max or (1 << 30), chunk=16)
        e1.record(s)
        e1.synchronize()
        _, _, steps, done = ens.state()
        return e0.elapsed_time(e1), steps.astype(np.float64), active, ens.launch_count() - l0, taken

    out = {}
    finals = {}
    for prec in ("fp64", "mixed"):
        ens = _ens_build(specs, prec)
        load(ens)
        grid, tune_ms = ens.autotune(reps=3)
        tuned = ens.variant()
        for _ in range(args.warmup):  # partial runs: kernels, graph, first touch
            load(ens)
            ens.run(max_steps=min(64, args.it_max or 64), chunk=16)
        ms_all, zu = [], 0.0
        clk = ClockSampler(local) if prec == "fp64" else None
        if clk:
            clk.__enter__()
        for _ in range(runs):
            load(ens)
            _barrier(ws)
            ms, steps, active, launches, taken = timed_run(ens)
            ms_all.append(_allmax(ms, ws))
            zu = float((cells * steps).sum())
            if active and not args.it_max:
                raise SystemExit(f"bench.py: {active} instances did not finish")
        if clk:
            clk.__exit__()
        flags, per = ens.status()
        finals[prec] = [ens.download(i) for i in range(len(specs))]
        ms = float(np.mean(ms_all))
        alg_bytes = float((cells * steps * 72.0 * nw).sum())  # 72*nw B per zone-update: 3 stages + getdt
        out[prec] = dict(ms=ms, value=ws * zu / (ms * 1e-3), steps=steps, grid=grid, tune_ms=tune_ms, tuned=tuned,
                         launches=launches, chunk_steps=taken, status=flags,
                         hbm_gbs=alg_bytes / (ms * 1e-3) / 1e9, clocks=clk.summary() if clk else None)
        if prec == "fp64":
            # e2e: pinned host arrays in, run, host arrays out
            pins = [torch.empty(b.shape, dtype=torch.float64).pin_memory() for b in init]
            for p_, b in zip(pins, init):
                p_.numpy()[...] = b
            s = torch.cuda.ExternalStream(ens.stream_ptr())
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            torch.cuda.synchronize()
            e0.record(s)
            for i, p_ in enumerate(pins):
                ens.upload(i, p_.numpy())
            ens.reset_time()
            ens.run(max_steps=args.it_max or (1 << 30), chunk=16)
            res = [ens.download(i) for i in range(len(specs))]
            e1.record(s)
            e1.synchronize()
            e2e_ms = _allmax(e0.elapsed_time(e1), ws)
            nbytes = float(sum(b.nbytes for b in init))
            out["e2e"] = {"value": ws * zu / (e2e_ms * 1e-3), "unit": UNIT, "h2d_bytes_per_step": nbytes,
                          "d2h_bytes_per_step": float(sum(r.nbytes for r in res)),
                          "what": "C-ABI: upload of every instance from pinned host block arrays, the run to "
                                  "t=0.2, download of every instance with ghost cells"}
        ens.close()
    l1 = []
    for i, sp in enumerate(specs):
        a = _interior(finals["fp64"][i], sp["ndim"])[:, 0]
        b = _interior(finals["mixed"][i], sp["ndim"])[:, 0]
        l1.append(float(np.abs(b - a).sum() / np.abs(a).sum()))
    f = out["fp64"]
    cpu = None
    if rank == 0 and ws == 1 and not args.no_cpu_baseline:
        v, cores, sample = _ens_cpu_sample(specs, init)
        cpu = {"value": v, "unit": UNIT, "cores": cores, "kind": "port", "sample": sample}
    if rank == 0:
        print(json.dumps({
            "metric": METRIC, "value": f["value"], "unit": UNIT, "n_gpus": ws, "steps": runs,
            "warmup": args.warmup, "ms_per_step": f["ms"], "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": _config(args.workload),
            "run": {"step": ("one full run of every instance to t=0.2" if not args.it_max else
                                f"every instance for at most {args.it_max} steps (it_max)"),
                       "typeboundspeed": ENS_BOUNDSPEED,
                       "instances": len(specs), "cells": float(cells.sum()),
                       "zone_updates_per_run": float((cells * f["steps"]).sum()),
                       "max_steps_of_an_instance": int(f["steps"].max()), "graph_chunk_steps": 16,
                       "grid_ctas": f["grid"], "autotuned_stage_ms": f["tune_ms"],
                       "stage_variant": f["tuned"],
                       "parallelism": "replicas" if ws > 1 else "single GPU",
                       "l2": "no flush: working set %.0f MB (3 registers) > 126 MB L2" % (
                           3 * float((cells * nw).sum()) * 8 / 1e6)},
            "roofline": {"bound": "hbm", "achieved": f["hbm_gbs"], "peak": peaks["hbm_gbs"], "unit": "GB/s",
                         "frac": f["hbm_gbs"] / peaks["hbm_gbs"], "peak_source": peak_kind, "traffic": None,
                         "kernel": "whole run (ens_getdt + 3 x ens_stage per step)",
                         "algorithmic_bytes_per_zone_update": "72*nw (nw = 3 in 1-D, 4 in 2-D)"},
            "cpu_baseline": cpu, "e2e": out["e2e"],
            "mixed": {"value": out["mixed"]["value"], "unit": UNIT, "ms_per_step": out["mixed"]["ms"],
                      "speedup_vs_fp64": f["ms"] / out["mixed"]["ms"], "grid_ctas": out["mixed"]["grid"],
                      "stage_variant": out["mixed"]["tuned"],
                      "l1_rel_err_density_vs_fp64": {"max": max(l1), "median": float(np.median(l1))},
                      "status": out["mixed"]["status"]},
            "gpu_launches": int(f["launches"]), "clocks": f["clocks"], "status": f["status"],
        }))


def run_adjoint(args, ws, rank, local):
    """Adjoint workload: a step is one gradient evaluation (forward run of all
    steps + the checkpointed adjoint sweep)."""
    import torch
    from tests import _blast as B
    from amrvac_b200.adjoint import FrozenDtSolver, blocks_to_domain, domain_to_blocks, solve
    if not torch.cuda.is_available():
        raise SystemExit("bench.py: no CUDA device")
    torch.cuda.set_device(local)
    w = WORKLOADS[args.workload]
    n, nsteps, every = w["adjoint"]["n"], w["adjoint"]["steps"], w["adjoint"]["every"]
    dev = "cuda"
    prim = B.blast_prim(n)
    rho0 = torch.tensor(prim[0, 0], dtype=torch.float64, device=dev)
    p0 = torch.tensor(prim[3, 0], dtype=torch.float64, device=dev)
    mask = torch.tensor(B.loss_mask(n), dtype=torch.float64, device=dev)
    grid = ((n, n), (0.0, 0.0), (1.0, 1.0))
    kw = dict(limiter="minmod", typeboundary=["cont"] * 4)
    G = lambda x: torch.tensor(x, dtype=torch.float64, device=dev)  # noqa: E731

    def U0_of(r, g):
        z = torch.zeros_like(r)
        return domain_to_blocks(torch.stack([r, z, z, p0 / (g - 1.0)]))

    solver = FrozenDtSolver(*grid, B.GAMMA, **kw)
    dts = solver.cfl_dts(U0_of(rho0, G(B.GAMMA)), nsteps)

    def loss(r, g):
        UN = solve(U0_of(r, g), g, dts, *grid, checkpoint_every=every, **kw)
        rho = blocks_to_domain(UN, n, n)[0]
        return (mask * rho * rho).sum()

    # ---- timing: forward sweep and adjoint sweep, CUDA events on the library stream
    s = torch.cuda.ExternalStream(solver.ctx.stream_ptr())
    U0 = U0_of(rho0, G(B.GAMMA)).contiguous()
    lamN = torch.zeros(solver.shape, dtype=torch.float64, device=dev)
    lamN[:, 0] = 1.0
    for _ in range(args.warmup):
        UN, ck = solver.forward(U0, dts, every)
        solver.backward(lamN, dts, ck, every)
    fwd, bwd = [], []
    l0 = solver.ctx.launch_count()
    clk = ClockSampler(local)
    clk.__enter__()
    for _ in range(args.steps):
        e0, e1, e2 = (torch.cuda.Event(enable_timing=True) for _ in range(3))
        torch.cuda.synchronize()
        e0.record(s)
        UN, ck = solver.forward(U0, dts, every)
        e1.record(s)
        solver.backward(lamN, dts, ck, every)
        e2.record(s)
        e2.synchronize()
        fwd.append(e0.elapsed_time(e1))
        bwd.append(e1.elapsed_time(e2))
    clk.__exit__()
    launches = solver.ctx.launch_count() - l0
    tf, tb = float(np.mean(fwd)), float(np.mean(bwd))
    cells = n * n
    # ---- the gradient through the autograd API, and its checks
    r = rho0.clone().requires_grad_(True)
    g = G(B.GAMMA).requires_grad_(True)
    L = loss(r, g)
    L.backward()
    grad_r, grad_g = r.grad.detach(), float(g.grad)
    rng = np.random.default_rng(B.SEED)
    fd_err = {1e-7: [], 1e-8: []}
    with torch.no_grad():
        for _ in range(args.grad_checks):
            d = G(rng.standard_normal((n, n)))
            ad = float((grad_r * d).sum())
            for eps in fd_err:
                fd = (float(loss(rho0 + eps * d, G(B.GAMMA))) - float(loss(rho0 - eps * d, G(B.GAMMA)))) / (2 * eps)
                fd_err[eps].append(abs(fd - ad) / max(abs(ad), 1e-300))
        epg = 1e-7
        fdg = (float(loss(rho0, G(B.GAMMA + epg))) - float(loss(rho0, G(B.GAMMA - epg)))) / (2 * epg)
    # ---- e2e: pinned host rho0 in, gradient out, through the autograd API
    pin = torch.empty((n, n), dtype=torch.float64).pin_memory()
    pin.copy_(torch.from_numpy(prim[0, 0]))
    gout = torch.empty((n, n), dtype=torch.float64).pin_memory()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    e0.record()
    r2 = pin.to(dev, non_blocking=True).requires_grad_(True)
    g2 = G(B.GAMMA).requires_grad_(True)
    loss(r2, g2).backward()
    gout.copy_(r2.grad, non_blocking=True)
    gg2 = g2.grad.to("cpu")
    e1.record()
    e1.synchronize()
    e2e_ms = e0.elapsed_time(e1)
    # ---- dual-number oracle reference on the host cores (one density direction and gamma)
    dual = None
    if rank == 0 and not args.no_cpu_baseline:
        import oracle as O
        O.build()
        c = O.make_cfg(physics="hd", ndim=2, gamma=B.GAMMA, flux_scheme="hll", limiter="minmod", courantpar=0.8)
        w0 = B.to_cons_blocks(prim)
        mb = B.mask_blocks(n)
        drho = np.random.default_rng(5).standard_normal((n, n))
        nth = os.cpu_count() or 1
        t0 = time.perf_counter()
        Lr, dr, _ = O.dual_run(c, [n, n], [0.0, 0.0], [1.0, 1.0], ["cont"] * 4, w0,
                               B.cons_direction(prim, drho, 0.0), 0.0, dts, mb, nth)
        t_dual = time.perf_counter() - t0
        _, dgr, _ = O.dual_run(c, [n, n], [0.0, 0.0], [1.0, 1.0], ["cont"] * 4, w0,
                               B.cons_direction(prim, np.zeros((n, n)), 1.0), 1.0, dts, mb, nth)
        ad = float((grad_r.cpu().numpy() * drho).sum())
        dual = {"loss_rel_diff": abs(float(L.detach()) - Lr) / abs(Lr),
                "rho_direction_rel_err": abs(ad - dr) / abs(dr), "gamma_rel_err": abs(grad_g - dgr) / abs(dgr),
                "dual_run_s": t_dual, "cores": nth,
                "zone_updates_per_s_dual_cpu": cells * nsteps / t_dual}
    solver.close()
    peaks, peak_kind = _measured_peaks()
    if rank == 0:
        zu = cells * nsteps
        print(json.dumps({
            "metric": METRIC, "value": zu / ((tf + tb) * 1e-3), "unit": UNIT, "n_gpus": ws, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": tf + tb, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": _config(args.workload),
            "run": {"step": "one gradient: forward run of 200 steps + adjoint sweep",
                       "cells": cells, "blocks": solver.ctx.nblocks, "time_steps": nsteps,
                       "checkpoint_every": every, "l2": "no flush: 3 registers + checkpoints (%.0f MB) > 126 MB L2"
                       % ((3 + nsteps / every) * cells * 4 * 8 / 1e6)},
            "adjoint": {"forward_ms": tf, "backward_ms": tb, "adjoint_cost_vs_forward": tb / tf,
                        "forward_zone_updates_per_s": zu / (tf * 1e-3),
                        "what": "backward = segment recomputation from checkpoints keeping every stage "
                                "input + three adjoint stages per step",
                        "loss": float(L.detach()), "dL_dgamma": grad_g,
                        "fd_check": {"directions": args.grad_checks,
                                     "rel_err_by_eps": {str(e): {"median": float(np.median(v)), "max": float(np.max(v))}
                                                        for e, v in fd_err.items() if v},
                                     "gamma_eps": 1e-7, "gamma_rel_err": abs(fdg - grad_g) / abs(grad_g),
                                     "note": "central differences of the FP64 forward at frozen dt: a larger step "
                                             "crosses limiter kinks, a smaller one meets the roundoff of a loss of "
                                             "~5e4; the exact check is dual_oracle_check"},
                        "dual_oracle_check": dual},
            "roofline": None,
            "e2e": {"value": zu / (e2e_ms * 1e-3), "unit": UNIT, "h2d_bytes_per_step": float(pin.nbytes),
                    "d2h_bytes_per_step": float(gout.nbytes + 8),
                    "what": "torch autograd through the C-ABI: rho0 from pinned host, forward, loss, backward, "
                            "dL/drho0 and dL/dgamma to host"},
            "cpu_baseline": None if dual is None else {
                "value": dual["zone_updates_per_s_dual_cpu"], "unit": UNIT, "cores": dual["cores"], "kind": "port",
                "sample": "one forward-mode (dual-number) run of the oracle over all 200 steps"},
            "gpu_launches": int(launches), "clocks": clk.summary(),
        }))


# ---------------------------------------------------------------- multi-level blast (3-D MHD)
AMR_X = ([-0.5] * 3, [0.5] * 3)


def _amr_cfg_kwargs():
    return dict(physics="mhd", ndim=3, ndir=3, flux_scheme="hlld", limiter="vanleer", typedivbfix="glm",
                courantpar=0.8, gamma=5.0 / 3.0)


def _amr_blast_prim(X, Y, Z):
    r = np.sqrt(X * X + Y * Y + Z * Z)
    out = np.zeros((9,) + X.shape)
    out[0] = 1.0
    out[4] = np.where(r < 0.1, 100.0, 0.1)
    out[5] = out[6] = 1.0 / np.sqrt(2.0)
    return out


def _amr_init(tree):
    from tests import _amr as A
    return A.fill_blocks(tree.leaves, 3, tree.nbase, _amr_blast_prim, "mhd", 3, 5.0 / 3.0, *AMR_X)


AMR_WEIGHT = [0.5, 0.0, 0.0, 0.0, 0.5, 0.0, 0.0, 0.0, 0.0]  # rho and e


def _amr_tree_gpu(w):
    """settree with the device's Löhner estimator."""
    from amrvac_b200 import Context, make_cfg
    from amrvac_b200.amr import Tree, initial_hierarchy, lohner_flags
    a = w["amr"]
    ctx = Context(make_cfg(typeboundary=["cont"] * 6, **_amr_cfg_kwargs()))

    def err(tree, blocks):
        r, c, _ = lohner_flags(ctx, tree, blocks, *AMR_X, AMR_WEIGHT)
        return r, c
    tree, blocks = initial_hierarchy(Tree(3, [a["nbase"]] * 3, a["levels"], periodic=[False] * 3), _amr_init, err)
    ctx.close()
    return tree, blocks


def _amr_tree_oracle(w):
    """settree with the oracle's lohner_grid (CPU)."""
    import oracle as O
    from amrvac_b200.amr import Tree, initial_hierarchy
    a = w["amr"]
    c = _amr_oracle_cfg()
    wt = np.array(AMR_WEIGHT)
    lf = np.zeros(9, np.int32)

    def err(tree, blocks):
        g = O.AmrGrid(c, tree.nbase, *AMR_X, tree.leaves, bc=["cont"] * 6)
        for b in range(len(tree.leaves)):
            g.set_block(b, blocks[b])
        g.getbc()
        ref, coa = [], []
        for b, t in enumerate(tree.leaves):
            _, rr, cc = O.lohner_block(c, g.get_block(b), wt, lf, 1.0e-2, 0.1, 0.125, t[0], tree.max_level)
            ref.append(bool(rr))
            coa.append(bool(cc))
        return ref, coa
    return initial_hierarchy(Tree(3, [a["nbase"]] * 3, a["levels"], periodic=[False] * 3), _amr_init, err)


def _amr_oracle_cfg():
    import oracle as O
    return O.make_cfg(physics="mhd", ndim=3, ndir=3, flux_scheme="hlld", limiter="vanleer", divb="glm",
                      courantpar=0.8, gamma=5.0 / 3.0)


def _amr_cpu_sample(tree, blocks, nthreads, steps=1):
    """The oracle's multi-level step (advect1 per stage, flux fix, getbc) on
    the whole hierarchy."""
    import oracle as O
    g = O.AmrGrid(_amr_oracle_cfg(), tree.nbase, *AMR_X, tree.leaves, bc=["cont"] * 6)
    for b in range(len(tree.leaves)):
        g.set_block(b, blocks[b])
    g.getbc()
    t0 = time.perf_counter()
    for _ in range(steps):
        dt, cm = g.getdt()
        g.advance(dt, cm, nthreads)
    el = time.perf_counter() - t0
    return tree.cells() * steps / el, g


def run_amr(args, ws, rank, local):
    import torch
    if not torch.cuda.is_available():
        raise SystemExit("bench.py: no CUDA device")
    torch.cuda.set_device(local)
    from amrvac_b200 import Context, make_cfg
    wl = args.workload
    w = WORKLOADS[wl]
    t_build = time.perf_counter()
    tree, blocks = _amr_tree_gpu(w)
    t_build = time.perf_counter() - t_build
    cells = tree.cells()
    cfg = make_cfg(typeboundary=["cont"] * 6, **_amr_cfg_kwargs())
    ctx = Context(cfg)
    ctx.set_amr_grid(tree.leaves, tree.nbase, *AMR_X)
    ctx.upload(blocks)
    nw = ctx.nw
    zchunk, tune_ms = ctx.autotune(reps=3, cache=False)
    ctx.upload(blocks)
    # FP64 parity of the first step against the oracle on the same hierarchy
    parity = None
    if rank == 0 and not args.no_cpu_baseline:
        nthreads = os.cpu_count() or 1
        v_cpu, g = _amr_cpu_sample(tree, blocks, nthreads, 1)
        ctx.set_time(0.0, 1.0e99, 0.0)
        ctx.step()
        got = ctx.download()
        worst = 0.0
        for b in range(len(tree.leaves)):
            ref = g.get_block(b)[:, 2:18, 2:18, 2:18]
            d = np.abs(got[b][:, 2:18, 2:18, 2:18] - ref).max() / max(np.abs(ref).max(), 1e-300)
            worst = max(worst, float(d))
        parity = {"steps": 1, "max_rel_diff_vs_oracle": worst, "tolerance": 1e-12, "ok": worst <= 1e-12}
        ctx.upload(blocks)
    ctx.set_time(0.0, 1.0e99, 0.0)
    ctx.run_timed(max(args.warmup, 3))
    if ctx.status():
        raise SystemExit(f"bench.py: runtime status {ctx.status()} during warm-up")
    _barrier(ws)
    torch.cuda.synchronize()
    l0 = ctx.launch_count()
    with ClockSampler(local) as clk:
        total_ms, stage_ms, getdt_ms = ctx.run_timed(args.steps)
    torch.cuda.synchronize()
    _barrier(ws)
    launches = ctx.launch_count() - l0
    st = ctx.status()
    state64 = ctx.download()
    ghost_ms, fix_ms = ctx.amr_kernel_ms(10)
    timed_blocks, timed_slots = ctx.nblocks, ctx.amr_slots  # the timed tree (the regrid run changes it)
    tmax = _allmax(total_ms, ws)
    value = ws * cells * args.steps / (tmax * 1e-3)
    nstage = 3 * args.steps
    stage_kernel_s = (stage_ms / nstage - ghost_ms - fix_ms) * 1e-3
    peaks, peak_kind = _measured_peaks()
    from amrvac_b200.api import fp64_peak_tflops
    bytes_per_cell = (2 + 3 + 3) / 3.0 * 8 * nw
    achieved_gbs = bytes_per_cell * cells / stage_kernel_s / 1e9
    fp64_peak = fp64_peak_tflops()
    fl = ALG_FLOPS[wl]["stage"]
    achieved_tf = fl * cells / stage_kernel_s / 1e12
    roofline = {"bound": "fp64", "achieved": achieved_tf, "peak": fp64_peak, "unit": "TFLOP/s",
                "frac": achieved_tf / fp64_peak, "alg_flops_per_cell_stage": fl,
                "peak_source": "measured in this run: FP64 FMA chains on every SM (amrvac_gpu_fp64_peak)",
                "traffic": None, "kernel": "fv_stage_kernel", "avg_launch_ms": stage_kernel_s * 1e3,
                "launches": nstage, "why_this_bound": "FP64 flops / FP64 peak is the slower roofline for 3-D MHD",
                "amr_overhead_ms_per_stage": {"ghost_pass": ghost_ms, "flux_fix": fix_ms}}
    roofline_other = {"bound": "hbm", "achieved": achieved_gbs, "peak": peaks["hbm_gbs"], "unit": "GB/s",
                      "frac": achieved_gbs / peaks["hbm_gbs"], "peak_source": peak_kind,
                      "algorithmic_bytes_per_cell": bytes_per_cell}
    # e2e through the public API from pinned host blocks
    e2e = None
    try:
        pinned = torch.empty(blocks.shape, dtype=torch.float64).pin_memory()
        host = pinned.numpy()
        host[...] = blocks
        s = torch.cuda.ExternalStream(ctx.stream_ptr())
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        e0.record(s)
        ctx.upload(host)
        ctx.set_time(0.0, 1.0e99, 0.0)
        for _ in range(args.steps):
            ctx.step()
            ctx.get_time()
            ctx.status()
        ctx.L.amrvac_gpu_download(ctx.h, 0, 0, ctx.nblocks, host.ctypes.data_as(
            __import__("ctypes").POINTER(__import__("ctypes").c_double)))
        e1.record(s)
        e1.synchronize()
        e2e_ms = _allmax(e0.elapsed_time(e1), ws)
        e2e = {"value": ws * cells * args.steps / (e2e_ms * 1e-3), "unit": UNIT,
               "h2d_bytes_per_step": (blocks.nbytes + 32 * args.steps) / args.steps,
               "d2h_bytes_per_step": (blocks.nbytes + 28 * args.steps) / args.steps,
               "what": "C-ABI from pinned host block arrays: upload, K steps with a host round trip each, "
                       "download with ghost cells (level-jump ghosts included); transfers amortised over K"}
    except Exception as ex:
        e2e = {"value": None, "unit": UNIT, "error": str(ex)}
    # the reference's time loop with ditregrid = 1: advance, then resettree
    # (device Löhner, C++ tree decision, device remap) after every step
    regrid_run = None
    try:
        ctx.set_amr_grid(tree.leaves, tree.nbase, *AMR_X)
        ctx.upload(blocks)
        ctx.set_time(0.0, 1.0e99, 0.0)
        rkw = dict(refine_max_level=w["amr"]["levels"], refine_threshold=0.1, derefine_ratio=0.125,
                   amr_wavefilter=1.0e-2)
        for _ in range(2):
            ctx.step()
            ctx.amr_resettree(AMR_WEIGHT, **rkw)
        s = torch.cuda.ExternalStream(ctx.stream_ptr())
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        cells_done, changes, nmin, nmax = 0, 0, ctx.nblocks, ctx.nblocks
        e0.record(s)
        for _ in range(args.steps):
            cells_done += ctx.nblocks * 16 ** 3
            ctx.step()
            changes += ctx.amr_resettree(AMR_WEIGHT, **rkw)
            nmin, nmax = min(nmin, ctx.nblocks), max(nmax, ctx.nblocks)
        e1.record(s)
        e1.synchronize()
        rg_ms = _allmax(e0.elapsed_time(e1), ws)
        regrid_run = {"value": ws * cells_done / (rg_ms * 1e-3), "unit": UNIT, "ms_per_step": rg_ms / args.steps,
                      "static_ms_per_step": tmax / args.steps, "regrids_that_changed_the_tree": changes,
                      "blocks_min_max": [nmin, nmax], "status": ctx.status(),
                      "what": "K steps each followed by amrvac_gpu_amr_resettree (Löhner on the device, tree "
                              "decision in C++ on the host, remap kernel); CUDA events on the library stream, "
                              "host work included"}
    except Exception as ex:
        regrid_run = {"error": str(ex)}
    mixed = None
    try:
        cm = Context(make_cfg(precision="mixed", typeboundary=["cont"] * 6, **_amr_cfg_kwargs()))
        cm.set_amr_grid(tree.leaves, tree.nbase, *AMR_X)
        cm.upload(blocks)
        zm, _ = cm.autotune(reps=3, cache=False)
        cm.upload(blocks)
        cm.set_time(0.0, 1.0e99, 0.0)
        cm.run_timed(max(args.warmup, 3))
        _barrier(ws)
        mt, ms_stage, _ = cm.run_timed(args.steps)
        mt = _allmax(mt, ws)
        ref = state64[:, :, 2:18, 2:18, 2:18]
        got = cm.download()[:, :, 2:18, 2:18, 2:18]
        l1 = [float(np.abs(got[:, v] - ref[:, v]).sum() / max(np.abs(ref[:, v]).sum(), 1e-300))
              for v in range(ref.shape[1])]
        mixed = {"value": ws * cells * args.steps / (mt * 1e-3), "unit": UNIT, "ms_per_step": mt / args.steps,
                 "speedup_vs_fp64": total_ms / mt, "zchunk": zm, "l1_rel_err_vs_fp64_per_var": l1,
                 "status": cm.status()}
        cm.close()
    except Exception as ex:
        mixed = {"error": str(ex)}
    cpu = None
    if parity is not None:
        cpu = {"value": v_cpu, "unit": UNIT, "cores": nthreads, "kind": "port",
               "sample": "1 SSP-RK3 step of the whole hierarchy (oracle multi-level advance)"}
    if rank == 0:
        out = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": ws, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": tmax / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": _config(wl),
            "run": {"cells": cells, "blocks": timed_blocks, "nw": nw,
                       "blocks_per_level": tree.counts(), "blocks_next_to_a_level_jump": timed_slots,
                       "tree_build_s": t_build, "tile": _tile(ctx, zchunk), "autotuned_stage_ms": tune_ms,
                       "parallelism": "replicas" if ws > 1 else "single GPU",
                       "l2": "no flush: working set %.0f MB (3 registers) > 126 MB L2" % (3 * cells * nw * 8 / 1e6),
                       "stage_weighted_cell_updates_per_s": 3 * value},
            "roofline": roofline, "roofline_other": roofline_other, "cpu_baseline": cpu, "parity": parity,
            "e2e": e2e, "mixed": mixed,
            "regrid_every_step": regrid_run,
            "gpu_launches": launches, "clocks": clk.summary(), "status": st,
            "kernel_ms": {"stage_total_incl_amr": stage_ms, "getdt_total": getdt_ms, "step_total": total_ms},
        }
        print(json.dumps(out))
    ctx.close()


def _graph_steps_ms(ctx, nsteps, flush_l2):
    """Device time of nsteps steps replayed from the context's captured step
    graph (amrvac_gpu_run), CUDA events on the library stream.  With
    flush_l2, a 256 MB write (outside the timed intervals) precedes every step."""
    import torch
    s = torch.cuda.ExternalStream(ctx.stream_ptr())
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    if not flush_l2:
        torch.cuda.synchronize()
        e0.record(s)
        ctx.run(nsteps)
        e1.record(s)
        e1.synchronize()
        return e0.elapsed_time(e1)
    buf = torch.empty(256 << 20, dtype=torch.uint8, device="cuda")
    tot = 0.0
    for _ in range(nsteps):
        with torch.cuda.stream(s):
            buf.fill_(1)
        e0.record(s)
        ctx.run(1)
        e1.record(s)
        e1.synchronize()
        tot += e0.elapsed_time(e1)
    return tot


def _ot256_line(args, peaks, fp64_peak):
    """OT-3D at 256^3 (4096 blocks, FP64): K graph-replayed steps after the
    autotuner and the warm-up, the average stage launch and its FP64 and HBM
    roofline fractions (the working set, 3.6 GB, is far above L2)."""
    from amrvac_b200 import Context, make_cfg
    wl = "ot256"
    w = WORKLOADS[wl]
    blocks, geo = _initial_blocks(wl)
    c = Context(make_cfg(**_cfg_kwargs(wl)))
    try:
        c.set_uniform_grid(geo["domain_nx"], geo["xprobmin"], geo["xprobmax"])
        c.upload(blocks)
        del blocks
        cells = w["n"] ** w["ndim"]
        z, tune_ms = c.autotune(reps=3, cache=False)
        c.set_time(0.0, 1.0e99, 0.0)
        c.run(max(args.warmup, 3))
        c.run_timed(1)
        t = _graph_steps_ms(c, args.steps, False)
        _, stage_ms, _ = c.run_timed(args.steps)
        stage_s = stage_ms * 1e-3 / (3 * args.steps)
        bytes_per_cell = (2 + 3 + 3) / 3.0 * 8 * c.nw
        fl = ALG_FLOPS[wl]["stage"]
        return {"value": cells * args.steps / (t * 1e-3), "unit": UNIT, "ms_per_step": t / args.steps,
                "stage_avg_ms": stage_s * 1e3, "tile": dict(_tile(c, z), autotuned_stage_ms=tune_ms),
                "roofline_fp64_frac": fl * cells / stage_s / 1e12 / fp64_peak,
                "roofline_hbm_frac": bytes_per_cell * cells / stage_s / 1e9 / peaks["hbm_gbs"],
                "status": c.status(),
                "what": "FP64, K steps replayed from the step graph; fractions of the stage kernel's average "
                        "launch as in the main roofline key"}
    finally:
        c.close()


def run_ours(args, ws, rank, local):
    import torch
    if not torch.cuda.is_available():
        raise SystemExit("bench.py: no CUDA device")
    torch.cuda.set_device(local)
    from amrvac_b200 import Context, make_cfg
    from amrvac_b200.api import fp64_peak_tflops
    wl = args.workload
    w = WORKLOADS[wl]
    blocks, geo = _initial_blocks(wl)
    cfg = make_cfg(**_cfg_kwargs(wl))
    ctx = Context(cfg)
    ctx.set_uniform_grid(geo["domain_nx"], geo["xprobmin"], geo["xprobmax"])
    ctx.upload(blocks)
    cells = w["n"] ** w["ndim"]
    nw = ctx.nw
    flush = 3 * cells * nw * 8 < 126e6
    zchunk, tune_ms = ctx.autotune(reps=3, cache=False)
    ctx.upload(blocks)
    ctx.set_time(0.0, 1.0e99, 0.0)
    # warm-up: the captured step graph (instantiated here) and the direct launches
    ctx.run(max(args.warmup, 3))
    ctx.run_timed(1)
    torch.cuda.synchronize()
    if ctx.status():
        raise SystemExit(f"bench.py: runtime status {ctx.status()} during warm-up")
    # ---------------- timed region: K steps replayed from the step graph
    _barrier(ws)
    torch.cuda.synchronize()
    l0 = ctx.launch_count()
    with ClockSampler(local) as clk:
        total_ms = _graph_steps_ms(ctx, args.steps, flush)
    launches = ctx.launch_count() - l0
    _barrier(ws)
    tmax = _allmax(total_ms, ws)
    value = ws * cells * args.steps / (tmax * 1e-3)
    # ---------------- per-kernel split of K more steps (events around every kernel)
    t_direct, stage_ms, getdt_ms = ctx.run_timed(args.steps)
    st = ctx.status()
    state64 = ctx.download()  # after warm-up + 2K steps: the reference state for the mixed form
    nstage = 3 * args.steps
    stage_avg_s = stage_ms * 1e-3 / nstage
    peaks, peak_kind = _measured_peaks()
    # algorithmic bytes of one stage launch: read wCT, read the RK base
    # (stages 2 and 3), write wnew -> (2 + 3 + 3) / 3 * 8 * nw per cell on average
    bytes_per_cell = (2 + 3 + 3) / 3.0 * 8 * nw
    achieved_gbs = bytes_per_cell * cells / stage_avg_s / 1e9
    fp64_peak = fp64_peak_tflops()
    fl = ALG_FLOPS[wl]["stage"]
    achieved_tf = fl * cells / stage_avg_s / 1e12
    t_hbm = bytes_per_cell * cells / (peaks["hbm_gbs"] * 1e9)
    t_fp64 = fl * cells / (fp64_peak * 1e12)
    traffic = NCU_TRAFFIC_PER_CELL.get(wl)
    traffic_note = (None if traffic is None else
                    "DRAM read+write of one stage-1 launch (algorithmic 2*8*nw B/cell for that launch) from the "
                    "committed ncu capture profiles/fv_stage_ot128_fp64_mixed.md, scaled per cell; not measured in "
                    "this run")
    hbm = {"bound": "hbm", "achieved": achieved_gbs, "peak": peaks["hbm_gbs"], "unit": "GB/s",
           "frac": achieved_gbs / peaks["hbm_gbs"], "peak_source": peak_kind + " (MEASURED_PEAKS.json hbm_gbs)",
           "algorithmic_bytes_per_cell": bytes_per_cell}
    f64 = {"bound": "fp64", "achieved": achieved_tf, "peak": fp64_peak, "unit": "TFLOP/s",
           "frac": achieved_tf / fp64_peak,
           "peak_source": "measured in this run: FP64 FMA chains on every SM (amrvac_gpu_fp64_peak); "
                          "MEASURED_PEAKS.json has no FP64 figure",
           "alg_flops_per_cell_stage": fl}
    binding = f64 if t_fp64 >= t_hbm else hbm
    other = hbm if binding is f64 else f64
    roofline = dict(binding)
    roofline.update({"traffic": None if traffic is None else traffic * cells, "traffic_note": traffic_note,
                     "kernel": "fv_stage_kernel", "avg_launch_ms": stage_avg_s * 1e3, "launches": nstage,
                     "why_this_bound": "the slower of algorithmic bytes / HBM peak (%.3f ms) and algorithmic "
                                       "FP64 flops / FP64 peak (%.3f ms) per stage launch" % (t_hbm * 1e3,
                                                                                            t_fp64 * 1e3)})
    # ---------------- e2e through the public API with host buffers
    e2e = None
    try:
        pinned = torch.empty(blocks.shape, dtype=torch.float64).pin_memory()
        host = pinned.numpy()
        host[...] = blocks
        s = torch.cuda.ExternalStream(ctx.stream_ptr())
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        e0.record(s)
        ctx.upload(host)
        ctx.set_time(0.0, 1.0e99, 0.0)
        for _ in range(args.steps):
            ctx.step()
            ctx.get_time()          # per-step D2H: dt, cmax_global, time
            ctx.status()            # per-step D2H: status word
        ctx.L.amrvac_gpu_download(ctx.h, 0, 0, ctx.nblocks, host.ctypes.data_as(
            __import__("ctypes").POINTER(__import__("ctypes").c_double)))
        e1.record(s)
        e1.synchronize()
        e2e_ms = _allmax(e0.elapsed_time(e1), ws)
        state_bytes = blocks.nbytes
        e2e = {"value": ws * cells * args.steps / (e2e_ms * 1e-3), "unit": UNIT,
               "h2d_bytes_per_step": (state_bytes + 32 * args.steps) / args.steps,
               "d2h_bytes_per_step": (state_bytes + 28 * args.steps) / args.steps,
               "what": "C-ABI from pinned host Fortran block arrays: upload of the initial state, K steps each "
                       "with a host round trip (set_time in, dt/cmax/time/status out), download of the final "
                       "state with ghost cells; state transfers amortised over K"}
    except Exception as ex:  # report, do not hide
        e2e = {"value": None, "unit": UNIT, "error": str(ex)}
    # ---------------- mixed form on the same workload, same timing
    mixed = None
    try:
        cm = Context(make_cfg(precision="mixed", **_cfg_kwargs(wl)))
        cm.set_uniform_grid(geo["domain_nx"], geo["xprobmin"], geo["xprobmax"])
        cm.upload(blocks)
        zm, _ = cm.autotune(reps=3, cache=False)
        cm.upload(blocks)
        cm.set_time(0.0, 1.0e99, 0.0)
        cm.run(max(args.warmup, 3))
        cm.run_timed(1)
        _barrier(ws)
        mt = _allmax(_graph_steps_ms(cm, args.steps, flush), ws)
        _, ms_stage, _ = cm.run_timed(args.steps)
        ref = _interior(state64, w["ndim"])
        got = _interior(cm.download(), w["ndim"])
        l1 = [float(np.abs(got[:, v] - ref[:, v]).sum() / max(np.abs(ref[:, v]).sum(), 1e-300))
              for v in range(ref.shape[1])]
        mixed = {"value": ws * cells * args.steps / (mt * 1e-3), "unit": UNIT, "ms_per_step": mt / args.steps,
                 "speedup_vs_fp64": tmax / mt, "tile": _tile(cm, zm), "stage_avg_ms": ms_stage / nstage,
                 "l1_rel_err_vs_fp64_per_var": l1,
                 "l1_note": "L1 of the mixed state against the FP64 GPU state after the same warm-up + 2K steps "
                            "from the same initial state; the FP64 path itself is checked against the oracle "
                            "(parity key)", "status": cm.status()}
        cm.close()
    except Exception as ex:
        mixed = {"error": str(ex)}
    # ---------------- the 256^3 variant of the workload (FP64), where the
    # north-star roofline target is stated: same timing, no parity or CPU leg
    ot256 = None
    if wl == "ot128" and ws == 1 and not args.no_ot256:
        try:
            ot256 = _ot256_line(args, peaks, fp64_peak)
        except Exception as ex:  # report, do not hide
            ot256 = {"error": str(ex)}
    # ---------------- parity of the first step and the CPU baseline (oracle, full grid)
    cpu, parity = None, None
    if rank == 0 and ws == 1 and not args.no_cpu_baseline:
        nthreads = os.cpu_count() or 1
        ctx.upload(blocks)
        ctx.set_time(0.0, 1.0e99, 0.0)
        ctx.step()
        parity, t_cpu = _parity_first_step(wl, blocks, geo, ctx.download(), nthreads)
        cpu = {"value": cells / t_cpu, "unit": UNIT, "cores": nthreads, "kind": "port",
               "sample": f"1 full SSP-RK3 step (setdt + 3 stages) of the whole {w['n']}^{w['ndim']} grid from the "
                         f"initial state, oracle (C++ restatement, OpenMP)"}
    if rank == 0:
        out = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": ws, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": tmax / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": _config(wl),
            "execution": ("replicas, one per GPU" if ws > 1 else "single GPU") + "; the K timed steps are "
                         "replays of the captured step graph",
            "tile": dict(_tile(ctx, zchunk), autotuned_stage_ms=tune_ms),
            "stage_weighted_cell_updates_per_s": 3 * value,
            "roofline": roofline, "roofline_other": other, "parity": parity, "cpu_baseline": cpu, "e2e": e2e,
            "mixed": mixed, "ot256": ot256, "gpu_launches": launches, "clocks": clk.summary(), "status": st,
            "kernel_ms": {"stage_total": stage_ms, "getdt_total": getdt_ms, "steps_direct_total": t_direct,
                          "note": "per-kernel CUDA events over K further steps launched directly"},
        }
        print(json.dumps(out))
    ctx.close()


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="ot128", choices=sorted(WORKLOADS))
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-ot256", action="store_true",
                    help="default workload: skip the extra 256^3 measurement")
    ap.add_argument("--grad-checks", type=int, default=64,
                    help="adjoint workload: seeded directions of the central-difference check")
    ap.add_argument("--it-max", type=int, default=None,
                    help="ensemble workloads: stop every instance after this many steps (the reference's it_max)")
    args = ap.parse_args()
    args.warmup = max(args.warmup, 3)
    ws, rank, local = _dist_init()
    try:
        if args.impl == "reference":
            run_reference(args, ws, rank)
        elif "ensemble" in WORKLOADS[args.workload]:
            run_ensemble(args, ws, rank, local)
        elif "adjoint" in WORKLOADS[args.workload]:
            run_adjoint(args, ws, rank, local)
        elif "amr" in WORKLOADS[args.workload]:
            run_amr(args, ws, rank, local)
        else:
            run_ours(args, ws, rank, local)
    finally:
        if ws > 1:
            import torch.distributed as dist
            dist.destroy_process_group()


if __name__ == "__main__":
    main()
