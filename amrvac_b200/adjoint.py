"""Differentiable runs of the finite-volume path (discrete adjoint).

``solve(U0, gamma, dts, ...)`` advances the block state U0 (a CUDA float64
tensor in register layout (nblocks, nw, 16, 16)) by len(dts) steps of the
configured scheme at the given, frozen time steps, and is differentiable in
U0 and gamma through a ``torch.autograd.Function`` whose backward runs the
library's hand-written adjoint kernels (``amrvac_gpu_adjoint_step``).  The
forward keeps a checkpoint every ``checkpoint_every`` steps; the backward
recomputes each segment from its checkpoint and walks it in reverse.

The time steps are inputs, not functions of the state: ``cfl_dts`` records
the CFL sequence of one forward run (setdt, src/mod_dt.t:10-99), and the
gradient is that of the scheme at those steps.  Scope of the adjoint: 2-D
hydrodynamics, HLL with minmod or vanleer, Einfeldt bounds, FP64, periodic
or cont boundaries, uniform blocks.

PyTorch is the device-memory and autograd plumbing here; all arithmetic of
the forward and adjoint steps runs in the library's CUDA kernels.
"""
from __future__ import annotations

import ctypes

import numpy as np

from . import _lib
from .api import Context
from .config import make_cfg


def _ptr(t):
    return ctypes.c_void_p(t.data_ptr())


class FrozenDtSolver:
    """One context for a fixed configuration and gamma: forward steps at given
    dt, checkpoints, and the reverse sweep."""

    def __init__(self, domain_nx, xprobmin, xprobmax, gamma, **cfg_kw):
        import torch
        self.torch = torch
        kw = dict(physics="hd", ndim=2, flux_scheme="hll", limiter="minmod")
        kw.update(cfg_kw)
        self.cfg = make_cfg(gamma=float(gamma), **kw)
        self.ctx = Context(self.cfg)
        self.ctx.set_uniform_grid(domain_nx, xprobmin, xprobmax)
        self.shape = (self.ctx.nblocks, self.ctx.nw) + (16,) * self.cfg.ndim
        self.L = self.ctx.L
        self._grid = (domain_nx, xprobmin, xprobmax)
        self._rctx = None

    def close(self):
        if self._rctx is not None:
            self._rctx.close()
            self._rctx = None
        self.ctx.close()

    def _sync_torch(self):
        self.torch.cuda.current_stream().synchronize()

    def _stream(self, ctx=None):
        return self.torch.cuda.ExternalStream((ctx or self.ctx).stream_ptr())

    def _after_torch(self, *ctxs):
        """Order the library streams after the work torch has queued so far
        (the tensors handed to them were made on torch's stream)."""
        ev = self.torch.cuda.Event()
        ev.record(self.torch.cuda.current_stream())
        for c in ctxs:
            self._stream(c).wait_event(ev)

    def _load(self, U, reg=0):
        self._sync_torch()
        _lib.check(self.L.amrvac_gpu_register_copy(self.ctx.h, reg, _ptr(U), 1), "register_copy")

    def _store(self, U, reg=0):
        _lib.check(self.L.amrvac_gpu_register_copy(self.ctx.h, reg, _ptr(U), 0), "register_copy")
        self.ctx.synchronize()

    def _recompute_ctx(self):
        """A second context of the same configuration and grid, whose stream
        recomputes the next segment while the adjoint sweep runs on the
        first one's."""
        if self._rctx is None:
            self._rctx = Context(self.cfg)
            self._rctx.set_uniform_grid(*self._grid)
        return self._rctx

    def cfl_dts(self, U0, nsteps):
        """The dt sequence of a forward run with setdt every step."""
        self._load(U0.contiguous())
        self.ctx.set_time(0.0, 1.0e99, 0.0)
        out = []
        for _ in range(nsteps):
            self.ctx.step()
            out.append(self.ctx.get_time()[0])
        return np.array(out)

    def _nstages(self):
        return 3 if self.cfg.time_stepper == _lib.TIME_STEPPER["threestep"] else 2

    def _step_states(self, ctx, dt, u0, seg_q, unew):
        """One step from u0 that writes its stage inputs U1, U2 into seg_q[1],
        seg_q[2] and U^{n+1} into unew (a pointer; None skips the last
        stage), on ctx's stream with no copies (amrvac_gpu_step_dt_states)."""
        u2 = _ptr(seg_q[2]) if seg_q.shape[0] == 3 else None
        _lib.check(self.L.amrvac_gpu_step_dt_states(ctx.h, float(dt), u0, _ptr(seg_q[1]), u2, unew),
                   "step_dt_states")

    def forward(self, U0, dts, checkpoint_every=20, keep_last=True):
        """U_N and the checkpoints {step: U^step}.  With keep_last, the last
        segment, the first one the backward walks, also keeps every stage
        input (ckpt["last"] = (first step, [step][stage] states); the
        segment's first U^n is its checkpoint), so the backward recomputes
        only the segments before it; a forward that no backward follows
        passes keep_last=False and keeps no stage input."""
        torch = self.torch
        U0 = U0.contiguous()
        ckpt = {0: U0.clone()}
        self._load(U0)
        N = len(dts)
        s_last = ((N - 1) // checkpoint_every) * checkpoint_every if N else 0
        reg0 = ctypes.c_void_p(self.ctx.register_ptr(0))
        seg = None
        for n, dt in enumerate(dts):
            if n > 0 and n % checkpoint_every == 0:
                c = torch.empty(self.shape, dtype=torch.float64, device=U0.device)
                # stream-ordered copy: the checkpoints are only read after
                # the synchronisation at the end of the sweep
                _lib.check(self.L.amrvac_gpu_register_copy(self.ctx.h, 0, _ptr(c), 0), "register_copy")
                ckpt[n] = c
            if keep_last and n >= s_last:
                if seg is None:
                    seg = torch.empty((checkpoint_every, self._nstages()) + self.shape, dtype=torch.float64,
                                      device=U0.device)
                    self._after_torch(self.ctx)
                q = n - s_last
                # U^n: register 0 for the segment's first step, else the row
                # the previous step wrote; U^{n+1} into the next row, or into
                # register 0 after the run's last step
                u0 = reg0 if q == 0 else _ptr(seg[q, 0])
                unew = _ptr(seg[q + 1, 0]) if n + 1 < N and q + 1 < checkpoint_every else reg0
                self._step_states(self.ctx, dt, u0, seg[q], unew)
            else:
                _lib.check(self.L.amrvac_gpu_step_dt(self.ctx.h, float(dt)), "step_dt")
        UN = torch.empty(self.shape, dtype=torch.float64, device=U0.device)
        self._store(UN)
        if seg is not None:
            ckpt["last"] = (s_last, seg)
        return UN, ckpt

    def backward(self, lamN, dts, ckpt, checkpoint_every=20):
        """dL/dU0 and dL/dgamma from dL/dU_N.

        The segments are walked from the last one.  Each segment's stage
        inputs are recomputed from its checkpoint on a second context's
        stream into one of two segment buffers while the adjoint sweep of the
        segment after it runs on the first context's stream: CUDA events
        order a sweep after its segment's recomputation, and a recomputation
        after the sweep that last read its buffer.  The backward therefore
        holds two segment buffers (the forward's kept one among them)."""
        torch = self.torch
        lam = lamN.contiguous().clone()
        gpart = torch.zeros(self.ctx.nblocks, dtype=torch.float64, device=lam.device)
        N = len(dts)
        starts = sorted((k for k in ckpt if isinstance(k, int)), reverse=True)
        nst = self._nstages()
        h = self.ctx.h
        kept = ckpt.pop("last", None)
        rc = self._recompute_ctx() if len(starts) > 1 or kept is None else None
        sa = self._stream()
        sr = self._stream(rc) if rc is not None else None
        self._after_torch(*([self.ctx, rc] if rc is not None else [self.ctx]))
        shape = (checkpoint_every, nst) + self.shape
        use_kept = kept is not None and kept[0] == starts[0] and kept[1].shape[:2] == (checkpoint_every, nst)
        bufs = [kept[1] if use_kept else None, None]
        rec_done = [None] * len(starts)
        adj_done = [None] * len(starts)

        def seg_of(i):
            if bufs[i % 2] is None:
                bufs[i % 2] = torch.empty(shape, dtype=torch.float64, device=lam.device)
                self._after_torch(self.ctx, *([rc] if rc is not None else []))
            return bufs[i % 2]

        def recompute(i):
            s0 = starts[i]
            s1 = min(s0 + checkpoint_every, N)
            seg = seg_of(i)
            if i >= 2:  # the sweep that last read this buffer
                sr.wait_event(adj_done[i - 2])
            for n in range(s0, s1):
                q = n - s0
                u0 = _ptr(ckpt[s0]) if q == 0 else _ptr(seg[q, 0])
                # U^{s1} is the next checkpoint: the segment's last stage is not needed
                unew = _ptr(seg[q + 1, 0]) if n + 1 < s1 else None
                self._step_states(rc, dts[n], u0, seg[q], unew)
            rec_done[i] = torch.cuda.Event()
            rec_done[i].record(sr)

        first_kept = bufs[0] is not None
        if not first_kept:
            recompute(0)
        if len(starts) > 1:
            recompute(1)
        for i, s0 in enumerate(starts):
            s1 = min(s0 + checkpoint_every, N)
            seg = bufs[i % 2]
            if rec_done[i] is not None:
                sa.wait_event(rec_done[i])
            for n in range(s1 - 1, s0 - 1, -1):
                q = n - s0
                u0 = _ptr(ckpt[s0]) if q == 0 else _ptr(seg[q, 0])
                u2 = _ptr(seg[q, 2]) if nst == 3 else None
                _lib.check(self.L.amrvac_gpu_adjoint_step_states(h, u0, _ptr(seg[q, 1]), u2, _ptr(lam),
                                                                 float(dts[n]), _ptr(gpart)), "adjoint_step_states")
            adj_done[i] = torch.cuda.Event()
            adj_done[i].record(sa)
            if i + 2 < len(starts):
                recompute(i + 2)
        self.ctx.synchronize()
        return lam, gpart.sum()


class _Solve:
    """Factory of the autograd Function (torch imported lazily)."""

    fn = None

    @classmethod
    def get(cls):
        if cls.fn is None:
            import torch

            class Solve(torch.autograd.Function):
                @staticmethod
                def forward(ctx, U0, gamma, dts, grid, checkpoint_every, cfg_kw, grad_on):
                    solver = FrozenDtSolver(*grid, float(gamma), **cfg_kw)
                    want = grad_on and any(ctx.needs_input_grad[:2])
                    UN, ckpt = solver.forward(U0.detach(), dts, checkpoint_every, keep_last=want)
                    if not want:
                        solver.close()  # no backward will come: release the context now
                        return UN
                    ctx.solver = solver
                    ctx.ckpt = ckpt
                    ctx.dts = dts
                    ctx.k = checkpoint_every
                    return UN

                @staticmethod
                def backward(ctx, gUN):
                    lam0, gg = ctx.solver.backward(gUN.detach(), ctx.dts, ctx.ckpt, ctx.k)
                    ctx.solver.close()
                    ctx.ckpt = None
                    return lam0, gg.reshape(()), None, None, None, None, None

            cls.fn = Solve
        return cls.fn


def solve(U0, gamma, dts, domain_nx, xprobmin, xprobmax, checkpoint_every=20, **cfg_kw):
    """U_N from U0 after len(dts) steps at the frozen dts; differentiable in U0
    and gamma (a 0-d float64 tensor)."""
    import torch
    grid = (tuple(domain_nx), tuple(xprobmin), tuple(xprobmax))
    return _Solve.get().apply(U0, gamma, np.asarray(dts, np.float64), grid, int(checkpoint_every), cfg_kw,
                              torch.is_grad_enabled())


def domain_to_blocks(u, bn=16):
    """(nw, ny, nx) -> (nblocks, nw, bn, bn), blocks x-fastest (torch, differentiable)."""
    nw, ny, nx = u.shape
    return (u.reshape(nw, ny // bn, bn, nx // bn, bn).permute(1, 3, 0, 2, 4)
            .reshape((ny // bn) * (nx // bn), nw, bn, bn))


def blocks_to_domain(b, ny, nx, bn=16):
    nb, nw = b.shape[:2]
    return (b.reshape(ny // bn, nx // bn, nw, bn, bn).permute(2, 0, 3, 1, 4).reshape(nw, ny, nx))
