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

    def close(self):
        self.ctx.close()

    def _sync_torch(self):
        self.torch.cuda.current_stream().synchronize()

    def _load(self, U, reg=0):
        self._sync_torch()
        _lib.check(self.L.amrvac_gpu_register_copy(self.ctx.h, reg, _ptr(U), 1), "register_copy")

    def _store(self, U, reg=0):
        _lib.check(self.L.amrvac_gpu_register_copy(self.ctx.h, reg, _ptr(U), 0), "register_copy")
        self.ctx.synchronize()

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

    def _step_keeping(self, seg_q, dt):
        """One step that leaves its stage inputs in seg_q[0..nst-1]: U^n
        before the step, U1 and U2 left in registers 1 and 2 by it."""
        h = self.ctx.h
        _lib.check(self.L.amrvac_gpu_register_copy(h, 0, _ptr(seg_q[0]), 0), "register_copy")
        _lib.check(self.L.amrvac_gpu_step_dt(h, float(dt)), "step_dt")
        for st in range(1, seg_q.shape[0]):
            _lib.check(self.L.amrvac_gpu_register_copy(h, st, _ptr(seg_q[st]), 0), "register_copy")

    def forward(self, U0, dts, checkpoint_every=20, keep_last=True):
        """U_N and the checkpoints {step: U^step}.  With keep_last, the last
        segment, the first one the backward walks, also keeps every stage
        input (ckpt["last"] = (first step, [step][stage] states)), so the
        backward recomputes only the segments before it; a forward that no
        backward follows passes keep_last=False and copies no stage input."""
        torch = self.torch
        U0 = U0.contiguous()
        self._load(U0)
        ckpt = {0: U0.clone()}
        N = len(dts)
        s_last = ((N - 1) // checkpoint_every) * checkpoint_every if N else 0
        seg = None
        for n, dt in enumerate(dts):
            if n > 0 and n % checkpoint_every == 0:
                c = torch.empty(self.shape, dtype=torch.float64, device=U0.device)
                self._store(c)
                ckpt[n] = c
            if keep_last and n >= s_last:
                if seg is None:
                    seg = torch.empty((checkpoint_every, self._nstages()) + self.shape, dtype=torch.float64,
                                      device=U0.device)
                self._step_keeping(seg[n - s_last], dt)
            else:
                _lib.check(self.L.amrvac_gpu_step_dt(self.ctx.h, float(dt)), "step_dt")
        UN = torch.empty(self.shape, dtype=torch.float64, device=U0.device)
        self._store(UN)
        if seg is not None:
            ckpt["last"] = (s_last, seg)
        return UN, ckpt

    def backward(self, lamN, dts, ckpt, checkpoint_every=20):
        """dL/dU0 and dL/dgamma from dL/dU_N."""
        torch = self.torch
        lam = lamN.contiguous().clone()
        gpart = torch.zeros(self.ctx.nblocks, dtype=torch.float64, device=lam.device)
        N = len(dts)
        starts = sorted(k for k in ckpt if isinstance(k, int))
        nst = self._nstages()
        h = self.ctx.h
        kept = ckpt.pop("last", None)
        seg = None
        for s0 in reversed(starts):
            s1 = min(s0 + checkpoint_every, N)
            if kept is not None and kept[0] == s0 and kept[1].shape[0] == checkpoint_every:
                seg = kept[1]  # the forward kept this segment's stage inputs
            else:
                if seg is None:
                    # stage inputs of one segment: [step][stage]; after the
                    # kept segment has been walked its buffer is reused, so the
                    # backward holds one segment buffer at a time
                    seg = torch.empty((checkpoint_every, nst) + self.shape, dtype=torch.float64, device=lam.device)
                # recompute the segment from its checkpoint, keeping every stage input
                self._load(ckpt[s0])
                for n in range(s0, s1):
                    self._step_keeping(seg[n - s0], dts[n])
            for n in range(s1 - 1, s0 - 1, -1):
                q = n - s0
                u2 = _ptr(seg[q, 2]) if nst == 3 else None
                _lib.check(self.L.amrvac_gpu_adjoint_step_states(h, _ptr(seg[q, 0]), _ptr(seg[q, 1]), u2, _ptr(lam),
                                                                 float(dts[n]), _ptr(gpart)), "adjoint_step_states")
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
