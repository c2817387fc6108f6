"""Thin torch.autograd wrapper of the device adjoint (tmb_adjoint_rk4), for tests and studies.

``LLGObjective(ctx, ...)`` holds a configured Context (mesh, BEM, material, DMI form) and the run
(initial state, steps, substeps, checkpoint interval, objective weights); ``objective(ku, bz)``
returns J = sum(w * m_final) as a 0-d tensor whose backward gives dJ/dKu (per node, J/m^3) and
dJ/dBz (per pulse sample, T) from one forward sweep plus one checkpointed backward sweep.  The
parameters may be FP32 (the gradients come back in the parameters' dtype); the library computes
in FP64 vectors either way.  No tetmag counterpart (tetmag has no adjoint).
"""
from __future__ import annotations

import numpy as np
import torch


class LLGObjective:
    def __init__(self, ctx, Js, A, ku_axis, D, alpha, m0, w, nsteps, dt_ps, nsub=1, ckpt_every=10, t0_ps=0.0,
                 bz_t0=0.0, bz_t1=None):
        self.ctx = ctx
        self.Js, self.A, self.axis, self.D, self.alpha = Js, A, ku_axis, D, alpha
        self.m0 = np.ascontiguousarray(m0, dtype=np.float64)
        self.w = np.ascontiguousarray(w, dtype=np.float64)
        self.nsteps, self.dt_ps, self.nsub, self.ckpt = int(nsteps), float(dt_ps), int(nsub), int(ckpt_every)
        self.t0_ps = float(t0_ps)
        self.bz_t0 = float(bz_t0)
        self.bz_t1 = float(self.t0_ps + self.nsteps * self.dt_ps if bz_t1 is None else bz_t1)
        self.last = None

    def _configure(self, ku: np.ndarray, bz: np.ndarray):
        self.ctx.set_material(self.Js, self.A, Ku=ku, ku_axis=self.axis, D=self.D, alpha=self.alpha)
        self.ctx.set_bz_pulse(bz, self.bz_t0, self.bz_t1)

    def forward_only(self, ku, bz) -> float:
        """J without the adjoint (the map the gradient differentiates): tmb_step_rk4."""
        self._configure(np.asarray(ku, np.float64), np.asarray(bz, np.float64))
        m = self.m0.copy()
        self.ctx.step_rk4(m, self.nsteps, self.dt_ps, self.nsub, self.t0_ps)
        return float(np.sum(self.w * m))

    def run(self, ku: np.ndarray, bz: np.ndarray) -> dict:
        self._configure(ku, bz)
        self.last = self.ctx.adjoint_rk4(self.m0, self.w, self.nsteps, self.dt_ps, self.nsub, self.ckpt, self.t0_ps,
                                         n_bz=bz.size)
        return self.last

    def objective(self, ku: torch.Tensor, bz: torch.Tensor) -> torch.Tensor:
        return _AdjointFn.apply(ku, bz, self)


class _AdjointFn(torch.autograd.Function):
    @staticmethod
    def forward(fctx, ku, bz, prob: LLGObjective):
        r = prob.run(ku.detach().double().cpu().numpy().copy(), bz.detach().double().cpu().numpy().copy())
        fctx.save_for_backward(torch.as_tensor(r["grad_ku"], dtype=ku.dtype, device=ku.device),
                               torch.as_tensor(r["grad_bz"], dtype=bz.dtype, device=bz.device))
        return torch.tensor(r["J"], dtype=torch.float64, device=ku.device)

    @staticmethod
    def backward(fctx, gJ):
        gku, gbz = fctx.saved_tensors
        return gJ.to(gku.dtype) * gku, gJ.to(gbz.dtype) * gbz, None
