"""torch.autograd.Function wrappers of a solver rollout: the forward is the
GPU step (ippi_adjoint_forward, checkpointed), the backward the hand-written
adjoint (ippi_adjoint_backward).  torch only carries the tensors; every
derivative comes from the library.

    rollout = Rollout(lattice, reset, nsteps, t0, ckpt_every)
    forces, macros = TauFieldRollout.apply(tau, rollout)   # tau [ny][nx] float64
    forces, macros = NetworkRollout.apply(w, rollout)      # w [1313] float32
    loss = f(forces, macros); loss.backward()

forces is [nsteps][nbody][2] (body force of every step), macros [3][ny][nx]
(rho, ux, uy of the last step's post-stream state).  `reset(lattice)` puts
the lattice in the rollout's initial state before every forward pass (the
gradient treats that state as fixed).
"""
from __future__ import annotations

import numpy as np
import torch

from . import _lib as L


class Rollout:
    def __init__(self, lattice, reset, nsteps, t0=1, ckpt_every=64, stats=None):
        self.lat = lattice
        self.reset = reset
        self.nsteps = nsteps
        self.t0 = t0
        self.ckpt = ckpt_every
        self.stats = stats  # feature statistics of the network (NetworkRollout)

    def run(self):
        lat = self.lat
        lat.adjoint_forward(self.nsteps, self.t0, self.ckpt)
        forces = lat.force_history(self.nsteps)
        macros = np.stack([lat.download(k) for k in (L.FIELD_RHO, L.FIELD_UX, L.FIELD_UY)])
        return torch.from_numpy(np.ascontiguousarray(forces)), torch.from_numpy(macros)

    def grads(self, g_forces, g_macros, **which):
        dF = None if g_forces is None else g_forces.detach().cpu().double().numpy()
        dM = None if g_macros is None else g_macros.detach().cpu().double().numpy()
        return self.lat.adjoint_backward(dl_dforce=dF, dl_dmacro=dM, **which)


class TauFieldRollout(torch.autograd.Function):
    """(tau field, Rollout) -> (forces, macros); gradient with respect to tau."""

    @staticmethod
    def forward(ctx, tau, rollout):
        rollout.reset(rollout.lat)
        rollout.lat.set_tau_field(tau.detach().cpu().double().numpy())
        ctx.rollout = rollout
        return rollout.run()

    @staticmethod
    def backward(ctx, g_forces, g_macros):
        g = ctx.rollout.grads(g_forces, g_macros, tau=True)
        return torch.from_numpy(g["tau"]), None


class NetworkRollout(torch.autograd.Function):
    """(network weights, Rollout) -> (forces, macros); gradient with respect
    to the FP32 weights (used as given, no BF16 rounding)."""

    @staticmethod
    def forward(ctx, w, rollout):
        rollout.reset(rollout.lat)
        rollout.lat.load_tau_mlp_f32(w.detach().cpu().float().numpy(), rollout.stats)
        ctx.rollout = rollout
        ctx.dtype = w.dtype
        return rollout.run()

    @staticmethod
    def backward(ctx, g_forces, g_macros):
        g = ctx.rollout.grads(g_forces, g_macros, mlp=True)
        return torch.from_numpy(g["mlp"]).to(ctx.dtype), None
