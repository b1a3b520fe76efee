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

The same Functions written in C++ against libtorch (torch_ext/ippi_autograd.cpp,
torch::autograd::Function) are loaded by native():

    ext = native()
    roll = ext.tau_field_rollout(lattice.handle.value, nsteps, t0, ckpt_every, base_tau)
    forces, macros = roll(tau)          # differentiable in tau
    roll = ext.network_rollout(lattice.handle.value, nx, ny, nsteps, t0, ckpt_every, base_w, stats)
    forces, macros = roll(w)            # differentiable in w

where the starting state is the lattice's state when the rollout is made and
base_tau / base_w the parameters in force then.
"""
from __future__ import annotations

import importlib.util
import os

import numpy as np
import torch

from . import _lib as L

NATIVE_SO = os.path.join(L.PKG_DIR, "torch_ext", "_build", "ippi_autograd.so")
_native = None


def native():
    """The libtorch extension (built in-tree by build.py); raises ImportError
    when it has not been built."""
    global _native
    if _native is None:
        if not os.path.exists(NATIVE_SO):
            raise ImportError(f"{NATIVE_SO} is missing; run build.py")
        L.lib()  # the C-ABI library the extension links against
        spec = importlib.util.spec_from_file_location("ippi_autograd", NATIVE_SO)
        mod = importlib.util.module_from_spec(spec)
        spec.loader.exec_module(mod)
        _native = mod
    return _native


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
