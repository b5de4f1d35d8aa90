"""Gradients of a DEM rollout through the hand-written adjoint of the step.

``rollout(sim, k_n, gamma_n, mu, v0, nsteps)`` runs ``nsteps`` FP64 steps of
``sim`` on the GPU with the given contact parameters and initial velocities
and returns the final positions as a torch tensor whose backward pass is the
C ABI's sph_adjoint_backward: the contact set of each step is frozen, each
contact law is differentiated on the branch it took, and the state is
recomputed from checkpoints taken every ``ckpt`` steps.

Scope (the C ABI returns SPH_ERR_UNSUPPORTED otherwise): contact model 2
(linear), E = 0, kappa = 0, no bonds, no dynamic walls (nw = 0), fixed grid,
gamma_wt = 0.  mu sets mu_s and mu_d together; k_t is held fixed.
"""
import copy

import numpy
import torch

from .runner import Stepper


class DemRollout(torch.autograd.Function):
    """x_T = rollout(k_n, gamma_n, mu, v0); gradients for all four inputs."""

    @staticmethod
    def forward(ctx, k_n, gamma_n, mu, v0, sim, nsteps, ckpt, device):
        s = copy.deepcopy(sim)
        s.k_n[0] = float(k_n)
        s.gamma_n[0] = float(gamma_n)
        s.mu_s[0] = s.mu_d[0] = float(mu)
        s.vel[:, :] = v0.detach().to("cpu", torch.float64).numpy()
        st = Stepper([s], precision="fp64", length="fp64", device=device)
        st.upload()
        ctx.forward_ms = st.adjoint_forward(int(nsteps), int(ckpt))
        hp, _ = st.download()
        ctx.stepper = st
        ctx.dtype = v0.dtype
        ctx.device = v0.device
        return torch.from_numpy(numpy.ascontiguousarray(hp.x[:, :3])).to(v0.device)

    @staticmethod
    def backward(ctx, gx):
        st = ctx.stepper
        try:
            g, gv, ms = st.adjoint_backward(gx.detach().to("cpu", torch.float64).numpy())
        finally:
            st.close()
            ctx.stepper = None
        ctx.adjoint_ms = ms
        def scalar(v):
            return torch.tensor(v, dtype=torch.float64, device=ctx.device)
        return (scalar(g["k_n"]), scalar(g["gamma_n"]), scalar(g["mu"]),
                torch.from_numpy(gv).to(ctx.device, ctx.dtype), None, None, None, None)


def rollout(sim, k_n, gamma_n, mu, v0, nsteps, ckpt=100, device=0):
    """Final positions [np, 3] (float64) after nsteps steps of sim with the
    given k_n, gamma_n, mu (0-d tensors) and initial velocities v0 [np, 3];
    differentiable in all four."""
    return DemRollout.apply(k_n, gamma_n, mu, v0, sim, nsteps, ckpt, device)
