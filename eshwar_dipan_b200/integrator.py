"""PyTorch integrator: the grand-potential time loop as a differentiable
torch operation over the C ABI (gp_step forward, gp_adjoint backward).

    rollout = GPRollout(params, nsteps=1000)
    phi_T, mu_T = rollout(phi0, mu0, theta)      # theta = [Tau, dab, epsilon, GAMMA]
    loss = ((phi_T - target) ** 2).sum() / 2
    loss.backward()                               # phi0.grad, mu0.grad, theta.grad

theta holds the phase pair (0,1) values of Tau (the mobility is 1/Tau), dab
(anisotropy strength), epsilon and GAMMA (interface energy).  Tensors are
float64 on the CPU (the library copies them to its own device buffers); the
computation runs in the CUDA kernels behind the ABI.  Supported where
gp_adjoint is: NUMPHASES = 2, one BINARY component, FP64.
"""
import ctypes

import numpy as np
import torch

from . import Simulation
from ._abi import Params

__all__ = ["GPRollout", "with_theta"]


def with_theta(params, theta):
    """A copy of gp_params with Tau, dab, GAMMA of the pair (0,1) and epsilon
    taken from theta (4 numbers)."""
    q = Params()
    ctypes.memmove(ctypes.byref(q), ctypes.byref(params), ctypes.sizeof(params))
    t = [float(v) for v in theta]
    q.tau_ab[0][1] = q.tau_ab[1][0] = t[0]
    q.dab[0][1] = q.dab[1][0] = t[1]
    q.epsilon = t[2]
    q.gamma[0][1] = q.gamma[1][0] = t[3]
    return q


class _Rollout(torch.autograd.Function):
    @staticmethod
    def forward(ctx, phi0, mu0, theta, params, nsteps, checkpoint_every):
        p = with_theta(params, theta.detach().cpu().numpy())
        a = phi0.detach().cpu().numpy().astype(np.float64)
        m = mu0.detach().cpu().numpy().astype(np.float64)
        with Simulation(p, a, m) as s:
            s.step(nsteps, stats=False)
            phi_t, mu_t = s.get()
        ctx.save_for_backward(phi0, mu0, theta)
        ctx.params, ctx.nsteps, ctx.every = params, nsteps, checkpoint_every
        return torch.from_numpy(phi_t), torch.from_numpy(mu_t)

    @staticmethod
    def backward(ctx, g_phi, g_mu):
        phi0, mu0, theta = ctx.saved_tensors
        p = with_theta(ctx.params, theta.detach().cpu().numpy())
        gphi = (g_phi if g_phi is not None else torch.zeros_like(phi0)).detach().cpu().numpy()
        gmu = (g_mu if g_mu is not None else torch.zeros_like(mu0)).detach().cpu().numpy()
        with Simulation(p, phi0.detach().cpu().numpy(), mu0.detach().cpu().numpy()) as s:
            r = s.adjoint(ctx.nsteps, phi_bar=gphi, mu_bar=gmu, checkpoint_every=ctx.every)
        d_theta = torch.tensor([r["d_tau"], r["d_dab"], r["d_epsilon"], r["d_gamma"]], dtype=theta.dtype)
        return torch.from_numpy(r["phi0_bar"]), torch.from_numpy(r["mu0_bar"]), d_theta, None, None, None


class GPRollout:
    """nsteps FP64 time steps of one simulation as a differentiable function
    (phi0, mu0, theta) -> (phi_T, mu_T)."""

    def __init__(self, params, nsteps, checkpoint_every=0):
        self.params = params
        self.nsteps = int(nsteps)
        self.every = int(checkpoint_every)

    def __call__(self, phi0, mu0, theta):
        return _Rollout.apply(phi0, mu0, theta, self.params, self.nsteps, self.every)

    def theta0(self):
        """theta of the parameters the rollout was built with"""
        p = self.params
        return torch.tensor([p.tau_ab[0][1], p.dab[0][1], p.epsilon, p.gamma[0][1]], dtype=torch.float64)
