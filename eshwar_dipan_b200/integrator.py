"""PyTorch integrator: the grand-potential time loop as a differentiable
torch operation over the C ABI (gp_step forward, gp_adjoint backward).

    rollout = GPRollout(params, nsteps=1000)
    phi_T, mu_T = rollout(phi0, mu0, theta)      # theta = [Tau, dab, epsilon, GAMMA]
    loss = ((phi_T - target) ** 2).sum() / 2
    loss.backward()                               # phi0.grad, mu0.grad, theta.grad

theta holds the phase pair (0,1) values of Tau (the mobility is 1/Tau), dab
(anisotropy strength), epsilon and GAMMA (interface energy).  The fields may be
float64 CUDA tensors on the device the library runs on: they then go in and
out by device pointers (gp_set_dev, gp_get_dev, gp_adjoint with device
buffers) and never through host memory; CPU tensors are copied in and out.
The computation runs in the CUDA kernels behind the ABI.  Supported where
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


def _simulation(p, phi, mu):
    if phi.is_cuda:
        return Simulation.from_tensors(p, phi, mu)
    return Simulation(p, phi.detach().numpy().astype(np.float64), mu.detach().numpy().astype(np.float64))


class _Rollout(torch.autograd.Function):
    @staticmethod
    def forward(ctx, phi0, mu0, theta, params, nsteps, checkpoint_every):
        p = with_theta(params, theta.detach().cpu().numpy())
        with _simulation(p, phi0, mu0) as s:
            s.step(nsteps, stats=False)
            if phi0.is_cuda:
                phi_t, mu_t = s.get_tensors()
            else:
                phi_t, mu_t = (torch.from_numpy(a) for a in s.get())
        ctx.save_for_backward(phi0, mu0, theta)
        ctx.params, ctx.nsteps, ctx.every = params, nsteps, checkpoint_every
        return phi_t, mu_t

    @staticmethod
    def backward(ctx, g_phi, g_mu):
        phi0, mu0, theta = ctx.saved_tensors
        p = with_theta(ctx.params, theta.detach().cpu().numpy())
        gphi = (g_phi if g_phi is not None else torch.zeros_like(phi0)).detach()
        gmu = (g_mu if g_mu is not None else torch.zeros_like(mu0)).detach()
        with _simulation(p, phi0, mu0) as s:
            if phi0.is_cuda:
                r = s.adjoint(ctx.nsteps, phi_bar=gphi.to(phi0.device), mu_bar=gmu.to(phi0.device),
                              checkpoint_every=ctx.every)
                g0, m0 = r["phi0_bar"], r["mu0_bar"]
            else:
                r = s.adjoint(ctx.nsteps, phi_bar=gphi.cpu().numpy(), mu_bar=gmu.cpu().numpy(),
                              checkpoint_every=ctx.every)
                g0, m0 = torch.from_numpy(r["phi0_bar"]), torch.from_numpy(r["mu0_bar"])
        d_theta = torch.tensor([r["d_tau"], r["d_dab"], r["d_epsilon"], r["d_gamma"]], dtype=theta.dtype,
                               device=theta.device)
        return g0, m0, d_theta, None, None, None


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
