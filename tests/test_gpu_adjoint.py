"""Adjoint of the FP64 step (gp_adjoint): the cell functions it differentiates
reproduce the step bit for bit, and its gradients agree with central finite
differences of the forward runs."""
import ctypes

import numpy as np
import pytest

import eshwar_dipan_b200 as gp
from gp_cases import write_case

pytestmark = pytest.mark.gpu

# binary 2-phase solidification: a solid seed in a supersaturated liquid,
# obstacle potential, anti-trapping on (D_solid = 0)
CASES = {
    "dendrite_aniso": dict(kw=dict(N=2, K=1, mesh=(40, 36), aniso=True, dab=0.04, d_solid=0.0, d_liquid=[1.0],
                                   dt=0.02, eps=4.0, T=1.0, liquid_c=[0.42]),
                           seeds=[(0, 20, 18, 9.0)]),
    "dendrite_iso_periodic": dict(kw=dict(N=2, K=1, mesh=(36, 40), aniso=False, dab=0.0, d_solid=0.0,
                                          d_liquid=[1.0], dt=0.02, eps=4.0, T=1.0, liquid_c=[0.42],
                                          bc_phi=(3, 3, 3, 3)),
                                  seeds=[(0, 6, 20, 8.0), (0, 26, 8, 6.0)]),
}
PARAMS = ["tau", "dab", "epsilon", "gamma"]


def _params(tmp_path, name):
    c = CASES[name]
    ip, fp = write_case(str(tmp_path), name, c["kw"], seeds=c["seeds"])
    p = gp.load_params(ip)
    phi, mu = gp.fill(p, fp)
    return p, phi, mu


def _start(p, phi, mu):
    """the state after the smoothing sweeps: the start of the differentiated run"""
    with gp.Simulation(p, phi, mu) as s:
        s.smooth(p.nsmooth - 1)
        return s.get()


def _with(p, name, value):
    q = gp.Params()
    ctypes.memmove(ctypes.byref(q), ctypes.byref(p), ctypes.sizeof(p))
    if name == "tau":
        q.tau_ab[0][1] = q.tau_ab[1][0] = value
    elif name == "dab":
        q.dab[0][1] = q.dab[1][0] = value
    elif name == "epsilon":
        q.epsilon = value
    elif name == "gamma":
        q.gamma[0][1] = q.gamma[1][0] = value
    return q


def _get(p, name):
    return {"tau": p.tau_ab[0][1], "dab": p.dab[0][1], "epsilon": p.epsilon, "gamma": p.gamma[0][1]}[name]


def _loss(p, phi, mu, nsteps, target):
    with gp.Simulation(p, phi, mu) as s:
        s.step(nsteps, stats=False)
        ph, _ = s.get()
    return 0.5 * float(((ph - target) ** 2).sum())


@pytest.mark.parametrize("name", sorted(CASES))
def test_adjoint_cell_functions_replay_the_step(tmp_path, name):
    p, phi, mu = _params(tmp_path, name)
    with gp.Simulation(p, phi, mu) as s:
        s.smooth(p.nsmooth - 1)
        s.step(5, stats=False)
        diff, ndiff = s.adjoint_replay(25)
    assert ndiff == 0, "%d values differ, max %.3e" % (ndiff, diff)


def _target(p, phi, mu, nsteps):
    """the final phi of a run with every differentiable parameter 5% larger"""
    q = p
    for n in PARAMS:
        if n == "dab" and _get(p, n) == 0.0:
            continue
        q = _with(q, n, 1.05 * _get(q, n))
    with gp.Simulation(q, phi, mu) as s:
        s.step(nsteps, stats=False)
        return s.get()[0]


@pytest.mark.parametrize("name", sorted(CASES))
def test_adjoint_parameter_gradients_vs_finite_differences(tmp_path, name):
    p, phi0, mu0 = _params(tmp_path, name)
    phi, mu = _start(p, phi0, mu0)
    nsteps = 40
    target = _target(p, phi, mu, nsteps)
    with gp.Simulation(p, phi, mu) as s:
        g = s.adjoint(nsteps, target_phi=target)
    assert g["loss"] == pytest.approx(_loss(p, phi, mu, nsteps, target), rel=1e-12)
    for n in PARAMS:
        if n == "dab" and _get(p, n) == 0.0:
            continue
        v = _get(p, n)
        h = 1e-5 * abs(v)
        fd = (_loss(_with(p, n, v + h), phi, mu, nsteps, target) -
              _loss(_with(p, n, v - h), phi, mu, nsteps, target)) / (2 * h)
        ad = g["d_" + n]
        assert abs(ad - fd) <= 1e-5 * max(abs(fd), 1e-12 * g["loss"]), "%s: adjoint %.10e fd %.10e" % (n, ad, fd)


def test_adjoint_start_state_gradient_vs_finite_differences(tmp_path):
    """8 random directions supported on the interface cells (where the step is
    smooth in phi); central differences with step 1e-6."""
    p, phi0, mu0 = _params(tmp_path, "dendrite_aniso")
    phi, mu = _start(p, phi0, mu0)
    nsteps = 30
    target = _target(p, phi, mu, nsteps)
    with gp.Simulation(p, phi, mu) as s:
        g = s.adjoint(nsteps, target_phi=target)
    rng = np.random.default_rng(7)
    inner = (phi[0] > 0.05) & (phi[0] < 0.95)
    assert inner.sum() > 20
    h = 1e-6
    for _ in range(8):
        vphi = rng.standard_normal(phi.shape) * inner
        vmu = rng.standard_normal(mu.shape) * inner
        fd = (_loss(p, phi + h * vphi, mu + h * vmu, nsteps, target) -
              _loss(p, phi - h * vphi, mu - h * vmu, nsteps, target)) / (2 * h)
        ad = float((g["phi0_bar"] * vphi).sum() + (g["mu0_bar"] * vmu).sum())
        assert abs(ad - fd) <= 1e-5 * abs(fd) + 1e-9, "adjoint %.10e fd %.10e" % (ad, fd)


def test_adjoint_checkpoint_spacing_does_not_change_the_gradient(tmp_path):
    p, phi0, mu0 = _params(tmp_path, "dendrite_aniso")
    phi, mu = _start(p, phi0, mu0)
    nsteps = 23
    rng = np.random.default_rng(3)
    pb = rng.standard_normal(phi.shape)
    res = []
    for every in (0, 1, 7, 23):
        with gp.Simulation(p, phi, mu) as s:
            res.append(s.adjoint(nsteps, phi_bar=pb, checkpoint_every=every))
            end = s.get()
        with gp.Simulation(p, phi, mu) as s:
            s.step(nsteps, stats=False)
            ref = s.get()
        assert np.array_equal(end[0], ref[0]) and np.array_equal(end[1], ref[1])
    for r in res[1:]:
        np.testing.assert_allclose(r["phi0_bar"], res[0]["phi0_bar"], rtol=1e-10, atol=1e-12)
        for n in PARAMS:
            assert r["d_" + n] == pytest.approx(res[0]["d_" + n], rel=1e-10, abs=1e-14)


def test_adjoint_rejects_unsupported(tmp_path):
    from gp_cases import build_case
    ip, fp = build_case(tmp_path, "ternary3_aniso_periodic")
    p = gp.load_params(ip)
    phi, mu = gp.fill(p, fp)
    with gp.Simulation(p, phi, mu) as s:
        with pytest.raises(gp.GpError):
            s.adjoint(3, target_phi=phi)


def test_torch_integrator_gradients(tmp_path):
    """GPRollout (torch.autograd.Function over gp_step / gp_adjoint): torch's
    backward returns the adjoint's gradients, and a torch gradient check of
    the parameter gradient along one direction agrees with central differences."""
    import torch
    from eshwar_dipan_b200.integrator import GPRollout
    p, phi0, mu0 = _params(tmp_path, "dendrite_aniso")
    phi, mu = _start(p, phi0, mu0)
    nsteps = 25
    target = torch.from_numpy(_target(p, phi, mu, nsteps))
    roll = GPRollout(p, nsteps)
    th = roll.theta0().clone().requires_grad_(True)
    a = torch.from_numpy(phi.copy()).requires_grad_(True)
    m = torch.from_numpy(mu.copy()).requires_grad_(True)
    phi_t, mu_t = roll(a, m, th)
    loss = 0.5 * ((phi_t - target) ** 2).sum()
    loss.backward()
    with gp.Simulation(p, phi, mu) as s:
        g = s.adjoint(nsteps, target_phi=target.numpy())
    assert float(loss.detach()) == pytest.approx(g["loss"], rel=1e-12)
    np.testing.assert_allclose(a.grad.numpy(), g["phi0_bar"], rtol=1e-9, atol=1e-14)
    np.testing.assert_allclose(th.grad.numpy(), [g["d_tau"], g["d_dab"], g["d_epsilon"], g["d_gamma"]], rtol=1e-9)
    v = torch.tensor([1.0, 0.5, -0.25, 0.75], dtype=torch.float64)
    h = 1e-6
    with torch.no_grad():
        lp = 0.5 * ((roll(a, m, th + h * v)[0] - target) ** 2).sum()
        lm = 0.5 * ((roll(a, m, th - h * v)[0] - target) ** 2).sum()
    fd = float((lp - lm) / (2 * h))
    ad = float((th.grad * v).sum())
    assert abs(ad - fd) <= 1e-5 * abs(fd), (ad, fd)
