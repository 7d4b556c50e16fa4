"""Adjoint of the FP64 step (gp_adjoint): the cell functions it differentiates
reproduce the step bit for bit; its gradients agree with the FP64 tape
reference (tests/torch_tape.py) and with central finite differences of the
forward runs, at the test sizes and at the benchmarked 512x512, 1000-step
configuration; every checkpointing schedule gives the same gradients."""
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


@pytest.mark.parametrize("name", sorted(CASES) + ["well_aniso"])
def test_adjoint_matches_the_fp64_tape(tmp_path, name):
    """The CUDA adjoint against the FP64 tape reference: the same step written
    in float64 torch operations (bit for bit the oracle's) and differentiated
    by torch's autograd tape.  Loss equal, parameter gradients within 1e-9
    relative, start-state gradients within 1e-8 of their largest entry."""
    from torch_tape import tape_gradients
    if name == "well_aniso":
        from test_torch_tape import CASES as TCASES
        c = TCASES[name]
        ip, fp = write_case(str(tmp_path), name, c["kw"], seeds=c["seeds"])
        p = gp.load_params(ip)
        phi0, mu0 = gp.fill(p, fp)
    else:
        p, phi0, mu0 = _params(tmp_path, name)
    phi, mu = _start(p, phi0, mu0)
    nsteps = 30
    target = _target(p, phi, mu, nsteps)
    with gp.Simulation(p, phi, mu) as s:
        g = s.adjoint(nsteps, target_phi=target)
    loss, gth, gphi, gmu = tape_gradients(p, phi, mu, nsteps, target=target)
    assert g["loss"] == pytest.approx(loss, rel=1e-13)
    ad = np.array([g["d_tau"], g["d_dab"], g["d_epsilon"], g["d_gamma"]])
    np.testing.assert_allclose(ad, gth, rtol=1e-9, atol=1e-12 * np.abs(gth).max())
    np.testing.assert_allclose(g["phi0_bar"], gphi, rtol=0, atol=1e-8 * np.abs(gphi).max())
    np.testing.assert_allclose(g["mu0_bar"], gmu, rtol=0, atol=1e-8 * np.abs(gmu).max())


@pytest.mark.parametrize("name", sorted(CASES) + ["well_aniso"])
def test_hand_reverse_matches_dual_passes(tmp_path, name, monkeypatch):
    """The concentration pass's hand-derived reverse (GP_ADJOINT_HAND_UPDATE)
    against its dual-number passes (the default): the same derivatives, up to
    the rounding of the derivative arithmetic and the order of the atomic
    sums."""
    if name == "well_aniso":
        from test_torch_tape import CASES as TCASES
        c = TCASES[name]
        ip, fp = write_case(str(tmp_path), name, c["kw"], seeds=c["seeds"])
        p = gp.load_params(ip)
        phi0, mu0 = gp.fill(p, fp)
    else:
        p, phi0, mu0 = _params(tmp_path, name)
    phi, mu = _start(p, phi0, mu0)
    nsteps = 30
    target = _target(p, phi, mu, nsteps)
    res = []
    for dual in (False, True):
        if dual:
            monkeypatch.delenv("GP_ADJOINT_HAND_UPDATE", raising=False)
        else:
            monkeypatch.setenv("GP_ADJOINT_HAND_UPDATE", "1")
        with gp.Simulation(p, phi, mu) as s:
            res.append(s.adjoint(nsteps, target_phi=target))
    h, d = res
    for n in PARAMS:
        assert h["d_" + n] == pytest.approx(d["d_" + n], rel=1e-10, abs=1e-13 * abs(d["d_tau"])), n
    for k in ("phi0_bar", "mu0_bar"):
        np.testing.assert_allclose(h[k], d[k], rtol=0, atol=1e-10 * np.abs(d[k]).max(), err_msg=k)


def binomial_cost(l, s):
    """fewest forward steps that reverse l steps with the start state and s
    more states kept (binomial checkpointing: r*l - C(s+1+r, r-1) with r the
    least repetition number such that C(s+1+r, r) >= l)"""
    from math import comb
    if l <= 1:
        return 0
    if s <= 0:
        return l * (l - 1) // 2
    r = 0
    while comb(s + 1 + r, r) < l:
        r += 1
    return r * l - comb(s + 1 + r, r - 1)


def test_binomial_cost_is_the_optimum():
    """the schedule's cost bound equals the optimum of the recursion it
    follows (advance m, reverse the rest with one slot less, then the first m)"""
    from functools import lru_cache

    @lru_cache(None)
    def best(l, s):
        if l <= 1:
            return 0
        if s == 0:
            return l * (l - 1) // 2
        return min(m + best(l - m, s - 1) + best(m, s) for m in range(1, l))
    for s in range(0, 6):
        for l in range(1, 90):
            assert binomial_cost(l, s) == best(l, s), (l, s)


@pytest.mark.parametrize("kw", [dict(), dict(snapshots=22), dict(snapshots=1), dict(snapshots=3),
                                dict(snapshots=7), dict(checkpoint_every=7), dict(checkpoint_every=23)])
def test_adjoint_schedule_does_not_change_the_gradient(tmp_path, kw):
    """Every checkpointing schedule (the whole tape, binomial with 1, 3 or 7
    kept states, the states of every 7th or 23rd step) gives the same
    gradients, recomputes the binomial bound's number of steps and leaves the
    context at the final state."""
    p, phi0, mu0 = _params(tmp_path, "dendrite_aniso")
    phi, mu = _start(p, phi0, mu0)
    nsteps = 23
    rng = np.random.default_rng(3)
    pb = rng.standard_normal(phi.shape)
    with gp.Simulation(p, phi, mu) as s:
        ref = s.adjoint(nsteps, phi_bar=pb, snapshots=nsteps - 1)
    with gp.Simulation(p, phi, mu) as s:
        r = s.adjoint(nsteps, phi_bar=pb, **kw)
        end = s.get()
    with gp.Simulation(p, phi, mu) as s:
        s.step(nsteps, stats=False)
        fin = s.get()
    assert np.array_equal(end[0], fin[0]) and np.array_equal(end[1], fin[1])
    snaps = kw.get("snapshots") or (-(-nsteps // kw["checkpoint_every"]) if "checkpoint_every" in kw else nsteps - 1)
    snaps = min(snaps, nsteps - 1)
    assert r["snapshots"] == snaps
    assert r["recomputed"] == binomial_cost(nsteps, snaps) - (nsteps - 1)
    np.testing.assert_allclose(r["phi0_bar"], ref["phi0_bar"], rtol=1e-10, atol=1e-12)
    np.testing.assert_allclose(r["mu0_bar"], ref["mu0_bar"], rtol=1e-10, atol=1e-12)
    for n in PARAMS:
        assert r["d_" + n] == pytest.approx(ref["d_" + n], rel=1e-10, abs=1e-14)


def test_adjoint_tape_does_not_read_stale_memory(tmp_path):
    """Whole-tape mode steps from slot to slot; the slots' memory may hold an
    earlier adjoint's states (here: of another start state of the same size).
    The gradients and the final state equal those of a schedule that steps in
    the context's own buffers (3 kept states)."""
    p, phi0, mu0 = _params(tmp_path, "dendrite_aniso")
    phi, mu = _start(p, phi0, mu0)
    nsteps = 40
    rng = np.random.default_rng(5)
    pb = rng.standard_normal(phi.shape)
    other_phi = np.clip(phi[:, ::-1, :].copy(), 0.0, 1.0)   # the seed mirrored: different tiles
    with gp.Simulation(p, other_phi, mu) as s:
        s.adjoint(nsteps, phi_bar=pb)
    with gp.Simulation(p, phi, mu) as s:
        r = s.adjoint(nsteps, phi_bar=pb)
        end = s.get()
    with gp.Simulation(p, phi, mu) as s:
        ref = s.adjoint(nsteps, phi_bar=pb, snapshots=3)
        fin = s.get()
    assert r["snapshots"] == nsteps - 1 and ref["recomputed"] > 0
    assert np.array_equal(end[0], fin[0]) and np.array_equal(end[1], fin[1])
    np.testing.assert_allclose(r["phi0_bar"], ref["phi0_bar"], rtol=1e-10, atol=1e-12)
    for n in PARAMS:
        assert r["d_" + n] == pytest.approx(ref["d_" + n], rel=1e-10, abs=1e-14)


@pytest.mark.parametrize("nsteps", [99, 100, 101, 257])
def test_whole_tape_graph_chunks(tmp_path, nsteps):
    """The whole tape goes to the GPU in graphs of 100 steps per sweep (the
    first of each captured before the forward pass, a last one shorter): at
    lengths around and across the chunk size the gradients, the target loss
    and the final state equal those of a schedule that launches its steps
    one by one (a few kept states, steps recomputed)."""
    p, phi0, mu0 = _params(tmp_path, "dendrite_aniso")
    phi, mu = _start(p, phi0, mu0)
    target = _target(p, phi, mu, nsteps)
    with gp.Simulation(p, phi, mu) as s:
        r = s.adjoint(nsteps, target_phi=target)
        end = s.get()
    with gp.Simulation(p, phi, mu) as s:
        ref = s.adjoint(nsteps, target_phi=target, snapshots=4)
    with gp.Simulation(p, phi, mu) as s:
        s.step(nsteps, stats=False)
        fin = s.get()
    assert r["snapshots"] == nsteps - 1 and r["recomputed"] == 0 and ref["recomputed"] > 0
    assert np.array_equal(end[0], fin[0]) and np.array_equal(end[1], fin[1])
    assert r["loss"] == pytest.approx(ref["loss"], rel=1e-13)
    np.testing.assert_allclose(r["phi0_bar"], ref["phi0_bar"], rtol=1e-10, atol=1e-12)
    np.testing.assert_allclose(r["mu0_bar"], ref["mu0_bar"], rtol=1e-10, atol=1e-12)
    for n in PARAMS:
        assert r["d_" + n] == pytest.approx(ref["d_" + n], rel=1e-10, abs=1e-14)


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


def test_torch_integrator_cuda_tensors(tmp_path):
    """GPRollout on float64 CUDA tensors: the fields go in and out by device
    pointer, the results and gradients equal those of CPU tensors."""
    import torch
    from eshwar_dipan_b200.integrator import GPRollout
    p, phi0, mu0 = _params(tmp_path, "dendrite_aniso")
    phi, mu = _start(p, phi0, mu0)
    nsteps = 25
    target = _target(p, phi, mu, nsteps)
    roll = GPRollout(p, nsteps)
    out = {}
    for dev in ("cpu", "cuda"):
        th = roll.theta0().clone().to(dev).requires_grad_(True)
        a = torch.from_numpy(phi.copy()).to(dev).requires_grad_(True)
        m = torch.from_numpy(mu.copy()).to(dev).requires_grad_(True)
        phi_t, mu_t = roll(a, m, th)
        assert phi_t.device.type == dev and mu_t.device.type == dev
        loss = 0.5 * ((phi_t - torch.from_numpy(target).to(dev)) ** 2).sum()
        loss.backward()
        assert a.grad.device.type == dev and th.grad.device.type == dev
        out[dev] = (phi_t.detach().cpu().numpy(), a.grad.cpu().numpy(), m.grad.cpu().numpy(), th.grad.cpu().numpy())
    assert np.array_equal(out["cpu"][0], out["cuda"][0])
    for i in (1, 2, 3):
        np.testing.assert_allclose(out["cuda"][i], out["cpu"][i], rtol=1e-10, atol=1e-14)


def test_adjoint_benchmark_size_vs_finite_differences(tmp_path):
    """The adjoint's configuration as benchmarked: a 512x512 dendrite over
    1000 steps, gradients of the mismatch with the run whose parameters are 5%
    larger.  Each parameter gradient within 1e-5 relative of the central
    difference with step 1e-6 of the value, and the start-state gradient
    along 8 random directions on the interface cells likewise; every state is
    kept (no recomputed step).  The step is the branch-wise smooth map the
    trajectory takes: over 1000 steps a perturbation of 1e-5 in epsilon
    already moves the edge of the obstacle potential's active set (a kink),
    and its central difference is 2.2e-4 off; from 1e-6 down the differences
    converge to the adjoint (9e-9 at 1e-6, 7e-10 at 1e-7 for epsilon; every
    parameter within 4e-8 at 1e-6)."""
    from eshwar_dipan_b200.workloads import workload
    it, ft, desc, _ = workload("cfg5", 1)
    ip, fp = str(tmp_path / "i.in"), str(tmp_path / "f.in")
    open(ip, "w").write(it)
    open(fp, "w").write(ft)
    p = gp.load_params(ip)
    phi, mu = _start(p, *gp.fill(p, fp))
    nsteps = 1000
    target = _target(p, phi, mu, nsteps)
    with gp.Simulation(p, phi, mu) as s:
        g = s.adjoint(nsteps, target_phi=target)
    assert g["recomputed"] == 0 and g["snapshots"] == nsteps - 1
    assert g["loss"] == pytest.approx(_loss(p, phi, mu, nsteps, target), rel=1e-12)
    for n in PARAMS:
        if n == "dab" and _get(p, n) == 0.0:
            continue
        v = _get(p, n)
        h = 1e-6 * abs(v)
        fd = (_loss(_with(p, n, v + h), phi, mu, nsteps, target) -
              _loss(_with(p, n, v - h), phi, mu, nsteps, target)) / (2 * h)
        ad = g["d_" + n]
        assert abs(ad - fd) <= 1e-5 * abs(fd), "%s: adjoint %.10e fd %.10e (%s)" % (n, ad, fd, desc)
    # the start state along 8 random directions supported on the interface
    # cells (where the step is smooth in phi); central differences, step 1e-6
    rng = np.random.default_rng(11)
    inner = (phi[0] > 0.05) & (phi[0] < 0.95)
    assert inner.sum() > 100
    h = 1e-6
    for _ in range(8):
        vphi = rng.standard_normal(phi.shape) * inner
        vmu = rng.standard_normal(mu.shape) * inner
        fd = (_loss(p, phi + h * vphi, mu + h * vmu, nsteps, target) -
              _loss(p, phi - h * vphi, mu - h * vmu, nsteps, target)) / (2 * h)
        ad = float((g["phi0_bar"] * vphi).sum() + (g["mu0_bar"] * vmu).sum())
        assert abs(ad - fd) <= 1e-5 * abs(fd) + 1e-9, "start state: adjoint %.10e fd %.10e" % (ad, fd)
