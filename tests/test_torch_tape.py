"""The FP64 tape reference of the adjoint (tests/torch_tape.py): its step,
float64 torch operations, is the oracle's step bit for bit, and the gradients
its autograd tape gives agree with central differences of its own runs."""
import numpy as np
import pytest
import torch

import eshwar_dipan_b200 as gp
from gp_cases import write_case
from oracle_py import Oracle, bits_equal, mismatch_report
from torch_tape import TapeStep, tape_gradients

# the adjoint's cases: binary 2-phase dendrites, obstacle potential, anti-trapping on
CASES = {
    "dendrite_aniso": dict(kw=dict(N=2, K=1, mesh=(40, 36), aniso=True, dab=0.04, d_solid=0.0, d_liquid=[1.0],
                                   dt=0.02, eps=4.0, T=1.0, liquid_c=[0.42]),
                           seeds=[(0, 20, 18, 9.0)]),
    "dendrite_iso_periodic": dict(kw=dict(N=2, K=1, mesh=(36, 40), aniso=False, dab=0.0, d_solid=0.0,
                                          d_liquid=[1.0], dt=0.02, eps=4.0, T=1.0, liquid_c=[0.42],
                                          bc_phi=(3, 3, 3, 3)),
                                  seeds=[(0, 6, 20, 8.0), (0, 26, 8, 6.0)]),
    "well_aniso": dict(kw=dict(N=2, K=1, mesh=(32, 32), well=True, dab=0.03, d_solid=0.0, d_liquid=[1.0],
                               T=1.0, liquid_c=[0.42]),
                       seeds=[(0, 16, 16, 8.0)]),
}


def _start(tmp_path, name):
    c = CASES[name]
    ip, fp = write_case(str(tmp_path), name, c["kw"], seeds=c["seeds"])
    p = gp.load_params(ip)
    phi, mu = gp.fill(p, fp)
    o = Oracle(p, recip_div=1)
    o.set(phi, mu)
    o.smooth(p.nsmooth - 1)
    return p, o


@pytest.mark.parametrize("name", sorted(CASES))
def test_tape_step_is_the_oracle_step(tmp_path, name):
    p, o = _start(tmp_path, name)
    ph0, mu0 = o.get()
    ts = TapeStep(p)
    a, m = torch.from_numpy(ph0), torch.from_numpy(mu0)
    th = ts.theta0()
    for t in range(1, 31):
        o.step(1)
        a, m = ts.step(a, m, th)
        oph, omu = o.get()
        assert bits_equal(a.numpy(), oph), "phi after %d steps: %s" % (t, mismatch_report(a.numpy(), oph))
        assert bits_equal(m.numpy(), omu), "mu after %d steps: %s" % (t, mismatch_report(m.numpy(), omu))
    assert not np.all((oph == 0) | (oph == 1))


@pytest.mark.parametrize("name", ["dendrite_aniso", "well_aniso"])
def test_tape_gradients_vs_finite_differences(tmp_path, name):
    p, o = _start(tmp_path, name)
    ph0, mu0 = o.get()
    nsteps = 20
    ts = TapeStep(p)
    th = ts.theta0()
    start = (torch.from_numpy(ph0), torch.from_numpy(mu0))
    with torch.no_grad():
        target = ts.run(*start, th * 1.05, nsteps)[0].numpy()
    loss, g, _, _ = tape_gradients(p, ph0, mu0, nsteps, target=target)
    for i in range(4):
        if float(th[i]) == 0.0:
            continue
        h = 1e-5 * abs(float(th[i]))
        e = torch.zeros(4, dtype=torch.float64)
        e[i] = h
        with torch.no_grad():
            lp = 0.5 * ((ts.run(*start, th + e, nsteps)[0].numpy() - target) ** 2).sum()
            lm = 0.5 * ((ts.run(*start, th - e, nsteps)[0].numpy() - target) ** 2).sum()
        fd = (lp - lm) / (2 * h)
        assert abs(g[i] - fd) <= 1e-6 * abs(fd), (i, g[i], fd)
