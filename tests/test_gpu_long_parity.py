"""The CUDA path against the CPU oracle over long runs and on the benchmarked
configurations (shrunk to sizes the oracle finishes in about 20 s).

The contract for the plain FP64 step is at most 1e-9 max-abs from the CPU
reference after 2000 steps; the step is bit-identical, so these tests ask for
identical bits (zeros of either sign equal) and report the largest difference
when they fail.  The oracle itself is pinned to the reference built from its
own sources (tests/test_oracle_golden.py).
"""
import os

import numpy as np
import pytest

import eshwar_dipan_b200 as gp
from eshwar_dipan_b200.workloads import workload
from oracle_py import Oracle, bits_equal, mismatch_report

pytestmark = pytest.mark.gpu

CONTRACT_MAX_ABS = 1e-9


def _case(tmp_path, name, scale):
    it, ft, desc, _ = workload(name, scale)
    ip, fp = os.path.join(str(tmp_path), name + ".in"), os.path.join(str(tmp_path), name + "_fill.in")
    open(ip, "w").write(it)
    open(fp, "w").write(ft)
    p = gp.load_params(ip)
    phi, mu = gp.fill(p, fp)
    return p, phi, mu, desc


def _compare(sim, o, when):
    a_phi, a_mu = sim.get()
    b_phi, b_mu = o.get()
    dmax = max(float(np.abs(a_phi - b_phi).max()), float(np.abs(a_mu - b_mu).max()))
    assert dmax <= CONTRACT_MAX_ABS, "%s: max |diff| %.3e above the 1e-9 contract" % (when, dmax)
    assert bits_equal(a_phi, b_phi), "%s phi: %s" % (when, mismatch_report(a_phi, b_phi))
    assert bits_equal(a_mu, b_mu), "%s mu: %s" % (when, mismatch_report(a_mu, b_mu))
    return a_phi


@pytest.mark.parametrize("name,scale,chunks", [
    ("cfg1", 1, (1000, 1000)),        # 256^2 binary, r=40 seed, 2000 steps (the contract's horizon)
    ("cfg2", 4, (100, 100)),          # 512^2 ternary 3-phase, anisotropic, periodic, 4 seeds
    ("cfg4", 8, (100, 100)),          # 512^2 ternary 3-phase, isotropic, Neumann, 4 seeds
])
def test_long_run_bitwise(tmp_path, name, scale, chunks):
    p, phi, mu, desc = _case(tmp_path, name, scale)
    o = Oracle(p, recip_div=1)
    o.set(phi, mu)
    o.smooth(p.nsmooth - 1)
    with gp.Simulation(p, phi, mu) as sim:
        sim.smooth(p.nsmooth - 1)
        done = 0
        for n in chunks:
            o.step(n)
            st = sim.step(n)
            done += n
            ph = _compare(sim, o, "%s after %d steps" % (desc, done))
        ost = o.stats()
        for k in ("phi_max", "phi_min", "mu_max", "mu_min"):
            assert st[k] == ost[k], k
        # the sums run in another order on the GPU: about n*eps relative
        for k in ("rel_change_phi", "rel_change_mu", "phi_sum", "comp_sum"):
            np.testing.assert_allclose(st[k], ost[k], rtol=1e-10, atol=1e-300, err_msg=k)
    # the interface moved: the run exercises the interface tiles throughout
    solid = ph[:-1].sum()
    assert solid > 0 and not np.all((ph == 0) | (ph == 1))
