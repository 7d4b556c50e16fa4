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


@pytest.mark.parametrize("name", ["dirsolid_binary", "dirsolid_ternary3"])
def test_directional_solidification_bitwise(tmp_path, name):
    """Non-isothermal runs (a temperature gradient moving along y): 300 steps
    bit-identical to the oracle, which equals the reference on these decks."""
    from gp_cases import PARITY_CASES, build_case
    ip, fp = build_case(tmp_path, name)
    p = gp.load_params(ip)
    phi, mu = gp.fill(p, fp)
    o = Oracle(p, recip_div=1)
    o.set(phi, mu)
    o.smooth(p.nsmooth - 1)
    with gp.Simulation(p, phi, mu) as sim:
        sim.smooth(p.nsmooth - 1)
        _compare(sim, o, name + " after smoothing")
        done = 0
        assert bits_equal(sim.temperature(), o.temperature()), "temperature at the start"
        for n in (1, 99, 200):
            o.step(n)
            st = sim.step(n)
            done += n
            _compare(sim, o, "%s after %d steps" % (name, done))
            assert bits_equal(sim.temperature(), o.temperature()), "temperature after %d steps" % done
        ost = o.stats()
        for k in ("phi_max", "phi_min", "mu_max", "mu_min"):
            assert st[k] == ost[k], k
        for k in ("rel_change_phi", "rel_change_mu", "phi_sum", "comp_sum"):
            np.testing.assert_allclose(st[k], ost[k], rtol=1e-10, atol=1e-300, err_msg=k)


def test_moving_frame_bitwise(tmp_path):
    """Directional solidification with the moving frame (Shift = 1): the
    fields shift down at step 100 once the interface passes Shiftj, the
    temperature field follows (its offset moves with the frame); 250 steps
    bit-identical to the oracle, which equals the reference on this deck.
    (After a shift the reference's ghost columns hold shifted values until its
    next boundary copy; with solid at the bottom and liquid at the top of the
    frame no phase is active there and the delta-phi they feed is 0 either
    way.)"""
    from gp_cases import PARITY_CASES
    from eshwar_dipan_b200.workloads import write_case
    c = PARITY_CASES["dirsolid_binary"]
    ip, fp = write_case(str(tmp_path), "frame", dict(c["kw"], shift=True, shiftj=20), seeds=c["seeds"],
                        cubes=c["cubes"])
    p = gp.load_params(ip)
    phi, mu = gp.fill(p, fp)
    o = Oracle(p, recip_div=1)
    o.set(phi, mu)
    o.smooth(p.nsmooth - 1)
    with gp.Simulation(p, phi, mu) as sim:
        sim.smooth(p.nsmooth - 1)
        done = 0
        for n in (99, 1, 50, 100):   # the shift after step 100, the graph path after it
            o.step(n)
            st = sim.step(n)
            done += n
            _compare(sim, o, "moving frame after %d steps" % done)
            # the temperature field as the reference holds it (moved with the frame at step 100)
            assert bits_equal(sim.temperature(), o.temperature()), "temperature after %d steps" % done
        ost = o.stats()
        assert st["shift_offset"] == ost["shift_offset"] > 0
        for k in ("phi_max", "phi_min", "mu_max", "mu_min"):
            assert st[k] == ost[k], k
