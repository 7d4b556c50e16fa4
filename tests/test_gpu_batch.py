"""Batched engine (gp_batch_*): FP64 batches bit-identical to the oracle per
simulation; FP32 batches within the stated error of the FP64 path."""
import numpy as np
import pytest

import eshwar_dipan_b200 as gp
from gp_cases import PARITY_CASES, write_case
from oracle_py import Oracle, bits_equal, mismatch_report

pytestmark = pytest.mark.gpu

# Same NUMPHASES / NUMCOMPONENTS / anisotropy inside a group, different sizes,
# boundary conditions and physical parameters.
BINARY_ANISO = ["bin_aniso_neumann", "bin_aniso_periodic", "well_aniso", "bin_mixed_bc"]


def _case(tmp_path, name, **over):
    c = PARITY_CASES[name]
    kw = dict(c["kw"])
    kw.update(over)
    tag = name + "".join("_%s" % k for k in sorted(over))
    ip, fp = write_case(str(tmp_path), tag, kw, seeds=c.get("seeds", ()), cubes=c.get("cubes", ()))
    p = gp.load_params(ip)
    phi, mu = gp.fill(p, fp)
    return p, phi, mu


def _ternary_group(tmp_path):
    out = [_case(tmp_path, "ternary3_aniso_periodic")]
    out.append(_case(tmp_path, "ternary3_aniso_periodic", mesh=(70, 34), dab=0.035))
    out.append(_case(tmp_path, "ternary3_aniso_periodic", mesh=(33, 97), bc_phi=(1, 1, 3, 3), dt=0.015))
    return out


def _binary_group(tmp_path):
    out = [_case(tmp_path, n) for n in BINARY_ANISO]
    out.append(_case(tmp_path, "bin_aniso_neumann", mesh=(130, 66), dab=0.01))
    return out


def _oracle_run(p, phi, mu, nsmooth, nsteps):
    o = Oracle(p, recip_div=1)
    o.set(phi, mu)
    o.smooth(nsmooth)
    o.step(nsteps)
    r = o.get()
    st = o.stats()
    o.close()
    return r, st


@pytest.mark.parametrize("group", ["binary", "ternary"])
def test_fp64_batch_bitwise(tmp_path, group):
    """A batch of simulations of different sizes and parameters, stepped through
    the work queue and a 100-step CUDA graph: each simulation identical bit for
    bit to the oracle run alone."""
    sims = _binary_group(tmp_path) if group == "binary" else _ternary_group(tmp_path)
    b = gp.Batch([s[0] for s in sims], [(s[1], s[2]) for s in sims], precision=gp.GP_FP64)
    assert len(sims) == b.n
    b.smooth(9)
    b.step(3)
    st = b.step(127)
    for i, (p, phi, mu) in enumerate(sims):
        (ophi, omu), ost = _oracle_run(p, phi, mu, 9, 130)
        a_phi, a_mu = b.get(i)
        assert bits_equal(a_phi, ophi), "sim %d phi: %s" % (i, mismatch_report(a_phi, ophi))
        assert bits_equal(a_mu, omu), "sim %d mu: %s" % (i, mismatch_report(a_mu, omu))
        for k in ("phi_max", "phi_min", "mu_max", "mu_min"):
            assert st[i][k] == ost[k], (i, k)
        for k in ("phi_sum", "comp_sum", "rel_change_phi", "rel_change_mu"):
            np.testing.assert_allclose(st[i][k], ost[k], rtol=1e-12, atol=1e-300, err_msg="%d %s" % (i, k))
        assert st[i]["steps_done"] == 130 and st[i]["nonfinite"] == 0
    b.close()


def test_fp64_batch_set_get_roundtrip(tmp_path):
    """gp_batch_set of one simulation leaves the others untouched; get returns it."""
    sims = _binary_group(tmp_path)[:3]
    b = gp.Batch([s[0] for s in sims], [(s[1], s[2]) for s in sims], precision=gp.GP_FP64)
    p, phi, mu = sims[1]
    rng = np.random.default_rng(3)
    phi2 = np.clip(phi + 0.01 * rng.standard_normal(phi.shape), 0, 1)
    b.set(1, phi2, mu)
    g_phi, g_mu = b.get(1)
    assert bits_equal(g_phi, phi2) and bits_equal(g_mu, mu)
    for i in (0, 2):
        g_phi, g_mu = b.get(i)
        assert bits_equal(g_phi, sims[i][1]) and bits_equal(g_mu, sims[i][2])
    b.close()


def test_batch_rejects_mixed_shapes(tmp_path):
    a = _case(tmp_path, "bin_aniso_neumann")
    t = _case(tmp_path, "ternary3_aniso_periodic")
    with pytest.raises(gp.GpError):
        gp.Batch([a[0], t[0]], [(a[1], a[2]), (t[1], t[2])], precision=gp.GP_FP32)


# FP32 storage form: error budget against the FP64 path (which is the oracle
# bit for bit): max |dphi| <= 1e-4 and relative solute-mass difference <= 1e-6
# after 1e4 steps on the precision workload.  The parity grids are a few
# thousand cells, mostly interface, where the FP64 scheme's own mass change per
# step is largest and a 1e-4 difference of interface position moves it; they
# get a 1e-5 mass budget.
FP32_PHI_TOL = 1e-4
FP32_MASS_TOL = 1e-6
FP32_MASS_TOL_SMALL = 1e-5


def _fp64_run(p, phi, mu, nsmooth, nsteps):
    with gp.Simulation(p, phi, mu) as s:
        s.smooth(nsmooth)
        st = s.step(nsteps)
        return s.get(), st


@pytest.mark.parametrize("group", ["binary", "ternary"])
def test_fp32_batch_error_budget(tmp_path, group):
    sims = _binary_group(tmp_path) if group == "binary" else _ternary_group(tmp_path)
    b = gp.Batch([s[0] for s in sims], [(s[1], s[2]) for s in sims], precision=gp.GP_FP32)
    b.smooth(9)
    st32 = b.step(2000)
    for i, (p, phi, mu) in enumerate(sims):
        (phi64, mu64), st64 = _fp64_run(p, phi, mu, 9, 2000)
        phi32, mu32 = b.get(i)
        assert np.isfinite(phi32).all() and np.isfinite(mu32).all()
        err = np.abs(phi32 - phi64).max()
        assert err <= FP32_PHI_TOL, "sim %d: max|dphi| %.3e" % (i, err)
        for k in range(len(st64["comp_sum"])):
            m64, m32 = st64["comp_sum"][k], st32[i]["comp_sum"][k]
            drift = abs(m32 - m64) / abs(m64)
            assert drift <= FP32_MASS_TOL_SMALL, "sim %d comp %d: mass drift %.3e" % (i, k, drift)
        cells = p.mesh_x * p.mesh_y
        np.testing.assert_allclose(st32[i]["phi_sum"], st64["phi_sum"], rtol=1e-5, atol=1e-6 * cells)
    b.close()


def test_fp32_batch_matches_single(tmp_path):
    """A simulation stepped inside a batch is bit-identical to the same
    simulation stepped alone (a batch of one): tiles are independent of which
    CTA picks them up."""
    sims = _ternary_group(tmp_path)
    b = gp.Batch([s[0] for s in sims], [(s[1], s[2]) for s in sims], precision=gp.GP_FP32)
    b.smooth(5)
    b.step(150, stats=False)
    for i, (p, phi, mu) in enumerate(sims):
        with gp.Simulation(p, phi, mu, precision=gp.GP_FP32) as s:
            s.smooth(5)
            s.step(150, stats=False)
            a_phi, a_mu = s.get()
        b_phi, b_mu = b.get(i)
        assert bits_equal(a_phi, b_phi), "sim %d: %s" % (i, mismatch_report(a_phi, b_phi))
        assert bits_equal(a_mu, b_mu), "sim %d: %s" % (i, mismatch_report(a_mu, b_mu))
    b.close()


def test_fp32_graph_chunks_match_single_steps(tmp_path):
    """250 steps as graphs of 100 plus single steps == 250 single steps."""
    sims = _binary_group(tmp_path)[:2]
    args = ([s[0] for s in sims], [(s[1], s[2]) for s in sims])
    b1 = gp.Batch(*args, precision=gp.GP_FP32)
    b2 = gp.Batch(*args, precision=gp.GP_FP32)
    b1.step(250, stats=False)
    for _ in range(250):
        b2.step(1, stats=False)
    for i in range(len(sims)):
        x, y = b1.get(i), b2.get(i)
        assert bits_equal(x[0], y[0]) and bits_equal(x[1], y[1])
    b1.close()
    b2.close()


def test_fp32_precision_workload(tmp_path):
    """The precision workload (ternary 3-phase, isotropic, Neumann, 256 seeds
    per 4096^2) at 1024^2 with the same seed density, 1e4 steps: FP32 against
    FP64 within max|dphi| 1e-4 and relative solute-mass difference 1e-6 at
    every checkpoint (each 1000 steps), not only at the end."""
    from eshwar_dipan_b200.workloads import write_workload
    ip, fp, desc, kw = write_workload(str(tmp_path), "cfg4", scale=4)
    p = gp.load_params(ip)
    phi, mu = gp.fill(p, fp)
    s64 = gp.Simulation(p, phi, mu, precision=gp.GP_FP64)
    s32 = gp.Simulation(p, phi, mu, precision=gp.GP_FP32)
    for s in (s64, s32):
        s.smooth(p.nsmooth - 1)
    worst = []
    for chunk in range(10):
        st64 = s64.step(1000)
        st32 = s32.step(1000)
        err = float(np.abs(s32.get()[0] - s64.get()[0]).max())
        drift = max(abs(a - b) / abs(b) for a, b in zip(st32["comp_sum"], st64["comp_sum"]))
        worst.append((1000 * (chunk + 1), err, drift))
    s64.close()
    s32.close()
    bad = [w for w in worst if w[1] > FP32_PHI_TOL or w[2] > FP32_MASS_TOL]
    assert not bad, "checkpoints over the bounds (step, max|dphi|, mass drift): %s" % bad


@pytest.mark.parametrize("prec", ["fp64", "fp32"])
def test_single_launch_step_matches_two_kernels(tmp_path, monkeypatch, prec):
    """Steps as one launch (kf_step: interface tiles, then bulk tiles) and as
    two launches (kf_bulk, kf_general; GP_SPLIT_KERNELS=1 at batch creation)
    give the same bits."""
    sims = _ternary_group(tmp_path)
    args = ([s[0] for s in sims], [(s[1], s[2]) for s in sims])
    pr = gp.GP_FP64 if prec == "fp64" else gp.GP_FP32
    monkeypatch.setenv("GP_NO_TUNING", "1")   # the single-launch shape, not a tuned one
    b1 = gp.Batch(*args, precision=pr)
    monkeypatch.setenv("GP_SPLIT_KERNELS", "1")
    b2 = gp.Batch(*args, precision=pr)
    monkeypatch.delenv("GP_SPLIT_KERNELS")
    monkeypatch.delenv("GP_NO_TUNING")
    for b in (b1, b2):
        b.smooth(5)
        b.step(230, stats=False)
    for i in range(len(sims)):
        x, y = b1.get(i), b2.get(i)
        assert bits_equal(x[0], y[0]) and bits_equal(x[1], y[1]), "sim %d" % i
    b1.close()
    b2.close()


def test_autotuned_shapes_give_the_same_bits(tmp_path, monkeypatch):
    """The launch-shape autotuner times its candidates on the first 100-step
    chunks of the live simulation: the result equals an untuned run bit for
    bit (every shape steps the same tiles the same way)."""
    sims = _ternary_group(tmp_path)
    args = ([s[0] for s in sims], [(s[1], s[2]) for s in sims])
    monkeypatch.setenv("GP_NO_TUNING", "1")
    ref = gp.Batch(*args, precision=gp.GP_FP64)
    monkeypatch.delenv("GP_NO_TUNING")
    tuned = gp.Batch(*args, precision=gp.GP_FP64)
    for b in (ref, tuned):
        b.step(650, stats=False)
    for i in range(len(sims)):
        x, y = ref.get(i), tuned.get(i)
        assert bits_equal(x[0], y[0]) and bits_equal(x[1], y[1]), "sim %d" % i
    ref.close()
    tuned.close()
