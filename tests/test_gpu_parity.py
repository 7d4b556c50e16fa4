"""CUDA path (libgp, through the C ABI) against the CPU oracle, bit for bit."""
import os
import sys

import numpy as np
import pytest

sys.path.insert(0, os.path.join(os.path.dirname(__file__), "golden"))
import recipes  # noqa: E402

import eshwar_dipan_b200 as gp  # noqa: E402
from gp_cases import PARITY_CASES, build_case  # noqa: E402
from oracle_py import Oracle, bits_equal, mismatch_report  # noqa: E402

pytestmark = pytest.mark.gpu


def _both(ip, fp, nsmooth_iters, nsteps, recip_div=1):
    p = gp.load_params(ip)
    phi, mu = gp.fill(p, fp)
    o = Oracle(p, recip_div=recip_div)
    o.set(phi, mu)
    o.smooth(nsmooth_iters)
    sim = gp.Simulation(p, phi, mu)
    sim.smooth(nsmooth_iters)
    return p, o, sim


@pytest.mark.parametrize("name", sorted(PARITY_CASES))
def test_step_bitwise(tmp_path, name):
    """Smoothing sweeps then 25 steps: phi and mu identical bit for bit."""
    ip, fp = build_case(tmp_path, name)
    p, o, sim = _both(ip, fp, 9, 0)
    a_phi, a_mu = sim.get()
    b_phi, b_mu = o.get()
    assert bits_equal(a_phi, b_phi), "after smoothing: " + mismatch_report(a_phi, b_phi)
    assert bits_equal(a_mu, b_mu), "after smoothing: " + mismatch_report(a_mu, b_mu)
    for chunk in (1, 4, 20):
        o.step(chunk)
        st = sim.step(chunk)
        a_phi, a_mu = sim.get()
        b_phi, b_mu = o.get()
        assert bits_equal(a_phi, b_phi), "phi after +%d steps: %s" % (chunk, mismatch_report(a_phi, b_phi))
        assert bits_equal(a_mu, b_mu), "mu after +%d steps: %s" % (chunk, mismatch_report(a_mu, b_mu))
    ost = o.stats()
    for k in ("phi_max", "phi_min", "mu_max", "mu_min"):
        assert st[k] == ost[k], k
    for k in ("rel_change_phi", "rel_change_mu", "phi_sum", "comp_sum"):
        np.testing.assert_allclose(st[k], ost[k], rtol=1e-12, atol=1e-300, err_msg=k)
    assert st["nonfinite"] == 0 and st["steps_done"] == 25


@pytest.mark.parametrize("name", ["bin_iso_antitrap", "ternary3_aniso_periodic"])
def test_step_from_uploaded_state(tmp_path, name):
    """gp_set of an arbitrary in-range state, then steps: identical to the oracle."""
    ip, fp = build_case(tmp_path, name)
    p = gp.load_params(ip)
    phi, mu = gp.fill(p, fp)
    o = Oracle(p, recip_div=1)
    o.set(phi, mu)
    o.smooth(9)
    o.step(7)
    phi1, mu1 = o.get()
    sim = gp.Simulation(p, phi, mu)
    sim.set(phi1, mu1)
    o2 = Oracle(p, recip_div=1)
    o2.set(phi1, mu1)
    o2.step(10)
    sim.step(10, stats=False)
    a_phi, a_mu = sim.get()
    b_phi, b_mu = o2.get()
    assert bits_equal(a_phi, b_phi), mismatch_report(a_phi, b_phi)
    assert bits_equal(a_mu, b_mu), mismatch_report(a_mu, b_mu)


def _same_with_nans(a, b):
    """bit for bit (zeros of either sign equal), every NaN equal to every NaN"""
    na, nb = np.isnan(a), np.isnan(b)
    return np.array_equal(na, nb) and bits_equal(np.where(na, 0.0, a), np.where(nb, 0.0, b))


def test_nonfinite_mu_in_bulk_tiles(tmp_path):
    """A ternary case whose off-diagonal D, c_mu and A are zero (the bulk
    kernel leaves those terms out) with +inf and NaN planted in the mu of
    liquid bulk tiles: the cells they reach take every term, as the oracle
    does (NaN payloads aside)."""
    from gp_cases import write_case
    c = PARITY_CASES["four_phase_ternary_iso"]
    kw = dict(c["kw"], mesh=(96, 96))
    ip, fp = write_case(str(tmp_path), "nonfinite", kw, seeds=c["seeds"])
    p = gp.load_params(ip)
    phi, mu = gp.fill(p, fp)
    mu[0, 70, 70] = np.inf
    mu[1, 75, 40] = np.nan
    mu[0, 88, 10] = -np.inf
    o = Oracle(p, recip_div=1)
    o.set(phi, mu)
    sim = gp.Simulation(p, phi, mu)
    for chunk in (1, 2):
        o.step(chunk)
        sim.step(chunk, stats=False)
        a_phi, a_mu = sim.get()
        b_phi, b_mu = o.get()
        assert np.isnan(b_mu).sum() > 3
        assert _same_with_nans(a_phi, b_phi), mismatch_report(a_phi, b_phi)
        assert _same_with_nans(a_mu, b_mu), mismatch_report(a_mu, b_mu)
    # with a progress record the step reports the non-finite cells
    # (GP_ENONFINITE), after stepping as the reference does
    o.step(1)
    with pytest.raises(gp.NonFiniteError) as ei:
        sim.step(1, stats=True)
    assert ei.value.code == gp.GP_ENONFINITE
    b_phi, b_mu = o.get()
    n_bad = int((~(np.isfinite(b_phi).all(axis=0) & np.isfinite(b_mu).all(axis=0))).sum())
    assert n_bad > 0
    assert ei.value.stats["nonfinite"] == n_bad and ei.value.stats["steps_done"] == 4
    a_phi, a_mu = sim.get()
    assert _same_with_nans(a_phi, b_phi), mismatch_report(a_phi, b_phi)
    assert _same_with_nans(a_mu, b_mu), mismatch_report(a_mu, b_mu)


def test_smoothing_vs_reference_reciprocal(tmp_path):
    """Against the oracle with the reference's pow(x,-1) reciprocal the
    smoothing differs only by rounding of the dc/dmu inverse (mu, few ulp)."""
    ip, fp = build_case(tmp_path, "ternary3_aniso_periodic")
    p, o, sim = _both(ip, fp, 9, 0, recip_div=0)
    a_phi, a_mu = sim.get()
    b_phi, b_mu = o.get()
    assert bits_equal(a_phi, b_phi)
    rel = np.abs(a_mu - b_mu) / np.maximum(np.abs(b_mu), 1e-300)
    assert rel.max() <= 8 * np.finfo(np.float64).eps


@pytest.mark.parametrize("key", sorted(recipes.GOLDEN))
def test_golden_vtk_replay(tmp_path, key):
    """All twelve result files shipped with the reference, reproduced by the
    CUDA path at the files' printed precision."""
    kind, steps, fields = recipes.GOLDEN[key]
    ip, fp = recipes.write_golden_case(tmp_path, kind)
    p = gp.load_params(ip)
    phi, mu = gp.fill(p, fp)
    sim = gp.Simulation(p, phi, mu)
    if steps:
        sim.smooth(9)
        sim.step(steps, stats=False)
    phi, mu = sim.get()
    z = recipes.load_golden()
    for name, (fk, idx) in fields.items():
        ours = recipes.as_le((phi if fk == "phi" else mu)[idx])
        ref = recipes.golden_text(z, key, name)
        bad = sum(a != b for a, b in zip(ours, ref))
        assert bad == 0, "%s/%s: %d values differ" % (key, name, bad)


@pytest.mark.parametrize("ascii", [0, 1])
def test_vtk_write_async_matches_sync(tmp_path, ascii):
    """gp_vtk_write_async writes the bytes gp_get + gp_vtk_write write, while
    the steps queued after it go on (and are not disturbed by it)."""
    ip, fp = build_case(tmp_path, "ternary3_aniso_periodic")
    p = gp.load_params(ip)
    phi, mu = gp.fill(p, fp)
    with gp.Simulation(p, phi, mu) as s:
        s.smooth(p.nsmooth - 1)
        s.step(17, stats=False)
        ph, m = s.get()
        gp.vtk_write(p, str(tmp_path / "sync.vtk"), ph, m, ascii=ascii)
        s.vtk_write_async(str(tmp_path / "async.vtk"), ascii=ascii)
        s.step(9, stats=False)
        s.vtk_write_async(str(tmp_path / "async2.vtk"), ascii=ascii)   # waits for the first
        s.step(3, stats=False)
        s.vtk_wait()
        end = s.get()
    assert (tmp_path / "sync.vtk").read_bytes() == (tmp_path / "async.vtk").read_bytes()
    with gp.Simulation(p, ph, m) as s:
        s.step(9, stats=False)
        ph9, m9 = s.get()
        gp.vtk_write(p, str(tmp_path / "sync2.vtk"), ph9, m9, ascii=ascii)
        s.step(3, stats=False)
        ref = s.get()
    assert (tmp_path / "sync2.vtk").read_bytes() == (tmp_path / "async2.vtk").read_bytes()
    assert bits_equal(end[0], ref[0]) and bits_equal(end[1], ref[1])


@pytest.mark.parametrize("name", ["four_phase_ternary_iso", "ternary3_aniso_periodic"])
def test_bulk_box_wait_gives_up_and_reports(tmp_path, monkeypatch, name):
    """The bounded wait of the bulk tiles on their TMA boxes: with every box
    barrier set to expect 16 bytes more than a box brings
    (GP_TEST_TMA_SHORTFALL), each wait runs out after its few polls, the
    kernel raises its error flag and returns, and gp_step reports it.  The
    GPU stays usable: a new context then steps bit-identically to the oracle.
    (N=4 steps through kf_bulk, N=3 through kf_step.)"""
    from gp_cases import write_case
    c = PARITY_CASES[name]
    ip, fp = write_case(str(tmp_path), name + "_wait", dict(c["kw"], mesh=(96, 96)), seeds=c["seeds"])
    p = gp.load_params(ip)
    phi, mu = gp.fill(p, fp)
    monkeypatch.setenv("GP_TEST_TMA_SHORTFALL", "16")
    with gp.Simulation(p, phi, mu) as s:
        with pytest.raises(gp.GpError, match="did not arrive") as ei:
            s.step(1, stats=False)
        assert ei.value.code == gp.GP_ETIMEOUT
    monkeypatch.delenv("GP_TEST_TMA_SHORTFALL")
    o = Oracle(p, recip_div=1)
    o.set(phi, mu)
    o.step(3)
    with gp.Simulation(p, phi, mu) as s:
        s.step(3, stats=False)
        a_phi, a_mu = s.get()
    b_phi, b_mu = o.get()
    assert bits_equal(a_phi, b_phi) and bits_equal(a_mu, b_mu)


@pytest.mark.parametrize("mesh", [(8, 20), (5, 33), (40, 7)])
def test_grid_smaller_than_a_tile(tmp_path, mesh):
    """Grids narrower or shorter than one 8x32 tile (one ragged tile, a TMA box
    larger than the tensor): created, smoothed and stepped bit-identically to
    the oracle."""
    from gp_cases import write_case
    c = PARITY_CASES["bin_iso_antitrap"]
    seeds = [(0, mesh[0] // 2, mesh[1] // 2, 2.5)]
    ip, fp = write_case(str(tmp_path), "tiny", dict(c["kw"], mesh=mesh), seeds=seeds)
    p, o, sim = _both(ip, fp, 3, 0)
    o.step(12)
    sim.step(12, stats=False)
    a_phi, a_mu = sim.get()
    b_phi, b_mu = o.get()
    sim.close()
    assert bits_equal(a_phi, b_phi), mismatch_report(a_phi, b_phi)
    assert bits_equal(a_mu, b_mu), mismatch_report(a_mu, b_mu)
