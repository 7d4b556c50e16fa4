"""The CPU oracle against the reference's shipped result files and against the
reference built from its own sources (oracle/_ref)."""
import os
import sys

import numpy as np
import pytest

sys.path.insert(0, os.path.join(os.path.dirname(__file__), "golden"))
import recipes  # noqa: E402

import eshwar_dipan_b200 as gp  # noqa: E402
from gp_cases import PARITY_CASES, build_case  # noqa: E402
from oracle_py import (Oracle, bits_equal, harness_available, harness_run,  # noqa: E402
                       mismatch_report)


def _run_oracle(ip, fp, nsmooth_iters, nsteps, recip_div=0):
    p = gp.load_params(ip)
    phi, mu = gp.fill(p, fp)
    o = Oracle(p, recip_div=recip_div)
    o.set(phi, mu)
    o.smooth(nsmooth_iters)
    o.step(nsteps)
    return p, o


@pytest.mark.parametrize("key", ["output_out_0", "output_out_1000", "Output_iso_1000", "Output_iso_2000"])
def test_oracle_reproduces_golden_vtk(tmp_path, key):
    kind, steps, fields = recipes.GOLDEN[key]
    ip, fp = recipes.write_golden_case(tmp_path, kind)
    # the t=0 file is written before the smoothing sweeps (microsim_gp.c:86-100)
    p, o = _run_oracle(ip, fp, 9 if steps else 0, steps)
    phi, mu = o.get()
    z = recipes.load_golden()
    for name, (fk, idx) in fields.items():
        ours = recipes.as_le((phi if fk == "phi" else mu)[idx])
        ref = recipes.golden_text(z, key, name)
        bad = sum(a != b for a, b in zip(ours, ref))
        assert bad == 0, "%s/%s: %d of %d values differ at '%%le' precision" % (key, name, bad, len(ref))


needs_ref = pytest.mark.skipif(not harness_available(), reason="reference harness not built (oracle/_ref)")


@needs_ref
@pytest.mark.parametrize("name", sorted(PARITY_CASES))
def test_oracle_matches_reference_bitwise(tmp_path, name):
    """Full ghosted phi and mu, and interior delta-phi, bit for bit after the
    smoothing sweeps and 12 time steps."""
    ip, fp = build_case(tmp_path, name)
    p, o = _run_oracle(ip, fp, 9, 12, recip_div=0)
    ref = harness_run(ip, fp, 9, 12, tmp_path)
    phi, mu, dphi = o.get_full()
    assert bits_equal(phi, ref["phi"]), mismatch_report(phi, ref["phi"])
    assert bits_equal(mu, ref["mu"]), mismatch_report(mu, ref["mu"])
    mx, my = p.mesh_x, p.mesh_y
    inner = (slice(None), slice(3, mx + 3), slice(3, my + 3))
    assert bits_equal(dphi[inner], ref["dphi"][inner]), mismatch_report(dphi[inner], ref["dphi"][inner])


@needs_ref
@pytest.mark.parametrize("name", ["bin_iso_antitrap", "three_phase_rot45", "ternary3_aniso_periodic"])
def test_fill_matches_reference(tmp_path, name):
    """gp_fill (host C surface) against the reference's fill_domain + BCs at t=0."""
    ip, fp = build_case(tmp_path, name)
    p = gp.load_params(ip)
    phi, mu = gp.fill(p, fp)
    ref = harness_run(ip, fp, 0, 0, tmp_path)
    mx, my = p.mesh_x, p.mesh_y
    assert bits_equal(phi, ref["phi"][:, 3:mx + 3, 3:my + 3])
    assert bits_equal(mu, ref["mu"][:, 3:mx + 3, 3:my + 3])


@needs_ref
def test_oracle_smoothing_division_variant_close(tmp_path):
    """The smoothing sweeps invert dc/dmu with pow(x,-1) in the reference; the
    division variant used on the GPU may differ by a few ulp in mu only."""
    ip, fp = build_case(tmp_path, "ternary3_aniso_periodic")
    p, o_pow = _run_oracle(ip, fp, 9, 0, recip_div=0)
    _, o_div = _run_oracle(ip, fp, 9, 0, recip_div=1)
    a_phi, a_mu = o_pow.get()
    b_phi, b_mu = o_div.get()
    assert bits_equal(a_phi, b_phi)
    rel = np.abs(a_mu - b_mu) / np.maximum(np.abs(a_mu), 1e-300)
    assert rel.max() <= 8 * np.finfo(np.float64).eps


@needs_ref
def test_oracle_matches_reference_on_shrunk_cfg2(tmp_path):
    """The benchmarked ternary 3-phase anisotropic periodic configuration,
    shrunk to 512^2 with the same seed density (4 seeds), over 200 steps: the
    oracle equals the reference built from its own sources bit for bit (full
    ghosted phi and mu)."""
    from eshwar_dipan_b200.workloads import workload
    it, ft, _, _ = workload("cfg2", 4)
    ip, fp = str(tmp_path / "c2.in"), str(tmp_path / "c2_fill.in")
    open(ip, "w").write(it)
    open(fp, "w").write(ft)
    import concurrent.futures
    with concurrent.futures.ThreadPoolExecutor(1) as pool:   # the two CPU runs side by side
        fut = pool.submit(harness_run, ip, fp, 9, 200, tmp_path)
        p, o = _run_oracle(ip, fp, 9, 200, recip_div=0)
        ref = fut.result()
    phi, mu, _ = o.get_full()
    assert bits_equal(phi, ref["phi"]), mismatch_report(phi, ref["phi"])
    assert bits_equal(mu, ref["mu"]), mismatch_report(mu, ref["mu"])
    inner = phi[:, 3:p.mesh_x + 3, 3:p.mesh_y + 3]
    assert not np.all((inner == 0) | (inner == 1))


@needs_ref
@pytest.mark.parametrize("shift", [False, True])
def test_oracle_matches_reference_directional(tmp_path, shift):
    """Directional solidification over 250 steps: the temperature field moves
    with the gradient after every step (microsim_gp.c:108-113) and, with the
    moving frame, the fields shift down at steps 100 and 200
    (microsim_gp.c:115-126, shift.h): the oracle equals the reference bit for
    bit (full ghosted phi and mu)."""
    from gp_cases import PARITY_CASES
    from eshwar_dipan_b200.workloads import write_case
    c = PARITY_CASES["dirsolid_binary"]
    kw = dict(c["kw"], shift=shift, shiftj=20)
    ip, fp = write_case(str(tmp_path), "ds", kw, seeds=c["seeds"], cubes=c["cubes"])
    p, o = _run_oracle(ip, fp, 9, 250, recip_div=0)
    ref = harness_run(ip, fp, 9, 250, tmp_path)
    phi, mu, _ = o.get_full()
    assert bits_equal(phi, ref["phi"]), mismatch_report(phi, ref["phi"])
    assert bits_equal(mu, ref["mu"]), mismatch_report(mu, ref["mu"])
    if shift:
        # the frame moved: the solid front sits near column shiftj, not where it grew to
        solid_rows = (phi[0, 3:-3, 3:-3] > 0.5).sum(axis=1)
        assert solid_rows.max() < 25
