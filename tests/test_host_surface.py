"""The C host surface against the reference's own routines: the legacy-VTK
writer and reader (writetofile_serial2D[_binary], readfromfile_serial2D[_binary],
file_writer.h) and the command-line driver (main(), microsim_gp.c:41-151),
including a restart from a written file.

The reference side is oracle/_ref/gp_ref_harness, the reference's sources
built by oracle/Makefile; its state after the smoothing sweeps and steps is
the oracle's bit for bit (tests/test_oracle_golden.py), so the writer tests
feed the oracle's state to gp_vtk_write and need no GPU.
"""
import os
import shutil
import subprocess

import numpy as np
import pytest

import eshwar_dipan_b200 as gp
from gp_cases import write_case
from oracle_py import HARNESS, Oracle, bits_equal, harness_available, mismatch_report

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
CLI = os.path.join(ROOT, "eshwar_dipan_b200", "gp_microsim")

needs_ref = pytest.mark.skipif(not harness_available(), reason="reference harness not built (oracle/_ref)")

CASE = dict(N=3, K=2, mesh=(36, 44), dab=0.02, bc_phi=(3, 3, 1, 1), A_off=0.25)
SEEDS = [(0, 12, 12, 6.0), (1, 24, 30, 5.5)]


def _deck(tmp_path, name, ascii, writecomposition=0, ntimesteps=40, savet=20, starttime=0, restart=0):
    ip, fp = write_case(str(tmp_path), name, dict(CASE, ascii=ascii, writecomposition=writecomposition,
                                                  ntimesteps=ntimesteps), seeds=SEEDS)
    text = open(ip).read()
    text = text.replace("SAVET = %d;" % ntimesteps, "SAVET = %d;" % savet)
    text = text.replace("STARTTIME = 0;", "STARTTIME = %d;" % starttime)
    text = text.replace("RESTART = 0;", "RESTART = %d;" % restart)
    open(ip, "w").write(text)
    return ip, fp


def _run(cmd, cwd):
    """The reference crashes at random at start-up (a heap overflow in its
    parser); retry a few times."""
    last = None
    for _ in range(4):
        r = subprocess.run(cmd, capture_output=True, text=True, cwd=str(cwd))
        if r.returncode == 0:
            return r
        last = r
    raise RuntimeError("%s failed: rc=%s %s" % (cmd[0], last.returncode, last.stderr[-500:]))


@needs_ref
@pytest.mark.parametrize("ascii,wc", [(1, 0), (0, 0), (1, 1), (0, 1)])
def test_vtk_writer_matches_reference(tmp_path, ascii, wc):
    """gp_vtk_write writes the reference writer's bytes for the same state
    (ASCII '%le' text or big-endian binary, with and without the composition
    fields)."""
    ip, fp = _deck(tmp_path, "w", ascii, writecomposition=wc)
    ref_dir = tmp_path / "ref"
    ref_dir.mkdir()
    _run([HARNESS, os.path.abspath(ip), os.path.abspath(fp), "vtk", "5", "w"], ref_dir)
    p = gp.load_params(ip)
    phi, mu = gp.fill(p, fp)
    o = Oracle(p, recip_div=0)
    o.set(phi, mu)
    o.smooth(p.nsmooth - 1)
    o.step(5)
    ph, m = o.get()
    ours = str(tmp_path / "ours.vtk")
    gp.vtk_write(p, ours, ph, m)
    a = open(ours, "rb").read()
    b = (ref_dir / "DATA" / "w_5.vtk").read_bytes()
    assert a == b, "first difference at byte %d of %d/%d" % (
        next((i for i, (x, y) in enumerate(zip(a, b)) if x != y), min(len(a), len(b))), len(a), len(b))


@needs_ref
@pytest.mark.parametrize("ascii,wc,steps,shift", [(1, 1, 0, False), (0, 1, 0, False), (1, 0, 130, True),
                                                  (0, 1, 130, True), (0, 1, 60, False)])
def test_vtk_writer_nonisothermal_matches_reference(tmp_path, ascii, wc, steps, shift):
    """Directional solidification: the writer adds the Temperature field and
    takes the composition at each cell's temperature, as the reference's
    writer does; the field is the oracle's (laid down after the last step and
    moved with the frame, which here moves at step 100), or at step 0 the
    start-up field gp_vtk_write lays down itself."""
    from gp_cases import PARITY_CASES
    c = PARITY_CASES["dirsolid_binary"]
    ip, fp = write_case(str(tmp_path), "n", dict(c["kw"], shift=shift, shiftj=20, ascii=ascii, writecomposition=wc),
                        seeds=c["seeds"], cubes=c["cubes"])
    ref_dir = tmp_path / "ref"
    ref_dir.mkdir()
    _run([HARNESS, os.path.abspath(ip), os.path.abspath(fp), "vtk", str(steps), "n"], ref_dir)
    p = gp.load_params(ip)
    phi, mu = gp.fill(p, fp)
    o = Oracle(p, recip_div=0)
    o.set(phi, mu)
    o.smooth(p.nsmooth - 1)
    o.step(steps)
    if shift:
        assert o.stats()["shift_offset"] > 0
    ph, m = o.get()
    ours = str(tmp_path / "ours.vtk")
    gp.vtk_write(p, ours, ph, m, temperature=o.temperature() if steps else None)
    a = open(ours, "rb").read()
    b = (ref_dir / "DATA" / ("n_%d.vtk" % steps)).read_bytes()
    assert b"SCALARS Temperature double 1" in b
    assert a == b, "first difference at byte %d of %d/%d" % (
        next((i for i, (x, y) in enumerate(zip(a, b)) if x != y), min(len(a), len(b))), len(a), len(b))
    # the reader takes phi and mu and passes over the fields after them
    ph2, m2 = gp.vtk_read(p, ours)
    if ascii:
        rnd = np.vectorize(lambda v: float("%e" % v))
        ph, m = rnd(ph), rnd(m)
    assert bits_equal(ph2, ph) and bits_equal(m2, m)


@pytest.mark.parametrize("ascii", [0, 1])
def test_vtk_read_round_trip(tmp_path, ascii):
    """gp_vtk_read returns what gp_vtk_write wrote: the same bits in binary,
    the '%le'-rounded values in ASCII."""
    ip, fp = _deck(tmp_path, "r", ascii)
    p = gp.load_params(ip)
    phi, mu = gp.fill(p, fp)
    rng = np.random.default_rng(3)
    phi = phi + 1e-3 * rng.standard_normal(phi.shape)
    mu = mu + 1e-3 * rng.standard_normal(mu.shape)
    path = str(tmp_path / "state.vtk")
    gp.vtk_write(p, path, phi, mu)
    ph2, mu2 = gp.vtk_read(p, path)
    if ascii:
        rnd = np.vectorize(lambda v: float("%e" % v))
        phi, mu = rnd(phi), rnd(mu)
    assert bits_equal(ph2, phi), mismatch_report(ph2, phi)
    assert bits_equal(mu2, mu), mismatch_report(mu2, mu)


@needs_ref
@pytest.mark.parametrize("ascii", [0, 1])
def test_vtk_read_of_reference_file(tmp_path, ascii):
    """A file the reference wrote reads back as the reference's state (bit for
    bit from binary, at '%le' precision from ASCII)."""
    ip, fp = _deck(tmp_path, "x", ascii)
    ref_dir = tmp_path / "ref"
    ref_dir.mkdir()
    _run([HARNESS, os.path.abspath(ip), os.path.abspath(fp), "vtk", "7", "x"], ref_dir)
    p = gp.load_params(ip)
    ph, mu = gp.vtk_read(p, str(ref_dir / "DATA" / "x_7.vtk"))
    phi0, mu0 = gp.fill(p, fp)
    o = Oracle(p, recip_div=0)
    o.set(phi0, mu0)
    o.smooth(p.nsmooth - 1)
    o.step(7)
    oph, omu = o.get()
    if ascii:
        rnd = np.vectorize(lambda v: float("%e" % v))
        oph, omu = rnd(oph), rnd(omu)
    assert bits_equal(ph, oph), mismatch_report(ph, oph)
    assert bits_equal(mu, omu), mismatch_report(mu, omu)


def _progress(text):
    """(time lines, record lines) of a progress log (the reference also prints
    its parser's complaints about keys it does not know)"""
    lines = [ln for ln in text.splitlines() if ln.strip()]
    return [ln for ln in lines if ln.startswith("Time=")], [ln for ln in lines if ", Max = " in ln]


@pytest.mark.gpu
@needs_ref
@pytest.mark.parametrize("ascii", [0, 1])
def test_cli_matches_reference_main(tmp_path, ascii):
    """gp_microsim against the reference's main() on the same deck: the same
    DATA/NAME_<t>.vtk files byte for byte (t = 0, 20, 40), the same
    DATA/shift.dat and the same progress times; then both restart from the
    t=20 file (STARTTIME=20, RESTART=1) and again write the same t=40 file."""
    ip, fp = _deck(tmp_path, "c", ascii)
    runs = {}
    for who in ("ref", "ours"):
        d = tmp_path / who
        d.mkdir()
        if who == "ref":
            r = _run([HARNESS, os.path.abspath(ip), os.path.abspath(fp), "main", "c"], d)
        else:
            r = _run([CLI, os.path.abspath(ip), os.path.abspath(fp), "c"], d)
        runs[who] = (d, r.stdout)
    for t in (0, 20, 40):
        a = (runs["ours"][0] / "DATA" / ("c_%d.vtk" % t)).read_bytes()
        b = (runs["ref"][0] / "DATA" / ("c_%d.vtk" % t)).read_bytes()
        assert a == b, "DATA/c_%d.vtk differs" % t
    assert (runs["ours"][0] / "DATA" / "shift.dat").read_text() == (runs["ref"][0] / "DATA" / "shift.dat").read_text()
    assert _progress(runs["ours"][1])[0] == _progress(runs["ref"][1])[0]
    assert len(_progress(runs["ours"][1])[1]) == len(_progress(runs["ref"][1])[1])

    # restart from the t=20 file written by each program
    ip2, _ = _deck(tmp_path / "restart_deck", "c", ascii, ntimesteps=20, savet=20, starttime=20, restart=1)
    for who in ("ref", "ours"):
        d = tmp_path / (who + "_restart")
        (d / "DATA").mkdir(parents=True)
        shutil.copy(runs[who][0] / "DATA" / "c_20.vtk", d / "DATA" / "c_20.vtk")
        if who == "ref":
            _run([HARNESS, os.path.abspath(ip2), os.path.abspath(fp), "main", "c"], d)
        else:
            _run([CLI, os.path.abspath(ip2), os.path.abspath(fp), "c"], d)
    a = (tmp_path / "ours_restart" / "DATA" / "c_40.vtk").read_bytes()
    b = (tmp_path / "ref_restart" / "DATA" / "c_40.vtk").read_bytes()
    assert a == b, "restarted DATA/c_40.vtk differs"
    assert not (tmp_path / "ours_restart" / "DATA" / "c_0.vtk").exists()


@pytest.mark.gpu
@needs_ref
def test_cli_directional_moving_frame_matches_reference_main(tmp_path):
    """Directional solidification with the moving frame through gp_microsim and
    through the reference's main(): the same DATA/NAME_<t>.vtk files (t = 0,
    100, 200) and the same DATA/shift.dat (frame positions); then a restart
    from t = 100 (which reads the frame position back from DATA/shift.dat and
    resumes the temperature field) writes the same t = 200 file in both."""
    from gp_cases import PARITY_CASES
    c = PARITY_CASES["dirsolid_binary"]

    def deck(d, ntimesteps, starttime=0, restart=0):
        ip, fp = write_case(str(d), "f", dict(c["kw"], shift=True, shiftj=20, ascii=0, ntimesteps=ntimesteps),
                            seeds=c["seeds"], cubes=c["cubes"])
        text = open(ip).read()
        text = text.replace("SAVET = %d;" % ntimesteps, "SAVET = 100;")
        text = text.replace("STARTTIME = 0;", "STARTTIME = %d;" % starttime)
        text = text.replace("RESTART = 0;", "RESTART = %d;" % restart)
        open(ip, "w").write(text)
        return ip, fp

    ip, fp = deck(tmp_path / "deck", 200)
    dirs = {}
    for who in ("ref", "ours"):
        d = tmp_path / who
        d.mkdir()
        cmd = [HARNESS, os.path.abspath(ip), os.path.abspath(fp), "main", "f"] if who == "ref" else \
            [CLI, os.path.abspath(ip), os.path.abspath(fp), "f"]
        _run(cmd, d)
        dirs[who] = d
    for t in (0, 100, 200):
        a = (dirs["ours"] / "DATA" / ("f_%d.vtk" % t)).read_bytes()
        b = (dirs["ref"] / "DATA" / ("f_%d.vtk" % t)).read_bytes()
        assert a == b, "DATA/f_%d.vtk differs" % t
    shift_ref = (dirs["ref"] / "DATA" / "shift.dat").read_text()
    assert (dirs["ours"] / "DATA" / "shift.dat").read_text() == shift_ref
    assert int(shift_ref.split()[1]) > 0   # the frame moved

    ip2, _ = deck(tmp_path / "deck2", 100, starttime=100, restart=1)
    for who in ("ref", "ours"):
        d = tmp_path / (who + "_restart")
        (d / "DATA").mkdir(parents=True)
        shutil.copy(dirs[who] / "DATA" / "f_100.vtk", d / "DATA" / "f_100.vtk")
        shutil.copy(dirs[who] / "DATA" / "shift.dat", d / "DATA" / "shift.dat")
        cmd = [HARNESS, os.path.abspath(ip2), os.path.abspath(fp), "main", "f"] if who == "ref" else \
            [CLI, os.path.abspath(ip2), os.path.abspath(fp), "f"]
        _run(cmd, d)
    a = (tmp_path / "ours_restart" / "DATA" / "f_200.vtk").read_bytes()
    b = (tmp_path / "ref_restart" / "DATA" / "f_200.vtk").read_bytes()
    assert a == b, "restarted DATA/f_200.vtk differs"
    assert (tmp_path / "ours_restart" / "DATA" / "shift.dat").read_text() == \
        (tmp_path / "ref_restart" / "DATA" / "shift.dat").read_text()
