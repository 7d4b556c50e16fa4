"""Test-side drivers for the two oracles (never imported by the product):

* Oracle   -- oracle/liboracle.so, the CPU restatement of the reference step;
* RefRun   -- oracle/_ref/gp_ref_harness, the reference's own C sources built
              by oracle/Makefile (present only where the reference tree was
              available at build time).
"""
import ctypes
import os
import subprocess

import numpy as np

from eshwar_dipan_b200._abi import Params, Stats

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
ORACLE_SO = os.path.join(ROOT, "oracle", "liboracle.so")
HARNESS = os.path.join(ROOT, "oracle", "_ref", "gp_ref_harness")

_o = None


def olib():
    global _o
    if _o is None:
        if not os.path.exists(ORACLE_SO):
            subprocess.run(["make", "-C", os.path.join(ROOT, "oracle"), "oracle"], check=True,
                           capture_output=True)
        L = ctypes.CDLL(ORACLE_SO)
        L.gpo_create.restype = ctypes.c_void_p
        L.gpo_create.argtypes = [ctypes.POINTER(Params), ctypes.c_int, ctypes.c_char_p, ctypes.c_int]
        for n in ("gpo_destroy", "gpo_set", "gpo_get", "gpo_get_full", "gpo_smooth", "gpo_step",
                  "gpo_stats", "gpo_dims", "gpo_consts", "gpo_temperature"):
            getattr(L, n).argtypes = None
        L.gpo_smooth.argtypes = [ctypes.c_void_p, ctypes.c_long]
        L.gpo_step.argtypes = [ctypes.c_void_p, ctypes.c_long]
        _o = L
    return _o


def _p(a):
    return a.ctypes.data_as(ctypes.c_void_p)


class Oracle:
    def __init__(self, params, recip_div=1):
        err = ctypes.create_string_buffer(256)
        h = olib().gpo_create(ctypes.byref(params), int(recip_div), err, 256)
        if not h:
            raise RuntimeError(err.value.decode())
        self.h = ctypes.c_void_p(h)
        self.p = params
        self.N, self.K = params.numphases, params.numcomponents - 1
        self.mx, self.my = params.mesh_x, params.mesh_y

    def set(self, phi, mu):
        phi = np.ascontiguousarray(phi, dtype=np.float64)
        mu = np.ascontiguousarray(mu, dtype=np.float64)
        olib().gpo_set(self.h, _p(phi), _p(mu))

    def get(self):
        phi = np.zeros((self.N, self.mx, self.my))
        mu = np.zeros((self.K, self.mx, self.my))
        olib().gpo_get(self.h, _p(phi), _p(mu))
        return phi, mu

    def temperature(self):
        """the interior temperature field [mx][my] (gpo_temperature)"""
        T = np.zeros((self.mx, self.my), dtype=np.float64)
        olib().gpo_temperature(self.h, _p(T))
        return T

    def get_full(self):
        rx, ry = self.mx + 6, self.my + 6
        phi = np.zeros((self.N, rx, ry))
        mu = np.zeros((self.K, rx, ry))
        dphi = np.zeros((self.N, rx, ry))
        olib().gpo_get_full(self.h, _p(phi), _p(mu), _p(dphi))
        return phi, mu, dphi

    def smooth(self, n):
        olib().gpo_smooth(self.h, n)

    def step(self, n):
        olib().gpo_step(self.h, n)

    def stats(self):
        s = Stats()
        olib().gpo_stats(self.h, ctypes.byref(s))
        return s.as_dict(self.N, self.K)

    def consts(self):
        N, K = self.N, self.K
        cmu = np.zeros(N * K * K); B = np.zeros(N * K); C = np.zeros(N)
        Beq = np.zeros(N * K); dB = np.zeros(N * K); R = np.zeros(N * N * 9); Ri = np.zeros(N * N * 9)
        olib().gpo_consts(self.h, _p(cmu), _p(B), _p(C), _p(Beq), _p(dB), _p(R), _p(Ri))
        return dict(cmu=cmu.reshape(N, K, K), B=B.reshape(N, K), C=C, Beq=Beq.reshape(N, K),
                    dBbdT=dB.reshape(N, K), R=R.reshape(N, N, 3, 3), Rinv=Ri.reshape(N, N, 3, 3))

    def close(self):
        if self.h:
            olib().gpo_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def harness_available():
    return os.path.exists(HARNESS)


def _read_dump(path):
    raw = open(path, "rb").read()
    assert raw[:4] == b"GPRF"
    rx, ry, N, K = np.frombuffer(raw[4:20], dtype=np.int32)
    d = np.frombuffer(raw[20:], dtype=np.float64)
    n = rx * ry
    out = dict(phi=d[:N * n].reshape(N, rx, ry), mu=d[N * n:(N + K) * n].reshape(K, rx, ry),
               dphi=d[(N + K) * n:(2 * N + K) * n].reshape(N, rx, ry))
    rest = d[(2 * N + K) * n:]
    out["record"] = dict(phi_max=rest[:N], phi_min=rest[N:2 * N], mu_max=rest[2 * N:2 * N + K],
                         mu_min=rest[2 * N + K:2 * N + 2 * K])
    return out


def harness_run(inp, fill, nsmooth_iters, nsteps, workdir, tag="h"):
    """Reference: fill, BCs, nsmooth_iters smoothing sweeps, nsteps steps; full ghosted dump.
    The reference binary crashes at random at start-up (heap overflow in its
    boundary echo, avoided by the harness, and sscanf widths); retry a few times."""
    out = os.path.join(str(workdir), tag + ".bin")
    last = None
    for _ in range(4):
        r = subprocess.run([HARNESS, os.path.abspath(inp), os.path.abspath(fill), "run",
                            str(nsmooth_iters + 1), str(nsteps), out],
                           capture_output=True, text=True, cwd=str(workdir))
        if r.returncode == 0:
            return _read_dump(out)
        last = r
    raise RuntimeError("reference harness failed: rc=%s %s" % (last.returncode, last.stderr[-500:]))


def write_state(path, phi, mu):
    N, mx, my = phi.shape
    K = mu.shape[0]
    with open(path, "wb") as f:
        f.write(b"GPST")
        f.write(np.array([mx, my, N, K], dtype=np.int32).tobytes())
        f.write(np.ascontiguousarray(phi, dtype=np.float64).tobytes())
        f.write(np.ascontiguousarray(mu, dtype=np.float64).tobytes())


def harness_load(inp, fill, state_path, nsmooth_iters, nsteps, workdir, tag="hl"):
    out = os.path.join(str(workdir), tag + ".bin")
    for _ in range(4):
        r = subprocess.run([HARNESS, os.path.abspath(inp), os.path.abspath(fill), "load", state_path,
                            str(nsmooth_iters + 1), str(nsteps), out],
                           capture_output=True, text=True, cwd=str(workdir))
        if r.returncode == 0:
            return _read_dump(out)
    raise RuntimeError("reference harness failed: %s" % r.stderr[-500:])


def bits_equal(a, b):
    """Bit-for-bit equality, with -0.0 and +0.0 treated as equal."""
    a = np.ascontiguousarray(a, dtype=np.float64) + 0.0
    b = np.ascontiguousarray(b, dtype=np.float64) + 0.0
    return np.array_equal(a.view(np.int64), b.view(np.int64))


def mismatch_report(a, b):
    a = np.asarray(a) + 0.0
    b = np.asarray(b) + 0.0
    bad = a.view(np.int64) != b.view(np.int64)
    if not bad.any():
        return "identical"
    idx = np.argwhere(bad)
    d = np.abs(a - b)
    return "%d mismatches, first at %s, max |diff| %.3e" % (bad.sum(), tuple(idx[0]), np.nanmax(d))
