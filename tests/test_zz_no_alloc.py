"""gp_step_noalloc: the one time step that allocates nothing.

It serves callers that cannot call cudaMalloc (applications owning all device
memory through their own pool, or running under a fixed memory budget).  They
hand in their own device buffers; the step's scratch lives in a fixed array
inside libgp.  These checks call it through the C ABI on buffers the test owns
and compare with the context-based gp_step, bit for bit, on two calls in a row.
This file is collected last (test_zz_*) so that a run stopping at the first
failure has already run every other test.
"""
import ctypes

import numpy as np
import pytest

import eshwar_dipan_b200 as gp
from eshwar_dipan_b200 import _abi
from eshwar_dipan_b200.workloads import write_case


def _bits_equal(a, b):
    a = np.ascontiguousarray(a) + 0.0
    b = np.ascontiguousarray(b) + 0.0
    return np.array_equal(a.view(np.int64), b.view(np.int64))


# The caller's planes have no row padding (pitch = MESH_Y), unlike a
# context's; odd sizes check that layout on ragged tiles.
CASES = {
    "ternary3_aniso": (dict(N=3, K=2, mesh=(40, 44), dab=0.02, bc_phi=(3, 3, 3, 3), A_off=0.25),
                       [(0, 12, 12, 6.0), (1, 28, 26, 6.5)]),
    "binary_iso_neumann": (dict(N=2, K=1, mesh=(48, 40), aniso=False, dab=0.0, d_solid=0.0),
                           [(0, 24, 20, 9.0), (0, 2, 5, 5.0)]),
    "binary_aniso_odd": (dict(N=2, K=1, mesh=(37, 41), dab=0.03, bc_phi=(3, 3, 1, 1), d_solid=0.0),
                         [(0, 18, 20, 7.5), (0, 1, 39, 4.0)]),
    "four_phase_ternary_aniso_odd": (dict(N=4, K=2, mesh=(39, 45), dab=0.02, bc_phi=(1, 1, 3, 3)),
                                     [(0, 10, 12, 6.0), (1, 26, 14, 6.0), (2, 19, 33, 6.5)]),
}


@pytest.mark.gpu
@pytest.mark.parametrize("name", sorted(CASES))
def test_noalloc_matches_gp_step_twice(tmp_path, name):
    import torch
    kw, seeds = CASES[name]
    ip, fp = write_case(str(tmp_path), name, kw, seeds=seeds)
    p = gp.load_params(ip)
    phi, mu = gp.fill(p, fp)

    # existing entry point: a context with its own device buffers
    sim = gp.Simulation(p, phi, mu)
    sim.step(1, stats=False)
    ref1 = sim.get()
    sim.step(1, stats=False)
    ref2 = sim.get()
    sim.close()

    # caller-owned device buffers, two calls in a row (in -> out -> in)
    L = _abi.lib()
    dev = torch.device("cuda", torch.cuda.current_device())
    a_phi = torch.from_numpy(phi.copy()).to(dev)
    a_mu = torch.from_numpy(mu.copy()).to(dev)
    b_phi = torch.full_like(a_phi, float("nan"))
    b_mu = torch.full_like(a_mu, float("nan"))
    stream = torch.cuda.current_stream(dev)
    rc = L.gp_step_noalloc(ctypes.byref(p), a_phi.data_ptr(), a_mu.data_ptr(), b_phi.data_ptr(), b_mu.data_ptr(),
                           ctypes.c_void_p(stream.cuda_stream))
    assert rc == 0, L.gp_last_error(None)
    stream.synchronize()
    assert _bits_equal(b_phi.cpu().numpy(), ref1[0])
    assert _bits_equal(b_mu.cpu().numpy(), ref1[1])
    rc = L.gp_step_noalloc(ctypes.byref(p), b_phi.data_ptr(), b_mu.data_ptr(), a_phi.data_ptr(), a_mu.data_ptr(),
                           ctypes.c_void_p(stream.cuda_stream))
    assert rc == 0, L.gp_last_error(None)
    stream.synchronize()
    assert _bits_equal(a_phi.cpu().numpy(), ref2[0])
    assert _bits_equal(a_mu.cpu().numpy(), ref2[1])


@pytest.mark.gpu
def test_noalloc_rejects_grids_beyond_its_scratch(tmp_path):
    ip, fp = write_case(str(tmp_path), "big", dict(N=3, K=2, mesh=(2048, 2048)), seeds=[(0, 10, 10, 4.0)])
    p = gp.load_params(ip)
    L = _abi.lib()
    one = ctypes.c_void_p(16)
    two = ctypes.c_void_p(32)
    rc = L.gp_step_noalloc(ctypes.byref(p), one, one, two, two, None)
    assert rc == _abi.GP_EINVAL
    assert b"fixed maximum" in L.gp_last_error(None)


def test_noalloc_rejects_overlapping_buffers(tmp_path):
    """An output that shares any byte with an input, or with the other output,
    is refused before anything reaches the GPU (so this runs without one):
    the step reads neighbours of cells whose outputs are already written."""
    ip, fp = write_case(str(tmp_path), "small", dict(N=3, K=2, mesh=(40, 44)), seeds=[(0, 10, 10, 4.0)])
    p = gp.load_params(ip)
    L = _abi.lib()
    cells = 40 * 44
    base = 1 << 20
    phi_in, mu_in = base, base + 3 * cells * 8
    far = base + 64 * cells * 8
    cases = {
        "phi_out inside phi_in": (phi_in, mu_in, phi_in + 8 * cells, far),
        "phi_out tail over mu_in": (phi_in, mu_in, mu_in - 3 * cells * 8 + 8, far),
        "mu_out head in phi_in": (phi_in, mu_in, far, phi_in + 3 * cells * 8 - 8),
        "outputs overlap": (phi_in, mu_in, far, far + 3 * cells * 8 - 16),
    }
    for what, (a, b, c, d) in cases.items():
        rc = L.gp_step_noalloc(ctypes.byref(p), ctypes.c_void_p(a), ctypes.c_void_p(b), ctypes.c_void_p(c),
                               ctypes.c_void_p(d), None)
        assert rc == _abi.GP_EINVAL, what
        assert b"overlap" in L.gp_last_error(None), what
