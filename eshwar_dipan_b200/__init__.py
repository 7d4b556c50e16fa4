"""eshwar_dipan_b200 -- MicroSim's 2D grand-potential finite-difference step on B200.

Python side of libgp (include/gp.h).  The physics runs in hand-written sm_100a
CUDA kernels behind the C ABI; this module only marshals arguments:

    p = load_params("Input.in")                 # reading_input_parameters()
    phi, mu = fill(p, "Filling.in")             # fill_domain()
    sim = Simulation(p, phi, mu)                # gp_init on the current device
    sim.smooth(p.nsmooth - 1)                   # preconditioning sweeps
    stats = sim.step(1000)                      # time steps
    phi, mu = sim.get()

Arrays are float64 numpy arrays shaped (N, MESH_X, MESH_Y) and (K, MESH_X, MESH_Y),
y contiguous, as in the reference's VTK output.
"""
import ctypes

import numpy as np

from ._abi import (GP_ENONFINITE, GP_ETIMEOUT, GP_FP32, GP_FP64, AdjOut, AdjReq, GpError, KernelTimes,
                   NonFiniteError, Params, Stats, check, lib)

__all__ = ["Params", "Stats", "GpError", "NonFiniteError", "Simulation", "Batch", "load_params", "fill", "vtk_write", "vtk_read",
           "GP_FP64", "GP_FP32", "version"]


def version():
    return lib().gp_version().decode()


def _ptr(a):
    return a.ctypes.data_as(ctypes.c_void_p)


def load_params(path):
    """Parse an Input.in file (gp_params_load)."""
    p = Params()
    check(lib().gp_params_load(ctypes.byref(p), str(path).encode()))
    return p


def _shapes(p):
    return (p.numphases, p.mesh_x, p.mesh_y), (p.numcomponents - 1, p.mesh_x, p.mesh_y)


def fill(p, filling_path):
    """Initial interior fields from a Filling.in file (gp_fill)."""
    sp, sm = _shapes(p)
    phi = np.zeros(sp, dtype=np.float64)
    mu = np.zeros(sm, dtype=np.float64)
    check(lib().gp_fill(ctypes.byref(p), str(filling_path).encode(), _ptr(phi), _ptr(mu)))
    return phi, mu


def vtk_write(p, path, phi, mu, ascii=None, temperature=None):
    """gp_vtk_write / gp_vtk_write_temperature: a non-isothermal run also
    writes its temperature field ([MESH_X][MESH_Y]; None = the field laid
    down at start-up)."""
    phi = np.ascontiguousarray(phi, dtype=np.float64)
    mu = np.ascontiguousarray(mu, dtype=np.float64)
    a = p.ascii if ascii is None else int(ascii)
    if temperature is None:
        check(lib().gp_vtk_write(ctypes.byref(p), str(path).encode(), _ptr(phi), _ptr(mu), a))
        return
    T = np.ascontiguousarray(temperature, dtype=np.float64)
    if T.shape != (p.mesh_x, p.mesh_y):
        raise ValueError("temperature must be [MESH_X][MESH_Y]")
    check(lib().gp_vtk_write_temperature(ctypes.byref(p), str(path).encode(), _ptr(phi), _ptr(mu), _ptr(T), a))


def vtk_read(p, path, ascii=None):
    sp, sm = _shapes(p)
    phi = np.zeros(sp, dtype=np.float64)
    mu = np.zeros(sm, dtype=np.float64)
    a = p.ascii if ascii is None else int(ascii)
    check(lib().gp_vtk_read(ctypes.byref(p), str(path).encode(), _ptr(phi), _ptr(mu), a))
    return phi, mu


def _adj_result(out, g_phi, g_mu):
    return {"loss": out.loss, "d_tau": out.d_tau, "d_dab": out.d_dab, "d_epsilon": out.d_epsilon,
            "d_gamma": out.d_gamma, "phi0_bar": g_phi, "mu0_bar": g_mu,
            "ms_forward": out.ms_forward, "ms_reverse": out.ms_reverse,
            "snapshots": out.snapshots, "recomputed": out.recomputed}


class Simulation:
    """One simulation resident on the current CUDA device (a gp_ctx)."""

    def __init__(self, params, phi, mu, precision=GP_FP64):
        self.params = params
        self.N, self.K = params.numphases, params.numcomponents - 1
        sp, sm = _shapes(params)
        phi = np.ascontiguousarray(phi, dtype=np.float64)
        mu = np.ascontiguousarray(mu, dtype=np.float64)
        if phi.shape != sp or mu.shape != sm:
            raise ValueError("phi/mu shapes %s/%s, expected %s/%s" % (phi.shape, mu.shape, sp, sm))
        h = ctypes.c_void_p()
        check(lib().gp_init(ctypes.byref(h), ctypes.byref(params), _ptr(phi), _ptr(mu), int(precision)))
        self._h = h

    @classmethod
    def from_tensors(cls, params, phi, mu, precision=GP_FP64):
        """A simulation whose start state comes from float64 CUDA tensors
        (gp_set_dev after a gp_init of zeros): the fields are copied on the
        device, not through host memory."""
        sp, sm = _shapes(params)
        sim = cls(params, np.zeros(sp), np.zeros(sm), precision)
        sim.set_tensors(phi, mu)
        return sim

    @property
    def handle(self):
        return self._h

    def smooth(self, n):
        check(lib().gp_smooth(self._h, int(n)), self._h)

    def step(self, n, stats=True):
        """n time steps; with stats, the progress record of the last one.
        Raises NonFiniteError (carrying that record) when the state then
        holds non-finite cells."""
        if stats:
            s = Stats()
            rc = lib().gp_step(self._h, int(n), ctypes.byref(s))
            if rc == GP_ENONFINITE:
                raise NonFiniteError(rc, lib().gp_last_error(self._h).decode(), s.as_dict(self.N, self.K))
            check(rc, self._h)
            return s.as_dict(self.N, self.K)
        check(lib().gp_step(self._h, int(n), None), self._h)
        return None

    def step_timed(self, n, stats=False, split=False):
        """Steps with device timing: (total_ms, bulk_kernel_ms, interface_kernel_ms, stats).
        The per-kernel times are measured only with split=True (the steps then
        run one by one instead of as CUDA graphs) and are None otherwise."""
        tot, a, b = ctypes.c_double(), ctypes.c_double(), ctypes.c_double()
        s = Stats() if stats else None
        check(lib().gp_step_timed(self._h, int(n), ctypes.byref(s) if stats else None, ctypes.byref(tot),
                                  ctypes.byref(a) if split else None, ctypes.byref(b) if split else None),
              self._h)
        return (tot.value, a.value if split else None, b.value if split else None,
                s.as_dict(self.N, self.K) if stats else None)

    def stats(self):
        """gp_get_stats: the progress record of the last step that asked for one"""
        s = Stats()
        check(lib().gp_get_stats(self._h, ctypes.byref(s)), self._h)
        return s.as_dict(self.N, self.K)

    def kernel_times(self, n):
        """gp_step_kernel_times: n steps launched one by one with events around
        each kernel of the launch shape in use; a dict of summed milliseconds
        (classify_ms and step_ms for the fused shape, bulk_ms and iface_ms for
        the two-launch shape) and launches_per_step."""
        t = KernelTimes()
        check(lib().gp_step_kernel_times(self._h, int(n), ctypes.byref(t)), self._h)
        return {"classify_ms": t.classify_ms, "step_ms": t.step_ms, "bulk_ms": t.bulk_ms, "iface_ms": t.iface_ms,
                "launches_per_step": t.launches_per_step, "fused": bool(t.fused)}

    def get(self):
        sp, sm = _shapes(self.params)
        phi = np.zeros(sp, dtype=np.float64)
        mu = np.zeros(sm, dtype=np.float64)
        check(lib().gp_get(self._h, _ptr(phi), _ptr(mu)), self._h)
        return phi, mu

    def get_tensors(self):
        """gp_get_dev: the state as float64 CUDA tensors on the current
        device, copied on the device"""
        import torch
        sp, sm = _shapes(self.params)
        phi = torch.empty(sp, dtype=torch.float64, device="cuda")
        mu = torch.empty(sm, dtype=torch.float64, device="cuda")
        torch.cuda.current_stream().synchronize()   # the buffers are allocated
        check(lib().gp_get_dev(self._h, ctypes.c_void_p(phi.data_ptr()), ctypes.c_void_p(mu.data_ptr())), self._h)
        return phi, mu

    def set_tensors(self, phi, mu):
        """gp_set_dev: the state from float64 CUDA tensors on the context's
        device, copied on the device"""
        import torch
        sp, sm = _shapes(self.params)
        phi = phi.detach().to(torch.float64).contiguous()
        mu = mu.detach().to(torch.float64).contiguous()
        if tuple(phi.shape) != sp or tuple(mu.shape) != sm:
            raise ValueError("phi/mu shapes %s/%s, expected %s/%s" % (tuple(phi.shape), tuple(mu.shape), sp, sm))
        torch.cuda.current_stream().synchronize()   # the tensors are written
        check(lib().gp_set_dev(self._h, ctypes.c_void_p(phi.data_ptr()), ctypes.c_void_p(mu.data_ptr())), self._h)

    def adjoint(self, nsteps, target_phi=None, phi_bar=None, mu_bar=None, checkpoint_every=0, snapshots=0):
        """gp_adjoint: run nsteps from the current state (the simulation ends at
        the final state) and return a dict with the loss (with target_phi), the
        parameter gradients d_tau, d_dab, d_epsilon, d_gamma (phase pair 0,1),
        phi0_bar / mu0_bar (gradient with respect to the start state), the
        device times of the two passes, the states kept and the steps
        recomputed.  The arrays may be numpy arrays or, all of them, CUDA
        tensors on the context's device (the gradients then come back as CUDA
        tensors, without a copy through host memory)."""
        sp, sm = _shapes(self.params)
        given = [a for a in (target_phi, phi_bar, mu_bar) if a is not None]
        if given and all(getattr(a, "is_cuda", False) for a in given):
            return self._adjoint_dev(nsteps, target_phi, phi_bar, mu_bar, checkpoint_every, snapshots)
        req = AdjReq()
        req.nsteps = int(nsteps)
        req.checkpoint_every = int(checkpoint_every)
        req.snapshots = int(snapshots)
        keep = []
        if phi_bar is not None:
            a = np.ascontiguousarray(phi_bar, dtype=np.float64)
            keep.append(a)
            req.phi_bar = a.ctypes.data
            if mu_bar is not None:
                m = np.ascontiguousarray(mu_bar, dtype=np.float64)
                keep.append(m)
                req.mu_bar = m.ctypes.data
        elif target_phi is not None:
            t = np.ascontiguousarray(target_phi, dtype=np.float64)
            keep.append(t)
            req.target_phi = t.ctypes.data
        else:
            raise ValueError("give target_phi or phi_bar")
        out = AdjOut()
        g_phi = np.zeros(sp, dtype=np.float64)
        g_mu = np.zeros(sm, dtype=np.float64)
        out.phi0_bar = g_phi.ctypes.data
        out.mu0_bar = g_mu.ctypes.data
        check(lib().gp_adjoint(self._h, ctypes.byref(req), ctypes.byref(out)), self._h)
        return _adj_result(out, g_phi, g_mu)

    def _adjoint_dev(self, nsteps, target_phi, phi_bar, mu_bar, checkpoint_every, snapshots):
        import torch
        sp, sm = _shapes(self.params)
        req = AdjReq()
        req.nsteps = int(nsteps)
        req.checkpoint_every = int(checkpoint_every)
        req.snapshots = int(snapshots)
        req.device = 1
        keep = []

        def dptr(t, shape):
            t = t.detach().to(torch.float64).contiguous()
            if tuple(t.shape) != shape:
                raise ValueError("shape %s, expected %s" % (tuple(t.shape), shape))
            keep.append(t)
            return t.data_ptr()
        if phi_bar is not None:
            req.phi_bar = dptr(phi_bar, sp)
            if mu_bar is not None:
                req.mu_bar = dptr(mu_bar, sm)
        elif target_phi is not None:
            req.target_phi = dptr(target_phi, sp)
        else:
            raise ValueError("give target_phi or phi_bar")
        dev = keep[0].device
        g_phi = torch.zeros(sp, dtype=torch.float64, device=dev)
        g_mu = torch.zeros(sm, dtype=torch.float64, device=dev)
        out = AdjOut()
        out.phi0_bar = g_phi.data_ptr()
        out.mu0_bar = g_mu.data_ptr()
        torch.cuda.current_stream(dev).synchronize()   # the inputs are written
        check(lib().gp_adjoint(self._h, ctypes.byref(req), ctypes.byref(out)), self._h)
        return _adj_result(out, g_phi, g_mu)

    def adjoint_replay(self, nsteps):
        """gp_adjoint_replay: (max |difference|, number of differing values)
        between the adjoint's cell functions and the step kernels over nsteps."""
        d = ctypes.c_double()
        n = ctypes.c_longlong()
        check(lib().gp_adjoint_replay(self._h, int(nsteps), ctypes.byref(d), ctypes.byref(n)), self._h)
        return d.value, n.value

    def set(self, phi, mu):
        phi = np.ascontiguousarray(phi, dtype=np.float64)
        mu = np.ascontiguousarray(mu, dtype=np.float64)
        check(lib().gp_set(self._h, _ptr(phi), _ptr(mu)), self._h)

    def temperature(self):
        """gp_temperature: the interior temperature field [MESH_X][MESH_Y]
        after the steps taken so far."""
        T = np.zeros((self.params.mesh_x, self.params.mesh_y), dtype=np.float64)
        check(lib().gp_temperature(self._h, _ptr(T)), self._h)
        return T

    def vtk_write_async(self, path, ascii=None):
        """gp_vtk_write_async: write the current state to `path` in the
        background while stepping goes on; complete after vtk_wait()."""
        a = self.params.ascii if ascii is None else int(ascii)
        check(lib().gp_vtk_write_async(self._h, str(path).encode(), a), self._h)

    def vtk_wait(self):
        check(lib().gp_vtk_wait(self._h), self._h)

    def close(self):
        if getattr(self, "_h", None):
            lib().gp_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()


def _bcheck(code, h):
    if code != 0:
        m = lib().gp_batch_last_error(h)
        raise GpError(code, m.decode() if m else "")


class Batch:
    """Many independent simulations stepped together (gp_batch_*): grids of any
    size and their own parameters; same NUMPHASES, NUMCOMPONENTS and
    Function_anisotropy.  precision=GP_FP32 stores and steps the fields in
    float with the dc/dmu inversion and all sums in FP64."""

    def __init__(self, params_list, fields, precision=GP_FP32):
        n = len(params_list)
        if n < 1 or len(fields) != n:
            raise ValueError("need one (phi, mu) pair per parameter set")
        self.params = list(params_list)
        arr = (Params * n)(*self.params)
        self._keep = []
        phis = (ctypes.c_void_p * n)()
        mus = (ctypes.c_void_p * n)()
        for s, ((phi, mu), p) in enumerate(zip(fields, self.params)):
            sp, sm = _shapes(p)
            phi = np.ascontiguousarray(phi, dtype=np.float64)
            mu = np.ascontiguousarray(mu, dtype=np.float64)
            if phi.shape != sp or mu.shape != sm:
                raise ValueError("simulation %d: shapes %s/%s, expected %s/%s" % (s, phi.shape, mu.shape, sp, sm))
            self._keep += [phi, mu]
            phis[s] = phi.ctypes.data
            mus[s] = mu.ctypes.data
        h = ctypes.c_void_p()
        _bcheck(lib().gp_batch_create(ctypes.byref(h), n, arr, phis, mus, int(precision)), None)
        self._keep = []
        self._h = h
        self.n = n
        self.N, self.K = self.params[0].numphases, self.params[0].numcomponents - 1

    def smooth(self, n):
        _bcheck(lib().gp_batch_smooth(self._h, int(n)), self._h)

    def step(self, n, stats=True):
        if stats:
            s = (Stats * self.n)()
            rc = lib().gp_batch_step(self._h, int(n), s)
            if rc == GP_ENONFINITE:
                raise NonFiniteError(rc, lib().gp_batch_last_error(self._h).decode(),
                                     [x.as_dict(self.N, self.K) for x in s])
            _bcheck(rc, self._h)
            return [x.as_dict(self.N, self.K) for x in s]
        _bcheck(lib().gp_batch_step(self._h, int(n), None), self._h)
        return None

    def step_timed(self, n, stats=False):
        ms = ctypes.c_double()
        s = (Stats * self.n)() if stats else None
        _bcheck(lib().gp_batch_step_timed(self._h, int(n), s, ctypes.byref(ms)), self._h)
        return ms.value, ([x.as_dict(self.N, self.K) for x in s] if stats else None)

    def get(self, sim):
        sp, sm = _shapes(self.params[sim])
        phi = np.zeros(sp, dtype=np.float64)
        mu = np.zeros(sm, dtype=np.float64)
        _bcheck(lib().gp_batch_get(self._h, int(sim), _ptr(phi), _ptr(mu)), self._h)
        return phi, mu

    def set(self, sim, phi, mu):
        phi = np.ascontiguousarray(phi, dtype=np.float64)
        mu = np.ascontiguousarray(mu, dtype=np.float64)
        _bcheck(lib().gp_batch_set(self._h, int(sim), _ptr(phi), _ptr(mu)), self._h)

    def close(self):
        if getattr(self, "_h", None):
            lib().gp_batch_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
