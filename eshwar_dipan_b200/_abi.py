"""ctypes mirror of include/gp.h and loader for the in-tree libgp.so.

The library is the product: every call here goes to the sm_100a kernels behind
the C ABI.  There is no Python or CPU fallback; if libgp.so is missing the
import fails with an explicit error.
"""
import ctypes
import os
from ctypes import POINTER, c_char, c_double, c_int, c_long, c_longlong, c_size_t, c_void_p

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libgp.so")

GP_MAX_PHASES = 6
GP_MAX_COMP = 4
GP_NAME_LEN = 52

GP_OK, GP_EINVAL, GP_ENOMEM, GP_ECUDA, GP_ETIMEOUT, GP_ENONFINITE, GP_EIO, GP_EUNSUPPORTED = 0, -1, -2, -3, -4, -5, -6, -7
GP_FP64, GP_FP32 = 0, 1

_MN = GP_MAX_PHASES
_MK = GP_MAX_COMP


def _arr(t, *dims):
    for d in reversed(dims):
        t = t * d
    return t


class Params(ctypes.Structure):
    """gp_params (include/gp.h)."""
    _fields_ = [
        ("dimension", c_int),
        ("mesh_x", c_long), ("mesh_y", c_long), ("mesh_z", c_long),
        ("deltax", c_double), ("deltay", c_double), ("deltaz", c_double), ("deltat", c_double),
        ("numphases", c_int), ("numcomponents", c_int),
        ("ntimesteps", c_long), ("savet", c_long), ("nsmooth", c_long), ("starttime", c_long),
        ("restart", c_long), ("track_progress", c_long),
        ("R", c_double), ("V", c_double), ("T", c_double), ("Teq", c_double), ("Tfill", c_double),
        ("temperature_scale", c_double), ("tilt_angle", c_double), ("Rtheta", c_double),
        ("epsilon", c_double), ("tau", c_double),
        ("function_f", c_int), ("function_w", c_int), ("function_anisotropy", c_int), ("anisotropy_type", c_int),
        ("obstacle_key", c_int),
        ("isothermal", c_int), ("tempgrady", c_int), ("binary", c_int), ("ternary", c_int), ("dilute", c_int),
        ("shift", c_int), ("shiftj", c_int), ("writecomposition", c_int), ("noise_phasefield", c_int), ("ascii", c_int),
        ("amp_noise_phase", c_double),
        ("tempgrady_v", _arr(c_double, 5)),
        ("gamma", _arr(c_double, _MN, _MN)),
        ("tau_ab", _arr(c_double, _MN, _MN)),
        ("dab", _arr(c_double, _MN, _MN)),
        ("gamma_abc", _arr(c_double, _MN, _MN, _MN)),
        ("diffusivity", _arr(c_double, _MN, _MK, _MK)),
        ("A", _arr(c_double, _MN, _MK, _MK)),
        ("ceq", _arr(c_double, _MN, _MN, _MK)),
        ("cfill", _arr(c_double, _MN, _MN, _MK)),
        ("slopes", _arr(c_double, _MN, _MN, _MK)),
        ("rot_angles", _arr(c_double, _MN, _MN, 3)),
        ("rot_set", _arr(c_int, _MN, _MN)),
        ("bc_type", _arr(c_int, 3, 6)),
        ("bc_value", _arr(c_double, 3, 6)),
        ("bc_value_set", _arr(c_int, 3)),
        ("bc_proxy_type", _arr(c_int, 3, 6)),
        ("have_gamma", c_int), ("have_tau_ab", c_int), ("have_dab", c_int), ("have_gamma_abc", c_int),
        ("phases", _arr(c_char, _MN, GP_NAME_LEN)),
        ("components", _arr(c_char, _MK + 1, GP_NAME_LEN)),
    ]

    @property
    def N(self):
        return self.numphases

    @property
    def K(self):
        return self.numcomponents - 1


class Stats(ctypes.Structure):
    """gp_stats (include/gp.h)."""
    _fields_ = [
        ("phi_max", _arr(c_double, _MN)), ("phi_min", _arr(c_double, _MN)),
        ("mu_max", _arr(c_double, _MK)), ("mu_min", _arr(c_double, _MK)),
        ("rel_change_phi", _arr(c_double, _MN)), ("rel_change_mu", _arr(c_double, _MK)),
        ("phi_sum", _arr(c_double, _MN)),
        ("comp_sum", _arr(c_double, _MK)),
        ("nonfinite", c_longlong),
        ("steps_done", c_longlong),
        ("shift_offset", c_longlong),
    ]

    def as_dict(self, N, K):
        d = {}
        for name in ("phi_max", "phi_min", "rel_change_phi", "phi_sum"):
            d[name] = list(getattr(self, name))[:N]
        for name in ("mu_max", "mu_min", "rel_change_mu", "comp_sum"):
            d[name] = list(getattr(self, name))[:K]
        d["nonfinite"] = int(self.nonfinite)
        d["steps_done"] = int(self.steps_done)
        d["shift_offset"] = int(self.shift_offset)
        return d


class AdjReq(ctypes.Structure):
    """gp_adj_req (include/gp.h)."""
    _fields_ = [("nsteps", c_long), ("phi_bar", c_void_p), ("mu_bar", c_void_p), ("target_phi", c_void_p),
                ("checkpoint_every", c_long), ("snapshots", c_long), ("device", c_int)]


class AdjOut(ctypes.Structure):
    """gp_adj_out (include/gp.h)."""
    _fields_ = [("loss", c_double), ("d_tau", c_double), ("d_dab", c_double), ("d_epsilon", c_double),
                ("d_gamma", c_double), ("phi0_bar", c_void_p), ("mu0_bar", c_void_p),
                ("ms_forward", c_double), ("ms_reverse", c_double), ("snapshots", c_long), ("recomputed", c_long)]


class KernelTimes(ctypes.Structure):
    """gp_kernel_times (include/gp.h)."""
    _fields_ = [("classify_ms", c_double), ("step_ms", c_double), ("bulk_ms", c_double), ("iface_ms", c_double),
                ("launches_per_step", c_int), ("fused", c_int)]


# Every entry point declared in include/gp.h, with its ctypes signature.
SIGNATURES = {
    "gp_params_load": (c_int, [POINTER(Params), ctypes.c_char_p]),
    "gp_fill": (c_int, [POINTER(Params), ctypes.c_char_p, c_void_p, c_void_p]),
    "gp_vtk_write": (c_int, [POINTER(Params), ctypes.c_char_p, c_void_p, c_void_p, c_int]),
    "gp_vtk_write_temperature": (c_int, [POINTER(Params), ctypes.c_char_p, c_void_p, c_void_p, c_void_p, c_int]),
    "gp_temperature": (c_int, [c_void_p, c_void_p]),
    "gp_set_stat_rows": (c_int, [c_void_p, ctypes.c_long, ctypes.c_long]),
    "gp_rows_pack": (c_int, [c_void_p, c_int, c_void_p, c_void_p, c_void_p]),
    "gp_rows_unpack": (c_int, [c_void_p, c_int, c_void_p, c_void_p, c_void_p]),
    "gp_vtk_read": (c_int, [POINTER(Params), ctypes.c_char_p, c_void_p, c_void_p, c_int]),
    "gp_vtk_write_async": (c_int, [c_void_p, ctypes.c_char_p, c_int]),
    "gp_vtk_wait": (c_int, [c_void_p]),
    "gp_init": (c_int, [POINTER(c_void_p), POINTER(Params), c_void_p, c_void_p, c_int]),
    "gp_smooth": (c_int, [c_void_p, c_long]),
    "gp_step": (c_int, [c_void_p, c_long, POINTER(Stats)]),
    "gp_get": (c_int, [c_void_p, c_void_p, c_void_p]),
    "gp_set": (c_int, [c_void_p, c_void_p, c_void_p]),
    "gp_get_dev": (c_int, [c_void_p, c_void_p, c_void_p]),
    "gp_set_dev": (c_int, [c_void_p, c_void_p, c_void_p]),
    "gp_get_stats": (c_int, [c_void_p, POINTER(Stats)]),
    "gp_step_timed": (c_int, [c_void_p, c_long, POINTER(Stats), POINTER(c_double), POINTER(c_double),
                              POINTER(c_double)]),
    "gp_step_kernel_times": (c_int, [c_void_p, c_long, POINTER(KernelTimes)]),
    "gp_step_noalloc": (c_int, [POINTER(Params), c_void_p, c_void_p, c_void_p, c_void_p, c_void_p]),
    "gp_batch_create": (c_int, [POINTER(c_void_p), c_int, POINTER(Params), POINTER(c_void_p), POINTER(c_void_p),
                                c_int]),
    "gp_batch_smooth": (c_int, [c_void_p, c_long]),
    "gp_batch_step": (c_int, [c_void_p, c_long, POINTER(Stats)]),
    "gp_batch_step_timed": (c_int, [c_void_p, c_long, POINTER(Stats), POINTER(c_double)]),
    "gp_batch_get": (c_int, [c_void_p, c_int, c_void_p, c_void_p]),
    "gp_batch_set": (c_int, [c_void_p, c_int, c_void_p, c_void_p]),
    "gp_batch_size": (c_int, [c_void_p]),
    "gp_batch_last_error": (ctypes.c_char_p, [c_void_p]),
    "gp_batch_destroy": (None, [c_void_p]),
    "gp_adjoint": (c_int, [c_void_p, POINTER(AdjReq), POINTER(AdjOut)]),
    "gp_adjoint_replay": (c_int, [c_void_p, c_long, POINTER(c_double), POINTER(c_longlong)]),
    "gp_stream": (c_void_p, [c_void_p]),
    "gp_destroy": (None, [c_void_p]),
    "gp_last_error": (ctypes.c_char_p, [c_void_p]),
    "gp_version": (ctypes.c_char_p, []),
}

_lib = None


def lib():
    """Load libgp.so once; raise if it has not been built."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError(
                "libgp.so not found at %s; build it with `python -m eshwar_dipan_b200.build`" % LIB_PATH)
        L = ctypes.CDLL(LIB_PATH)
        for name, (res, args) in SIGNATURES.items():
            fn = getattr(L, name)
            fn.restype = res
            fn.argtypes = args
        L.gp_params_size.restype = c_size_t
        if L.gp_params_size() != ctypes.sizeof(Params):
            raise ImportError("gp_params layout mismatch: C %d bytes, Python %d bytes"
                              % (L.gp_params_size(), ctypes.sizeof(Params)))
        _lib = L
    return _lib


class GpError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__("libgp error %d: %s" % (code, msg))
        self.code = code


class NonFiniteError(GpError):
    """GP_ENONFINITE: the steps are done, but the state holds non-finite
    cells; `stats` is the progress record of the last step (per simulation
    for a batch)."""

    def __init__(self, code, msg, stats):
        super().__init__(code, msg)
        self.stats = stats


def check(code, ctx=None):
    if code != GP_OK:
        m = lib().gp_last_error(ctx)
        raise GpError(code, m.decode() if m else "")
