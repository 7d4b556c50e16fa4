"""The C-ABI library: loads without a GPU and exports every entry point that
include/gp.h declares; host-side calls work without a device."""
import ctypes
import os
import re

import numpy as np
import pytest

import eshwar_dipan_b200 as gp
from eshwar_dipan_b200 import _abi
from eshwar_dipan_b200.workloads import write_case

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    names = set()
    for fn in os.listdir(os.path.join(ROOT, "include")):
        if fn.endswith(".h"):
            text = open(os.path.join(ROOT, "include", fn)).read()
            text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
            names |= set(re.findall(r"\b(gp_[a-z0-9_]+)\s*\(", text))
    return names


def test_library_exports_every_declared_symbol():
    L = _abi.lib()
    names = declared_symbols()
    assert "gp_init" in names and "gp_step" in names and len(names) >= 15
    missing = [n for n in sorted(names) if not hasattr(L, n)]
    assert not missing, missing


def test_ctypes_mirror_matches_c_layout():
    assert _abi.lib().gp_params_size() == ctypes.sizeof(_abi.Params)
    # every declared entry point has a ctypes signature in the integrator
    assert declared_symbols() <= set(_abi.SIGNATURES) | {"gp_params_size"}


def test_init_without_device_fails_loudly(tmp_path):
    """On a machine without a CUDA device the device path reports GP_ECUDA; there
    is no CPU fallback."""
    try:
        import torch
        if torch.cuda.is_available():
            pytest.skip("a CUDA device is present")
    except ImportError:
        pass
    ip, fp = write_case(str(tmp_path), "c", dict(N=2, K=1, mesh=(16, 16)), seeds=[(0, 8, 8, 3.0)])
    p = gp.load_params(ip)
    phi, mu = gp.fill(p, fp)
    with pytest.raises(gp.GpError) as e:
        gp.Simulation(p, phi, mu)
    assert e.value.code == _abi.GP_ECUDA


def test_unsupported_parameters_rejected(tmp_path):
    ip, fp = write_case(str(tmp_path), "c", dict(N=2, K=1, mesh=(16, 16), bc_phi=(0, 0, 1, 1)),
                        seeds=[(0, 8, 8, 3.0)])
    p = gp.load_params(ip)
    phi, mu = gp.fill(p, fp)
    with pytest.raises(gp.GpError) as e:
        gp.Simulation(p, phi, mu)
    assert e.value.code == _abi.GP_EINVAL
    assert "Neumann" in str(e.value)


def test_missing_files_report_eio(tmp_path):
    with pytest.raises(gp.GpError) as e:
        gp.load_params(str(tmp_path / "nope.in"))
    assert e.value.code == _abi.GP_EIO
