import os
import subprocess
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)
HERE = os.path.dirname(os.path.abspath(__file__))
if HERE not in sys.path:
    sys.path.insert(0, HERE)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200); run with -m gpu")
    config.addinivalue_line("markers", "slow: long CPU runs of the oracle")
    # build the product library and the CPU oracle if this tree has not been built yet
    lib = os.path.join(ROOT, "eshwar_dipan_b200", "libgp.so")
    if not os.path.exists(lib):
        from eshwar_dipan_b200.build import build
        build()
    if not os.path.exists(os.path.join(ROOT, "oracle", "liboracle.so")):
        subprocess.run(["make", "-C", os.path.join(ROOT, "oracle"), "oracle"], check=True, capture_output=True)


def pytest_collection_modifyitems(config, items):
    # keep the default order except that files named test_zz_* run last
    items.sort(key=lambda it: (os.path.basename(str(it.fspath)).startswith("test_zz_"),))
