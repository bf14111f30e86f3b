import ctypes
import os
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200); runs the sm_100a library")
    config.addinivalue_line("markers", "slow: longer oracle runs")


def has_gpu():
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


@pytest.fixture(scope="session")
def gpu():
    if not has_gpu():
        pytest.skip("no CUDA device")
    from m2c_b200 import gpu as g
    g.lib()  # fails loudly if the library is missing
    return g


@pytest.fixture(scope="session")
def ref():
    from oracle import ref as r
    if not r.available("ref"):
        pytest.skip("reference oracle not built (make -C oracle ref)")
    return r


@pytest.fixture(scope="session")
def host_riemann_lib(tmp_path_factory):
    """The library's exact Riemann solver compiled for the host
    (tests/host/riemann_host.cpp)."""
    out = str(tmp_path_factory.mktemp("riemann_host") / "libriemann_host.so")
    src = os.path.join(ROOT, "tests", "host", "riemann_host.cpp")
    subprocess.run(["g++", "-O2", "-ffp-contract=off", "-fPIC", "-shared", "-o", out, src], check=True)
    return ctypes.CDLL(out)
