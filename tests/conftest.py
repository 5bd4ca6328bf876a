import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
for p in (ROOT, os.path.join(ROOT, "oracle"), os.path.join(ROOT, "tests", "golden")):
    if p not in sys.path:
        sys.path.insert(0, p)

GOLDEN = os.path.join(ROOT, "tests", "golden")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200)")


def load_fixture(name):
    return dict(np.load(os.path.join(GOLDEN, name + ".npz")))


@pytest.fixture(scope="session")
def config1():
    return load_fixture("config1")


@pytest.fixture(scope="session")
def config2():
    return load_fixture("config2")


@pytest.fixture(scope="session")
def config3():
    return load_fixture("config3")


@pytest.fixture(scope="session")
def config4():
    return load_fixture("config4")


@pytest.fixture(scope="session")
def config4_psf():
    return load_fixture("config4_psf")


@pytest.fixture(scope="session")
def config5():
    return load_fixture("config5")


@pytest.fixture(scope="session")
def eos3():
    return load_fixture("eos_c3")


@pytest.fixture(scope="session")
def eos1():
    return load_fixture("eos_c1")


@pytest.fixture(scope="session")
def oracle_lib():
    from snapi_b200 import build as b
    b.build_oracle() if not os.path.exists(os.path.join(ROOT, "oracle", "_ref", "libsnapi_oracle.so")) else None
    import snapi_oracle
    return snapi_oracle


@pytest.fixture(scope="session")
def emu():
    from snapi_b200 import build as b
    import ctypes
    path = b.build_emulator()
    E = ctypes.CDLL(path)
    vp, ip, dbl = ctypes.c_void_p, ctypes.c_int, ctypes.c_double
    E.emu_synth.argtypes = [ip, ip, ip, vp, vp, dbl, vp, ip, vp, vp]
    E.emu_adjoint.argtypes = [ip, ip, ip, vp, vp, dbl, vp, dbl, ip, vp, vp, vp, vp, ip, vp, vp, vp, vp, vp]
    E.emu_voigt.argtypes = [ctypes.c_float, ctypes.c_float, vp]
    E.emu_jvp.argtypes = [ip, ip, ip, vp, vp, dbl, vp, ip, vp, ip, vp, vp]
    return E


def gpu_available():
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False
