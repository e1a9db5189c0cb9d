import importlib.util
import os
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PKG_DIR = os.path.join(ROOT, "hybrid_code-hfemic_wave_b200")
GOLDEN = os.path.join(ROOT, "tests", "golden")
ORACLE_LIB = os.path.join(ROOT, "oracle", "liboracle.so")


def _load_package():
    """The package directory name is not an identifier; import it as ``hfemic_b200``."""
    if "hfemic_b200" in sys.modules:
        return sys.modules["hfemic_b200"]
    spec = importlib.util.spec_from_file_location("hfemic_b200", os.path.join(PKG_DIR, "__init__.py"),
                                                  submodule_search_locations=[PKG_DIR])
    mod = importlib.util.module_from_spec(spec)
    sys.modules["hfemic_b200"] = mod
    spec.loader.exec_module(mod)
    return mod


_load_package()
sys.path.insert(0, GOLDEN)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200) and the built libh1d_gpu.so")


@pytest.fixture(scope="session")
def oracle_lib():
    """Path of the C oracle (the checker); built on first use."""
    src = os.path.join(ROOT, "oracle", "h1d_oracle.c")
    if not os.path.exists(ORACLE_LIB) or os.path.getmtime(ORACLE_LIB) < os.path.getmtime(src):
        subprocess.check_call(["make", "-C", os.path.join(ROOT, "oracle"), "all"],
                              stdout=subprocess.DEVNULL)
    return ORACLE_LIB


@pytest.fixture(scope="session")
def oracle_cdll(oracle_lib):
    import ctypes
    return ctypes.CDLL(oracle_lib)


@pytest.fixture(scope="session")
def gpu_lib():
    """Path of the CUDA library; a GPU test fails loudly when it or the device is missing."""
    import torch
    pkg = _load_package()
    path = pkg.library_path()
    if not os.path.exists(path):
        pytest.fail("libh1d_gpu.so is not built")
    if not torch.cuda.is_available():
        pytest.fail("no CUDA device")
    return path
