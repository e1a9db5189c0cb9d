"""CPU checks of the C-ABI library: it loads without a GPU and exports every entry point that
include/h1d_gpu.h declares; the ctypes mirror matches the C struct size."""
import ctypes
import os
import re

import pytest

import hfemic_b200 as h

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_functions():
    names = []
    for fn in os.listdir(os.path.join(ROOT, "include")):
        if fn.endswith(".h"):
            text = open(os.path.join(ROOT, "include", fn)).read()
            names += re.findall(r"^\s*(?:[\w\s\*]+?)\b(h1d_\w+)\s*\(", text, flags=re.M)
    return sorted(set(names))


@pytest.fixture(scope="module")
def lib():
    path = h.library_path()
    if not os.path.exists(path):
        from hfemic_b200 import build

        build.build()
    return ctypes.CDLL(path)


def test_exports_every_declared_symbol(lib):
    names = declared_functions()
    assert "h1d_advance" in names and len(names) > 15
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing


def test_params_layout(lib):
    lib.h1d_params_size.restype = ctypes.c_size_t
    assert lib.h1d_params_size() == ctypes.sizeof(h.abi.Params)
    assert lib.h1d_abi_version() == h.abi.ABI_VERSION


def test_create_without_device_fails_cleanly(lib):
    """No compute call without a GPU: create reports the missing device, it does not crash."""
    import torch

    if torch.cuda.is_available():
        pytest.skip("a device is present")
    p = h.abi.make_params(h.configs.parity_p1())
    handle = ctypes.c_void_p()
    st = lib.h1d_create(ctypes.byref(p), ctypes.byref(handle))
    assert st == h.abi.ERR_NO_DEVICE and not handle.value
