"""B200-native implementation of the hybrid_1d per-step hot path (kyungguk1/hybrid_code-hfemic_wave).

The product is the CUDA library ``libh1d_gpu.so`` built from ``csrc/`` for sm_100a and its
C-ABI (include/h1d_gpu.h).  This Python package is a thin host-side layer over that ABI:
run descriptions (:mod:`.configs`), the ctypes mirror of the ABI (:mod:`.abi`), a seeded
bi-Maxwellian particle loader (:mod:`.loader`), and the ensemble / serving drivers.

There is no CPU fallback: :func:`open_run` raises if the CUDA library is missing.
"""
from __future__ import annotations

import os

from . import abi, configs  # noqa: F401
from .abi import H1DError, MovedTooFar, Run  # noqa: F401

PKG_DIR = os.path.dirname(os.path.abspath(__file__))
LIB_NAME = "libh1d_gpu.so"


def library_path() -> str:
    return os.path.join(PKG_DIR, LIB_NAME)


def open_run(cfg: "configs.RunConfig") -> Run:
    """Create a run on the current CUDA device through the CUDA library."""
    path = library_path()
    if not os.path.exists(path):
        raise RuntimeError(f"{LIB_NAME} is not built; run __graft_entry__.build() (no CPU fallback exists)")
    return Run(cfg, path, "h1d_")
