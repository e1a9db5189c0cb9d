"""The allocation-free moment entry point against the run-based one.

h1d_collect_moments_noalloc is for callers that cannot allocate device memory themselves: their
application's pool allocator already owns the device memory, or their loop cannot afford an
allocation that may synchronise the device.  It takes particles in device buffers the caller
owns and writes the moments into device buffers the caller owns, using a fixed scratch array
compiled into the library.  Here the test owns those buffers (torch tensors) and checks, on two
calls in a row, that the entry point returns what h1d_download_moments returns for the same
particles, within the 1e-12 (max-norm relative) tolerance of the other FP64 parity tests: the
two differ only in the order in which the deposits are summed.
"""
import ctypes

import numpy as np
import pytest

import hfemic_b200 as h

pytestmark = pytest.mark.gpu

MAX_NX = 4096  # H1D_NOALLOC_MAX_NX in include/h1d_gpu.h


def _entry(gpu_lib):
    lib = ctypes.CDLL(gpu_lib)
    f = lib.h1d_collect_moments_noalloc
    vp = ctypes.c_void_p
    f.argtypes = [ctypes.c_int64, ctypes.c_double, ctypes.c_int, vp, vp, vp, vp, vp, ctypes.c_int64, vp, vp, vp, vp]
    f.restype = ctypes.c_int
    return f


def _rel(a, b):
    scale = np.max(np.abs(b))
    return float(np.max(np.abs(a - b)) / scale) if scale else float(np.max(np.abs(a - b)))


def test_noalloc_moments_match_run_moments(gpu_lib):
    import torch

    from hfemic_b200.loader import initial_state

    f = _entry(gpu_lib)
    cfg = h.configs.parity_p2().replace(Nx=256, xi=0.01, phase_retardation=(32, 1.0), amplitude_damping=(32, 0.2))
    for k in cfg.kinetic:
        k.Nc = 100
    state = initial_state(cfg, seed=11)
    M = cfg.Nx + 6
    with h.Run(cfg, gpu_lib, "h1d_") as run:
        run.upload_state(state)
        run.advance(2)
        for s, kin in enumerate(cfg.kinetic):
            n_ref, nV_ref, nvv_ref = run.moments(s)
            p = run.particles(s)
            dev = {key: torch.tensor(p[key], dtype=torch.float64, device="cuda") for key in ("q1", "vx", "vy", "vz", "w")}
            stream = torch.cuda.current_stream().cuda_stream
            for _ in range(2):
                outs = [torch.full((M * c,), float("nan"), dtype=torch.float64, device="cuda") for c in (1, 3, 6)]
                st = f(cfg.Nx, cfg.moment_norm(kin), cfg.particle_bc,
                       *[dev[key].data_ptr() for key in ("q1", "vx", "vy", "vz", "w")], p["q1"].size,
                       *[o.data_ptr() for o in outs], stream)
                assert st == h.abi.OK
                n, nV, nvv = (o.cpu().numpy() for o in outs)
                assert _rel(n, n_ref) <= 1e-12
                assert _rel(nV.reshape(M, 3), nV_ref) <= 1e-12
                assert _rel(nvv.reshape(M, 6), nvv_ref) <= 1e-12


def test_noalloc_rejects_grids_beyond_its_scratch(gpu_lib):
    f = _entry(gpu_lib)
    st = f(MAX_NX + 1, 1.0, 0, None, None, None, None, None, 0, 1, 1, 1, None)
    assert st == h.abi.ERR_INVALID_ARG
