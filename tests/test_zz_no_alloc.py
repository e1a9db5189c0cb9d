"""The allocation-free moment entry point against the run-based one.

h1d_collect_moments_noalloc is for callers that cannot allocate device memory themselves: their
application's pool allocator already owns the device memory, or their loop cannot afford an
allocation that may synchronise the device.  It takes particles in device buffers the caller
owns and writes the moments into device buffers the caller owns, using a fixed scratch array
compiled into the library.  Here the test owns those buffers (torch tensors) and checks, on two
calls in a row, that the entry point returns what h1d_download_moments returns for the same
particles, within the 1e-12 (max-norm relative) tolerance of the other FP64 parity tests: the
two differ only in the order in which the deposits are summed.  Covered: a small grid and the
largest one the fixed scratch holds, periodic and reflecting ghost folds, particles in the
caller's own order (shuffled), a ragged count in buffers that are not 16-byte aligned (the
kernel's scalar-load path), delta-f species (the caller adds the equilibrium moments), and
particles outside the grid (H1D_ERR_NAN, after which a clean call succeeds).
"""
import ctypes

import numpy as np
import pytest

import hfemic_b200 as h

pytestmark = pytest.mark.gpu

MAX_NX = 4096  # H1D_NOALLOC_MAX_NX in include/h1d_gpu.h
TOL = 1e-12
KEYS = ("q1", "vx", "vy", "vz", "w")


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


def _device_particles(p, order=None, offset=0, extra=None):
    """The particles as caller-owned device arrays: in `order` (a permutation) if given, with
    `extra` particles appended, each array starting `offset` doubles into its allocation."""
    import torch

    out = {}
    for key in KEYS:
        a = np.asarray(p[key])
        if order is not None:
            a = a[order]
        if extra is not None:
            a = np.concatenate([a, extra[key]])
        t = torch.empty(a.size + offset, dtype=torch.float64, device="cuda")
        t[offset:] = torch.from_numpy(np.ascontiguousarray(a)).cuda()
        out[key] = t[offset:]
    return out


def _collect(f, Nx, norm, bc, dev, n):
    """Two calls in a row into fresh NaN-filled outputs; returns the status and the second call's
    moments, and checks the first call's equal the second's to the tolerance."""
    import torch

    M = Nx + 6
    stream = torch.cuda.current_stream().cuda_stream
    res = []
    for _ in range(2):
        outs = [torch.full((M * c,), float("nan"), dtype=torch.float64, device="cuda") for c in (1, 3, 6)]
        st = f(Nx, norm, bc, *[dev[key].data_ptr() for key in KEYS], n, *[o.data_ptr() for o in outs], stream)
        if st != h.abi.OK:
            return st, None
        n_, nV, nvv = (o.cpu().numpy() for o in outs)
        res.append((n_, nV.reshape(M, 3), nvv.reshape(M, 6)))
    for a, b in zip(res[0], res[1]):
        assert _rel(a, b) <= TOL
    return h.abi.OK, res[1]


def _run_state(Nx, bc, seed=11):
    from hfemic_b200.loader import initial_state

    cfg = h.configs.parity_p2().replace(Nx=Nx, xi=0.001, particle_bc=bc, phase_retardation=(32, 1.0),
                                        amplitude_damping=(32, 0.2))
    for k in cfg.kinetic:
        k.Nc = 100 if Nx <= 256 else 12
    return cfg, initial_state(cfg, seed=seed)


@pytest.mark.parametrize("Nx", [256, MAX_NX])
@pytest.mark.parametrize("bc", ["periodic", "reflecting"])
def test_noalloc_moments_match_run_moments(gpu_lib, Nx, bc):
    f = _entry(gpu_lib)
    code = h.configs.BC_PERIODIC if bc == "periodic" else h.configs.BC_REFLECTING
    cfg, state = _run_state(Nx, code)
    with h.Run(cfg, gpu_lib, "h1d_") as run:
        run.upload_state(state)
        run.advance(2)
        for s, kin in enumerate(cfg.kinetic):
            ref = run.moments(s)
            p = run.particles(s)
            n = p["q1"].size
            st, got = _collect(f, cfg.Nx, cfg.moment_norm(kin), code, _device_particles(p), n)
            assert st == h.abi.OK
            for a, b in zip(got, ref):
                assert _rel(a, b) <= TOL
            # the caller's own (unsorted) order
            perm = np.random.default_rng(s).permutation(n)
            st, got = _collect(f, cfg.Nx, cfg.moment_norm(kin), code, _device_particles(p, order=perm), n)
            assert st == h.abi.OK
            for a, b in zip(got, ref):
                assert _rel(a, b) <= TOL


def test_noalloc_ragged_unaligned_buffers(gpu_lib):
    """A ragged particle count (one zero-weight particle appended) in buffers that start 8 bytes
    past a 16-byte boundary: the kernel's scalar-load path gives the same moments."""
    f = _entry(gpu_lib)
    cfg, state = _run_state(256, h.configs.BC_REFLECTING, seed=5)
    with h.Run(cfg, gpu_lib, "h1d_") as run:
        run.upload_state(state)
        run.advance(1)
        kin = cfg.kinetic[0]
        ref = run.moments(0)
        p = run.particles(0)
        extra = {"q1": np.array([0.25]), "vx": np.array([1.0]), "vy": np.array([-1.0]), "vz": np.array([0.5]),
                 "w": np.array([0.0])}
        dev = _device_particles(p, offset=1, extra=extra)
        assert all(dev[k].data_ptr() % 16 == 8 for k in KEYS)
        n = p["q1"].size + 1
        assert n % 32 != 0
        st, got = _collect(f, cfg.Nx, cfg.moment_norm(kin), cfg.particle_bc, dev, n)
        assert st == h.abi.OK
        for a, b in zip(got, ref):
            assert _rel(a, b) <= TOL


def test_noalloc_delta_f_needs_the_equilibrium_moments(gpu_lib):
    """For a delta-f species the entry point returns the weighted sums; adding the equilibrium
    n0 and nvv0 on the interior gives what h1d_download_moments returns."""
    import os

    from parity_util import with_reference_norms
    from state_io import read_state

    from hfemic_b200.loader import equilibrium

    f = _entry(gpu_lib)
    name = "p7_psd_tsc_mirror_reflecting"
    init = read_state(os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", f"{name}.init.bin"))
    cfg = with_reference_norms(h.configs.PARITY[name](), init)
    kin = cfg.kinetic[0]
    assert kin.scheme == h.configs.DELTA_F
    P, Nx = 3, cfg.Nx
    with h.Run(cfg, gpu_lib, "h1d_") as run:
        run.upload_state(init)
        run.advance(2)
        ref = run.moments(0)
        p = run.particles(0)
        st, (n, nV, nvv) = _collect(f, Nx, cfg.moment_norm(kin), cfg.particle_bc, _device_particles(p), p["q1"].size)
        assert st == h.abi.OK
    n0, vpar2, vperp2 = equilibrium(cfg, kin, np.arange(Nx) + cfg.q1min + 0.5)
    n[P:P + Nx] += n0
    nvv[P:P + Nx, 0] += n0 * vpar2
    nvv[P:P + Nx, 1] += n0 * vperp2
    nvv[P:P + Nx, 2] += n0 * vperp2
    assert _rel(n, ref[0]) <= TOL
    assert _rel(nV, ref[1]) <= TOL
    assert _rel(nvv, ref[2]) <= TOL


def test_noalloc_particle_outside_the_grid(gpu_lib):
    """A non-finite or out-of-grid position gives H1D_ERR_NAN; the status word is cleared on the
    next call, which succeeds."""
    f = _entry(gpu_lib)
    cfg, state = _run_state(256, h.configs.BC_PERIODIC, seed=7)
    p = state["particles"][0]
    kin = cfg.kinetic[0]
    n = p["q1"].size
    for bad in (float("nan"), 10.0 * cfg.Nx):
        q = dict(p)
        q["q1"] = p["q1"].copy()
        q["q1"][n // 2] = bad
        st, _ = _collect(f, cfg.Nx, cfg.moment_norm(kin), cfg.particle_bc, _device_particles(q), n)
        assert st == h.abi.ERR_NAN
        st, got = _collect(f, cfg.Nx, cfg.moment_norm(kin), cfg.particle_bc, _device_particles(p), n)
        assert st == h.abi.OK
        assert np.all(np.isfinite(got[0]))


def test_noalloc_rejects_grids_beyond_its_scratch(gpu_lib):
    f = _entry(gpu_lib)
    st = f(MAX_NX + 1, 1.0, 0, None, None, None, None, None, 0, 1, 1, 1, None)
    assert st == h.abi.ERR_INVALID_ARG
