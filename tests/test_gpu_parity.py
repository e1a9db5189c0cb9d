"""Parity of the CUDA path (through the C-ABI) with the oracle on identical particles.

The oracle reproduces the reference bit for bit (test_oracle_vs_reference.py).  The GPU path
differs from it only in floating-point association: deposits are summed in another order
(cell-sorted particles, warp reductions, atomics) and the particle push uses FMA and CUDA's
libm.  Tolerances (max-norm relative error against the oracle):
  - one step from an identical state: 1e-12 for fields, sources, moments and particles, and
    the full-grid cell index of every particle identical (a mismatch is allowed only for a
    particle within 1e-12 of a cell boundary, and none is expected);
  - ten steps: 1e-9 (the difference grows with the plasma's own error amplification).
"""
import os

import numpy as np
import pytest
from parity_util import by_pid, cell_keys, cell_mismatches, rel_err, state_errors, with_reference_norms
from state_io import read_state

import hfemic_b200 as h

pytestmark = pytest.mark.gpu
GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
CAMCL = [n for n in sorted(h.configs.PARITY) if h.configs.PARITY[n]().algorithm == h.configs.ALGO_CAMCL]
ALL = sorted(h.configs.PARITY)
TOL1, TOL10 = 1e-12, 1e-9


def run_both(cfg, init, steps, gpu_lib, oracle_lib, chunks=1):
    with h.Run(cfg, gpu_lib, "h1d_") as g, h.Run(cfg, oracle_lib, "orc_") as c:
        g.upload_state(init)
        c.upload_state(init)
        for _ in range(chunks):
            g.advance(steps)
            c.advance(steps)
        return g.state(), c.state(), g.energy(), c.energy()


@pytest.mark.parametrize("name", ALL)
def test_one_step(name, gpu_lib, oracle_lib):
    cfg = h.configs.PARITY[name]()
    init = read_state(os.path.join(GOLDEN, f"{name}.init.bin"))
    g, c, eg, ec = run_both(cfg, init, 1, gpu_lib, oracle_lib)
    errs = state_errors(g, c, cfg)
    print(name, "1 step:", {k: f"{v:.2e}" for k, v in errs.items()})
    bad = {k: v for k, v in errs.items() if not v <= TOL1}
    assert not bad, bad
    mism = cell_mismatches(g, c, cfg)
    assert all(d < 1e-12 for _, _, d in mism), mism
    for key in ("dB2O2", "dE2O2", "KE_lab", "KE_pla"):
        assert rel_err(eg[key], ec[key]) <= TOL1, key


@pytest.mark.parametrize("name", ["p1_cic_periodic", "p2_tsc_mirror_reflecting"])
def test_particles_at_the_right_end(name, gpu_lib, oracle_lib):
    """q1 one ulp below q1max is inside the grid although q1 - q1min rounds up to Nx there, and q1
    = q1max itself is where the boundary pass's wrap or reflection can round to (the reference
    deposits such a particle into the ghost cell and wraps it on its next pass): the sort (every
    step here) puts both in the last cell, and the step matches the oracle at the one-step bar."""
    cfg = h.configs.PARITY[name]().replace(sort_interval=1)
    init = read_state(os.path.join(GOLDEN, f"{name}.init.bin"))
    init["particles"][0]["q1"][:3] = [np.nextafter(cfg.q1max, -np.inf), cfg.q1max - 1e-13, cfg.q1max]
    assert init["particles"][0]["q1"][0] - cfg.q1min == cfg.Nx  # the subtraction rounds up
    g, c, eg, ec = run_both(cfg, init, 1, gpu_lib, oracle_lib)
    errs = state_errors(g, c, cfg)
    bad = {k: v for k, v in errs.items() if not v <= TOL1}
    assert not bad, bad


@pytest.mark.parametrize("name", ALL)
def test_ten_steps(name, gpu_lib, oracle_lib):
    cfg = h.configs.PARITY[name]()
    init = read_state(os.path.join(GOLDEN, f"{name}.init.bin"))
    g, c, eg, ec = run_both(cfg, init, 5, gpu_lib, oracle_lib, chunks=2)
    errs = state_errors(g, c, cfg)
    print(name, "10 steps:", {k: f"{v:.2e}" for k, v in errs.items()})
    bad = {k: v for k, v in errs.items() if not v <= TOL10}
    assert not bad, bad
    assert not [m for m in cell_mismatches(g, c, cfg) if m[2] >= 1e-9]


@pytest.mark.parametrize("name", ALL)
def test_against_reference_fixture(name, gpu_lib):
    """The GPU path against the reference's own output after ten steps (golden fixture)."""
    init = read_state(os.path.join(GOLDEN, f"{name}.init.bin"))
    cfg = with_reference_norms(h.configs.PARITY[name](), init)
    ref = read_state(os.path.join(GOLDEN, f"{name}.step10.bin"))
    with h.Run(cfg, gpu_lib, "h1d_") as g:
        g.upload_state(init)
        g.advance(10)
        st = g.state()
    for key in ("B", "E", "charge", "current"):
        assert rel_err(st[key], ref[key]) <= TOL10, key
    id0 = init["particles"][0]["id"]
    ids = ref["particles"][0]["id"]
    pg = by_pid(st["particles"][0])
    order = np.argsort(ids)
    assert rel_err(pg["q1"], ref["particles"][0]["q1"][order]) <= TOL10
    assert np.array_equal(np.sort(id0[st["particles"][0]["pid"]]), np.sort(ids))


def test_sort_order_is_stable_cell_sort(gpu_lib):
    """With a sort before every step, the device order after one step is exactly the CPU
    stable sort, by full-grid cell, of the uploaded particles."""
    cfg = h.configs.parity_p2().replace(sort_interval=1)
    init = read_state(os.path.join(GOLDEN, f"{cfg.name}.init.bin"))
    with h.Run(cfg, gpu_lib, "h1d_") as g:
        g.upload_state(init)
        g.advance(1)
        for s in range(len(cfg.kinetic)):
            pid = g.particles(s)["pid"]
            keys = cell_keys(init["particles"][s]["q1"], cfg.Nx)
            np.testing.assert_array_equal(pid, np.argsort(keys, kind="stable"))


def test_large_random_state(gpu_lib, oracle_lib):
    """A synthetic state with more particles than the fixtures (seeded loader)."""
    from hfemic_b200.loader import initial_state

    cfg = h.configs.parity_p2().replace(Nx=256, xi=0.01, phase_retardation=(32, 1.0), amplitude_damping=(32, 0.2))
    for k in cfg.kinetic:
        k.Nc = 200
    init = initial_state(cfg, seed=3)
    g, c, _, _ = run_both(cfg, init, 2, gpu_lib, oracle_lib)
    errs = state_errors(g, c, cfg)
    print("large 2 steps:", {k: f"{v:.2e}" for k, v in errs.items()})
    assert max(errs.values()) <= 1e-11


def test_absorbing_boundary(gpu_lib, oracle_lib):
    """Absorbing walls (an extension: the reference has periodic and reflecting particles only):
    the GPU path removes exactly the particles the oracle removes, and the rest agree."""
    from hfemic_b200.loader import initial_state

    cfg = h.configs.parity_p2().replace(particle_bc=h.configs.BC_ABSORBING, Nx=128, xi=0.02)
    for k in cfg.kinetic:
        k.Nc = 64
    init = initial_state(cfg, seed=9)
    g, c, eg, ec = run_both(cfg, init, 10, gpu_lib, oracle_lib)
    for s in range(len(cfg.kinetic)):
        pg, pc = by_pid(g["particles"][s]), by_pid(c["particles"][s])
        assert pg["q1"].size < init["particles"][s]["q1"].size  # the case does absorb particles
        np.testing.assert_array_equal(pg["pid"], pc["pid"])
    errs = state_errors(g, c, cfg)
    bad = {k: v for k, v in errs.items() if not v <= TOL10}
    assert not bad, bad


@pytest.mark.parametrize("precision,tol", [(h.configs.PREC_FP64, 1e-11), (h.configs.PREC_MIXED, 1e-4)])
def test_empty_and_ragged_species(gpu_lib, oracle_lib, precision, tol):
    """Particle counts at the edges of the pass's tiling (a 256-particle chunk of 4 warps x 32
    lanes x 2 particles, the mixed pass's lane pairs, the 4-wide vector tiles of collect_all):
    no particles, one, a pair, a warp minus and plus one, a chunk minus and plus one; five steps
    against the oracle."""
    import copy

    cfg = h.configs.parity_p2().replace(precision=precision)
    init = read_state(os.path.join(GOLDEN, f"{cfg.name}.init.bin"))
    for k in (0, 1, 2, 31, 33, 255, 257, 1023):
        st = copy.deepcopy(init)
        st["particles"][0] = {key: v[:k] for key, v in st["particles"][0].items()}
        with h.Run(cfg, gpu_lib, "h1d_") as g, h.Run(cfg.replace(precision=h.configs.PREC_FP64), oracle_lib, "orc_") as c:
            g.upload_state(st)
            c.upload_state(st)
            g.advance(5)
            c.advance(5)
            sg, sc = g.state(), c.state()
        assert sg["particles"][0]["q1"].size == k
        errs = state_errors(sg, sc, cfg)
        if k == 0:
            assert not np.any(sg["moments"][0]["n"])
        bad = {key: v for key, v in errs.items() if not v <= tol}
        assert not bad, (k, bad)


@pytest.mark.parametrize("precision,tol", [(h.configs.PREC_FP64, 1e-11), (h.configs.PREC_MIXED, 1e-4)])
def test_largest_grid(gpu_lib, oracle_lib, precision, tol):
    """A grid near the C ABI's largest (Nx = 65534 cells: 16-bit sort keys in two 8-bit passes,
    hundreds of field-kernel blocks, a mirror field near its validity limit), two TSC species of
    2 particles per cell, three steps against the oracle."""
    from hfemic_b200.loader import initial_state

    cfg = h.configs.parity_p2().replace(Nx=65534, xi=4e-5, phase_retardation=(512, 1.0),
                                       amplitude_damping=(512, 0.2), precision=precision)
    for k in cfg.kinetic:
        k.Nc = 2
    init = initial_state(cfg, seed=21)
    with h.Run(cfg, gpu_lib, "h1d_") as g, h.Run(cfg.replace(precision=h.configs.PREC_FP64), oracle_lib, "orc_") as c:
        g.upload_state(init)
        c.upload_state(init)
        g.advance(3)
        c.advance(3)
        errs = state_errors(g.state(), c.state(), cfg)
    bad = {k: v for k, v in errs.items() if not v <= tol}
    assert not bad, bad


@pytest.mark.parametrize("name", ["p2_tsc_mirror_reflecting", "p4_pc_tsc_mirror_reflecting"])
def test_gyrophase_randomization(gpu_lib, oracle_lib, name):
    """Reflected particles with their gyrophase randomised (Delegate::randomize_gyrophase,
    Boundary/Delegate.cc:146-156; the angle from a counter-based hash of seed, step, species and
    particle id instead of std::random_device): ten steps against the oracle's same draws."""
    cfg = h.configs.PARITY[name]().replace(randomize_gyrophase=True, gyrophase_seed=12345)
    init = read_state(os.path.join(GOLDEN, f"{name}.init.bin"))
    g, c, _, _ = run_both(cfg, init, 5, gpu_lib, oracle_lib, chunks=2)
    errs = state_errors(g, c, cfg)
    bad = {k: v for k, v in errs.items() if not v <= TOL10}
    assert not bad, bad
    # the randomisation acted: the same run without it differs
    g0, _, _, _ = run_both(cfg.replace(randomize_gyrophase=False), init, 5, gpu_lib, oracle_lib, chunks=2)
    assert rel_err(by_pid(g["particles"][0])["vy"], by_pid(g0["particles"][0])["vy"]) > 1e-3


@pytest.mark.parametrize("precision,tol", [(h.configs.PREC_FP64, TOL10), (h.configs.PREC_MIXED, 1e-4)])
def test_pc_species_sharing_a_launch(gpu_lib, oracle_lib, precision, tol):
    """Two TSC species under the predictor-corrector cycle: both particle passes of a step cover
    them in one launch (two parameter groups); ten steps against the oracle."""
    name = "p2_tsc_mirror_reflecting"
    cfg = h.configs.PARITY[name]().replace(algorithm=h.configs.ALGO_PC, precision=precision)
    init = read_state(os.path.join(GOLDEN, f"{name}.init.bin"))
    with h.Run(cfg, gpu_lib, "h1d_") as g, h.Run(cfg.replace(precision=h.configs.PREC_FP64), oracle_lib, "orc_") as c:
        g.upload_state(init)
        c.upload_state(init)
        g.advance(10)
        c.advance(10)
        errs = state_errors(g.state(), c.state(), cfg)
    bad = {k: v for k, v in errs.items() if not v <= tol}
    assert not bad, bad


def test_test_particles(gpu_lib, oracle_lib):
    """Test particles (TestParticleVDF, VDF/TestParticleVDF.cc:15-24: weight 0, f0 = 0) run as a
    full-f species without refresh: they are pushed and moved like the oracle's, and deposit
    nothing."""
    cfg = h.configs.parity_p2()
    init = read_state(os.path.join(GOLDEN, f"{cfg.name}.init.bin"))
    init["particles"][1]["w"] = np.zeros_like(init["particles"][1]["w"])
    g, c, _, _ = run_both(cfg, init, 5, gpu_lib, oracle_lib, chunks=2)
    errs = state_errors(g, c, cfg)
    bad = {k: v for k, v in errs.items() if not v <= TOL10}
    assert not bad, bad
    for key in ("n", "nV", "nvv"):
        assert not np.any(g["moments"][1][key]), key
    moved = by_pid(g["particles"][1])["q1"] - init["particles"][1]["q1"]
    assert np.count_nonzero(moved) > 0.9 * moved.size


def test_moved_too_far(gpu_lib):
    cfg = h.configs.parity_p1()
    init = read_state(os.path.join(GOLDEN, f"{cfg.name}.init.bin"))
    init["particles"][0]["vx"][5] = 2.0 * cfg.Dx / cfg.dt
    with h.Run(cfg, gpu_lib, "h1d_") as g:
        g.upload_state(init)
        with pytest.raises(h.MovedTooFar):
            g.advance(1)


def test_invalid_params(gpu_lib):
    cfg = h.configs.parity_p1()
    p = h.abi.make_params(cfg)
    p.kinetic[0].shape_order = 4
    lib, fn = h.abi.load_library(gpu_lib, "h1d_")
    import ctypes

    handle = ctypes.c_void_p()
    assert fn["create"](ctypes.byref(p), ctypes.byref(handle)) == h.abi.ERR_INVALID_ARG
    assert not handle.value
    # equilibrium distributions of evolving weights: unknown kind, out-of-range parameters
    C = h.configs
    for kind, param in ((7, (0, 0, 0)), (C.VDF_LOSSCONE, (-0.1, 0, 0)), (C.VDF_PARTIAL_SHELL, (1.5, 0, 0)),
                        (C.VDF_PARTIAL_SHELL, (2, -1, 0)), (C.VDF_COUNTER_BEAM, (0, 0, 0))):
        p = h.abi.make_params(C.parity_p7())
        p.kinetic[0].vdf = kind
        for j in range(3):
            p.kinetic[0].vdf_param[j] = param[j]
        assert fn["create"](ctypes.byref(p), ctypes.byref(handle)) == h.abi.ERR_INVALID_ARG, (kind, param)
        assert not handle.value


def test_device_rounding_and_trig(gpu_lib):
    """The kernels' exact floor / round / ceil (no conversion unit) equal the C library's on
    random, half-integer, integer and near-integer arguments; their Taylor sin/cos on
    [-pi/2, pi/2] are within 4e-16 (absolute) of the C library's."""
    import ctypes

    rng = np.random.default_rng(7)
    x = np.concatenate([
        rng.uniform(-5000, 5000, 200000),
        np.arange(-4000, 4000) + 0.5,
        np.arange(-4000, 4000, dtype=float),
        np.nextafter(np.arange(-100, 100, dtype=float), np.inf),
        np.nextafter(np.arange(-100, 100, dtype=float), -np.inf),
        np.nextafter(np.arange(-100, 100, dtype=float) + 0.5, np.inf),
        np.nextafter(np.arange(-100, 100, dtype=float) + 0.5, -np.inf),
        [0.0, -0.0, 0.49999999999999994, -0.49999999999999994],
    ])
    lib = ctypes.CDLL(gpu_lib)
    dp = ctypes.POINTER(ctypes.c_double)
    lib.h1d_math_check.argtypes = [dp, ctypes.c_int64, dp]
    out = np.empty((x.size, 5))
    assert lib.h1d_math_check(x.ctypes.data_as(dp), x.size, out.ctypes.data_as(dp)) == 0
    np.testing.assert_array_equal(out[:, 0], np.floor(x))
    away = np.where(np.abs(x - np.trunc(x)) == 0.5, np.trunc(x) + np.sign(x), np.round(x))  # std::round
    np.testing.assert_array_equal(out[:, 1], away)
    np.testing.assert_array_equal(out[:, 2], np.ceil(x))
    t = np.concatenate([rng.uniform(-np.pi / 2, np.pi / 2, 100000), [0.0, np.pi / 2, -np.pi / 2, 1e-300]])
    out = np.empty((t.size, 5))
    assert lib.h1d_math_check(t.ctypes.data_as(dp), t.size, out.ctypes.data_as(dp)) == 0
    assert np.max(np.abs(out[:, 3] - np.sin(t))) <= 4e-16
    assert np.max(np.abs(out[:, 4] - np.cos(t))) <= 4e-16


@pytest.mark.parametrize("precision, tol", [(h.configs.PREC_FP64, 1e-12), (h.configs.PREC_MIXED, 1e-5)])
def test_collect_all_formed_by_the_last_pass(gpu_lib, precision, tol):
    """For CIC species with fixed weights the particle pass of an advance_by's last step also
    deposits collect_all's second moments, and n, nV come from that step's end-position deposit.
    The moments equal the ones of the separate collect_all pass (sort, then moments kernel), which
    a run takes when its particle generation changed since that step (here: an upload of the
    same fields).  config 1's plasma at Nx 256; mixed precision sums FP32 lane partials in both."""
    from hfemic_b200.loader import initial_state

    cfg = h.configs.config1().replace(precision=precision)
    st = initial_state(cfg, seed=4)
    out = []
    for fused in (True, False):
        with h.Run(cfg, gpu_lib, "h1d_") as g:
            g.upload_state(st)
            g.advance(7)
            if not fused:
                B, E = g.fields()
                g.upload_fields(B, E)
            out.append([g.moments(s) for s in range(len(cfg.kinetic))] + [g.energy()])
    for (n, nV, nvv), (m, mV, mvv) in zip(out[0][:-1], out[1][:-1]):
        assert rel_err(n, m) <= tol and rel_err(nV, mV) <= tol and rel_err(nvv, mvv) <= tol
    for key in ("KE_lab", "KE_pla"):
        assert rel_err(out[0][-1][key], out[1][-1][key]) <= tol, key
