"""The mixed-precision particle pass (int32 cell + FP32 offset positions, FP32 velocities, weights,
interpolation and push, FP32 warp deposits summed into FP64 cells; FP64 field cycle) against FP64.

Tolerance: 1e-4 max-norm relative error in the moments (n, nV, nvv), the sources, the fields and
the wave and particle energies, against the FP64 oracle on the golden initial states and against
the FP64 GPU path on larger seeded states.  Cell indices and the sort order follow the same rules
as the FP64 path.
"""
import os

import numpy as np
import pytest
from parity_util import by_pid, cell_keys, rel_err
from state_io import read_state

import hfemic_b200 as h

pytestmark = pytest.mark.gpu
GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
ALL = sorted(h.configs.PARITY)
TOL = 1e-4
MIXED = h.configs.PREC_MIXED


def mixed_errors(gm, gd, em, ed, cfg):
    """Relative errors of the mixed run (gm, em) against an FP64 run (gd, ed)."""
    errs = {}
    for key in ("B", "E", "charge", "current"):
        errs[key] = rel_err(gm[key], gd[key])
    for s in range(len(cfg.kinetic)):
        for key in ("n", "nV", "nvv"):
            errs[f"moments[{s}].{key}"] = rel_err(gm["moments"][s][key], gd["moments"][s][key])
    for i in range(len(cfg.cold)):
        for key in ("n", "nV", "nvv"):
            errs[f"cold[{i}].{key}"] = rel_err(gm["cold"][i][key], gd["cold"][i][key])
    for key in ("dB2O2", "dE2O2", "KE_lab", "KE_pla"):
        errs[key] = rel_err(em[key], ed[key])
    return errs


def run_pair(cfg, init, steps, gpu_lib, ref_lib, ref_prefix):
    with h.Run(cfg.replace(precision=MIXED), gpu_lib, "h1d_") as m, h.Run(cfg, ref_lib, ref_prefix) as d:
        m.upload_state(init)
        d.upload_state(init)
        m.advance(steps)
        d.advance(steps)
        return m.state(), d.state(), m.energy(), d.energy()


@pytest.mark.parametrize("steps", [1, 10])
@pytest.mark.parametrize("name", ALL)
def test_mixed_against_fp64_oracle(name, steps, gpu_lib, oracle_lib):
    cfg = h.configs.PARITY[name]()
    init = read_state(os.path.join(GOLDEN, f"{name}.init.bin"))
    gm, gd, em, ed = run_pair(cfg, init, steps, gpu_lib, oracle_lib, "orc_")
    errs = mixed_errors(gm, gd, em, ed, cfg)
    print(name, steps, "steps mixed vs oracle:", {k: f"{v:.1e}" for k, v in errs.items()})
    bad = {k: v for k, v in errs.items() if not v <= TOL}
    assert not bad, bad
    for s in range(len(cfg.kinetic)):
        pm, pd = by_pid(gm["particles"][s]), by_pid(gd["particles"][s])
        assert pm["q1"].size == pd["q1"].size
        for key in ("vx", "vy", "vz"):
            assert rel_err(pm[key], pd[key]) <= TOL, key
        assert np.max(np.abs(pm["q1"] - pd["q1"])) <= 1e-4 * steps


def test_mixed_against_fp64_gpu_large(gpu_lib):
    """A seeded state with 200 particles per cell, 20 steps, mixed against the FP64 GPU path."""
    from hfemic_b200.loader import initial_state

    cfg = h.configs.parity_p2().replace(Nx=256, xi=0.01, phase_retardation=(32, 1.0), amplitude_damping=(32, 0.2))
    for k in cfg.kinetic:
        k.Nc = 200
    init = initial_state(cfg, seed=5)
    gm, gd, em, ed = run_pair(cfg, init, 20, gpu_lib, gpu_lib, "h1d_")
    errs = mixed_errors(gm, gd, em, ed, cfg)
    print("large 20 steps mixed vs FP64:", {k: f"{v:.1e}" for k, v in errs.items()})
    assert max(errs.values()) <= TOL


def test_mixed_absorbing(gpu_lib):
    """Absorbing boundaries remove the same particles as the FP64 path (none sits within the
    FP32 offset resolution of a wall here)."""
    from hfemic_b200.loader import initial_state

    cfg = h.configs.parity_p2().replace(particle_bc=h.configs.BC_ABSORBING, Nx=128, xi=0.02)
    for k in cfg.kinetic:
        k.Nc = 64
    init = initial_state(cfg, seed=9)
    gm, gd, em, ed = run_pair(cfg, init, 10, gpu_lib, gpu_lib, "h1d_")
    for s in range(len(cfg.kinetic)):
        nm, nd = gm["particles"][s]["q1"].size, gd["particles"][s]["q1"].size
        assert nd < init["particles"][s]["q1"].size  # the case does absorb particles
        assert nm == nd
        assert np.array_equal(np.sort(gm["particles"][s]["pid"]), np.sort(gd["particles"][s]["pid"]))
    errs = mixed_errors(gm, gd, em, ed, cfg)
    assert max(errs.values()) <= TOL, errs


def test_mixed_upload_download_round_trip(gpu_lib):
    """Upload converts q1 to (cell, offset) with cell = floor(q1 - q1min) exactly; download gives
    q1 back to the FP32 offset resolution and the velocities to FP32 rounding."""
    cfg = h.configs.parity_p2().replace(precision=MIXED)
    init = read_state(os.path.join(GOLDEN, f"{cfg.name}.init.bin"))
    with h.Run(cfg, gpu_lib, "h1d_") as m:
        m.upload_state(init)
        for s in range(len(cfg.kinetic)):
            p = m.particles(s)
            src = init["particles"][s]
            np.testing.assert_array_equal(p["pid"], np.arange(src["q1"].size))
            np.testing.assert_array_equal(cell_keys(p["q1"], cfg.Nx), cell_keys(src["q1"], cfg.Nx))
            assert np.max(np.abs(p["q1"] - src["q1"])) <= 2.0 ** -24
            for key in ("vx", "vy", "vz", "w"):
                assert rel_err(p[key], src[key]) <= 2.0 ** -24, key


@pytest.mark.parametrize("name", ["p1_cic_periodic", "p2_tsc_mirror_reflecting"])
def test_mixed_right_edge_stays_inside(gpu_lib, name):
    """A position within half a fixed-point step of q1max, or q1max itself (where the boundary
    pass's wrap can round to), rounds to Nx 2^F, one past the grid; upload (like the device loader,
    through the same conversion) keeps it on the last position Nx 2^F - 1, in cell Nx - 1, and the
    run sorts and steps it as an ordinary particle."""
    cfg = h.configs.PARITY[name]().replace(precision=MIXED, sort_interval=1)
    init = read_state(os.path.join(GOLDEN, f"{name}.init.bin"))
    step = 2.0 ** -h.configs.position_fraction_bits(cfg.Nx)
    edge = [np.nextafter(cfg.q1max, -np.inf), cfg.q1max - 0.25 * step, cfg.q1max - 0.49 * step, cfg.q1max]
    q1 = init["particles"][0]["q1"]
    q1[:4] = edge
    with h.Run(cfg, gpu_lib, "h1d_") as m:
        m.upload_state(init)
        p = m.particles(0)  # upload order until the first sort
        np.testing.assert_array_equal(p["pid"][:4], [0, 1, 2, 3])
        got = p["q1"][:4]
        assert np.all(got < cfg.q1max) and np.all(got >= cfg.q1max - step)
        assert np.all(np.floor(got - cfg.q1min) == cfg.Nx - 1)
        m.advance(2)  # sorts (interval 1) and pushes them: no particle is reported outside the grid
        assert m.particle_count(0) == q1.size


def test_mixed_sort_order_is_stable_cell_sort(gpu_lib):
    cfg = h.configs.parity_p2().replace(sort_interval=1, precision=MIXED)
    init = read_state(os.path.join(GOLDEN, f"{cfg.name}.init.bin"))
    with h.Run(cfg, gpu_lib, "h1d_") as g:
        g.upload_state(init)
        g.advance(1)
        for s in range(len(cfg.kinetic)):
            pid = g.particles(s)["pid"]
            keys = cell_keys(init["particles"][s]["q1"], cfg.Nx)
            np.testing.assert_array_equal(pid, np.argsort(keys, kind="stable"))


def test_mixed_moved_too_far(gpu_lib):
    cfg = h.configs.parity_p1().replace(precision=MIXED)
    init = read_state(os.path.join(GOLDEN, f"{cfg.name}.init.bin"))
    init["particles"][0]["vx"][5] = 2.0 * cfg.Dx / cfg.dt
    with h.Run(cfg, gpu_lib, "h1d_") as g:
        g.upload_state(init)
        with pytest.raises(h.MovedTooFar):
            g.advance(1)
