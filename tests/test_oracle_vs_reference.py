"""Pin the oracle to the reference itself: starting from particles made by the reference's own
loader, one and ten steps of the oracle reproduce the reference's Domain::advance_by bit for
bit (fixtures made by tests/golden/make_golden.py from the compiled reference sources)."""
import os

import numpy as np
import pytest
from parity_util import with_reference_norms
from state_io import read_state

import hfemic_b200 as h

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def compare_states(mine, ref, cfg, exact=True, rtol=0.0):
    """Return a list of mismatches; ``exact`` compares bit patterns (NaN == NaN)."""
    errs = []

    def cmp(name, a, b):
        a, b = np.asarray(a), np.asarray(b)
        if a.shape != b.shape:
            errs.append(f"{name}: shape {a.shape} != {b.shape}")
        elif exact:
            if not np.array_equal(a, b, equal_nan=True):
                errs.append(f"{name}: max |diff| {np.nanmax(np.abs(a - b)):.3e}")
        else:
            scale = max(np.nanmax(np.abs(b)), 1e-300)
            d = np.nanmax(np.abs(a - b)) / scale
            if not d <= rtol:
                errs.append(f"{name}: rel {d:.3e} > {rtol}")

    for s in range(len(cfg.kinetic)):
        p, q = mine["particles"][s], ref["particles"][s]
        for key in ("q1", "vx", "vy", "vz", "w"):
            cmp(f"particles[{s}].{key}", p[key], q[key])
        if cfg.kinetic[s].has_psd:  # phase-space densities of evolving weights
            for key in ("real_f", "marker"):
                cmp(f"particles[{s}].{key}", p[key], q[key])
        m, r = mine["moments"][s], ref["moments"][s]
        for key in ("n", "nV", "nvv"):
            cmp(f"moments[{s}].{key}", m[key], r[key])
    for key in ("B", "E", "charge", "current"):
        cmp(key, mine[key], ref[key])
    for i in range(len(cfg.cold)):
        for key in ("n_full", "nV_full", "n", "nV", "nvv"):
            cmp(f"cold[{i}].{key}", mine["cold"][i][key], ref["cold"][i][key])
    return errs


@pytest.mark.parametrize("name", sorted(h.configs.PARITY))
@pytest.mark.parametrize("steps", [1, 10])
def test_oracle_bit_exact_vs_reference(oracle_lib, name, steps):
    """Bit for bit, except for the counter-beam equilibrium (configs.PARITY_ROUNDING): its density
    and f0 need Dawson's integral, which the reference takes from the Faddeeva package
    (LibPIC/PIC/Misc/Faddeeva.cc) and the oracle evaluates by its own method, and its PartSpecies::Nc
    comes from the reference's numerical integration of the density (VDFHelper.h:47-70, about
    1e-9 from the exact integral), so there the oracle takes Nc from the state file and agrees to
    rounding (8e-15 in the weights after ten steps; bound 1e-13)."""
    cfg = h.configs.PARITY[name]()
    init = read_state(os.path.join(GOLDEN, f"{name}.init.bin"))
    ref = read_state(os.path.join(GOLDEN, f"{name}.step{steps}.bin"))
    exact = name not in h.configs.PARITY_ROUNDING
    # the reference normalises moments with PartSpecies::Nc; the config must give the same value
    norms = [cfg.moment_norm(k) for k in cfg.kinetic]
    if exact:
        assert norms == list(init["moment_norm"])
    else:
        np.testing.assert_allclose(norms, init["moment_norm"], rtol=1e-8)
        cfg = with_reference_norms(cfg, init)
    with h.Run(cfg, oracle_lib, "orc_") as run:
        run.upload_state(init)
        run.advance(steps)
        mine = run.state()
    errs = compare_states(mine, ref, cfg, exact=exact, rtol=1e-13)
    assert not errs, errs
    # particle order: the oracle's upload index maps to the reference's global particle id
    for s in range(len(cfg.kinetic)):
        id0 = init["particles"][s]["id"]
        np.testing.assert_array_equal(id0[mine["particles"][s]["pid"]], ref["particles"][s]["id"])


def test_oracle_moved_too_far(oracle_lib):
    """A particle faster than one cell per step raises like PartSpecies::update_pos."""
    cfg = h.configs.parity_p1()
    init = read_state(os.path.join(GOLDEN, f"{cfg.name}.init.bin"))
    init["particles"][0]["vx"][5] = 2.0 * cfg.Dx / cfg.dt
    with h.Run(cfg, oracle_lib, "orc_") as run:
        run.upload_state(init)
        with pytest.raises(h.MovedTooFar):
            run.advance(1)


def test_oracle_rejects_invalid_params(oracle_lib):
    cfg = h.configs.parity_p2().replace(xi=1.0)  # |xi*D1*q1| >= pi/2 (ParamSet.cc:25-29)
    with pytest.raises(ValueError):
        cfg.validate()
    cfg = h.configs.parity_p1().replace(n_subcycles=1)
    with pytest.raises(ValueError):
        h.Run(cfg, oracle_lib, "orc_")
