"""Ensembles (h1d_batch_*) and the autotuner against runs advanced alone.

A batch member computes exactly what the same run computes alone: the kernels are the same and
only the order of floating-point atomic additions differs.  Tolerances (max-norm relative):
1e-10 for FP64 members and 1e-4 (the mixed-precision tolerance) for mixed-precision members,
after 40 steps with CUDA-graph replays in between.  The autotuner only reorders particles, so a
tuned run still matches the oracle.
"""
import numpy as np
import pytest
from parity_util import by_pid, rel_err, state_errors

import hfemic_b200 as h

pytestmark = pytest.mark.gpu


def _members(precision, n=4, ppc_scale=0.05):
    from hfemic_b200.loader import initial_state

    cfgs = [h.configs.ensemble_member(seed, precision=precision, ppc_scale=ppc_scale) for seed in range(n)]
    return cfgs, [initial_state(c, seed=i) for i, c in enumerate(cfgs)]


def _field_errs(a, b, cfg):
    errs = {k: rel_err(a[k], b[k]) for k in ("B", "E", "charge", "current")}
    for s in range(len(cfg.kinetic)):
        for key in ("n", "nV", "nvv"):
            errs[f"moments[{s}].{key}"] = rel_err(a["moments"][s][key], b["moments"][s][key])
    return errs


@pytest.mark.parametrize("precision,tol", [(h.configs.PREC_FP64, 1e-10), (h.configs.PREC_MIXED, 1e-4)])
def test_batch_members_match_runs_alone(gpu_lib, precision, tol):
    cfgs, states = _members(precision)
    alone = []
    for c, st in zip(cfgs, states):
        with h.Run(c, gpu_lib) as r:
            h.abi.configure(r, sort_interval=4)
            r.upload_state(st)
            r.advance(40)
            alone.append(r.state())
    runs = [h.Run(c, gpu_lib) for c in cfgs]
    try:
        for r, st in zip(runs, states):
            h.abi.configure(r, sort_interval=4)
            r.upload_state(st)
        with h.abi.Batch(runs) as b:
            b.configure(sort_interval=4)
            b.advance(3)   # part of a block, eager
            b.advance(37)  # the rest of the block, graph pairs of 8 steps, eager tail
            stats = b.stats()
            assert stats["steps"] == 40
            assert stats["graph_launches"] >= 2 and stats["graphs_built"] == 1
            together = [r.state() for r in runs]
    finally:
        for r in runs:
            r.close()
    for c, a, t in zip(cfgs, alone, together):
        errs = _field_errs(t, a, c)
        print(c.name, c.Nx, {k: f"{v:.1e}" for k, v in errs.items()})
        assert max(errs.values()) <= tol, errs
        pa, pt = by_pid(a["particles"][0]), by_pid(t["particles"][0])
        assert rel_err(pt["vx"], pa["vx"]) <= tol


def test_batch_without_graphs_equals_with_graphs(gpu_lib):
    cfgs, states = _members(h.configs.PREC_FP64, n=2)
    out = []
    for graphs in (False, True):
        runs = [h.Run(c, gpu_lib) for c in cfgs]
        for r, st in zip(runs, states):
            r.upload_state(st)
        with h.abi.Batch(runs) as b:
            b.configure(sort_interval=4, use_graphs=graphs)
            b.advance(24)
            assert (b.stats()["graph_launches"] > 0) == graphs
        out.append([r.state() for r in runs])
        for r in runs:
            r.close()
    for c, a, t in zip(cfgs, out[0], out[1]):
        assert max(_field_errs(t, a, c).values()) <= 1e-10


def test_batch_rejects_bad_members(gpu_lib):
    c = h.configs.parity_p1()
    with h.Run(c, gpu_lib) as r:
        with pytest.raises(h.H1DError):
            h.abi.Batch([r, r])
        with h.abi.Batch([r]):
            with pytest.raises(h.H1DError):
                h.abi.Batch([r])


def test_autotuned_run_matches_oracle(gpu_lib, oracle_lib):
    from hfemic_b200.loader import initial_state

    cfg = h.configs.parity_p2().replace(Nx=256, xi=0.01, phase_retardation=(32, 1.0), amplitude_damping=(32, 0.2))
    for k in cfg.kinetic:
        k.Nc = 100
    init = initial_state(cfg, seed=4)
    with h.Run(cfg, gpu_lib) as g:
        g.upload_state(init)
        steps, k, c = h.abi.autotune(g)
        assert k in (8, 12, 16, 24, 32) and 1 <= c <= 3  # FP64 pass: up to 3 CTAs per SM
        assert steps == 2 * (8 + 12 + 16 + 24 + 32) + 3 * 2 * k
        g.advance(3)
        gs = g.state()
    with h.Run(cfg, oracle_lib, "orc_") as o:
        o.upload_state(init)
        o.advance(steps + 3)
        cs = o.state()
    errs = state_errors(gs, cs, cfg)
    print("autotuned", steps, k, c, {key: f"{v:.1e}" for key, v in errs.items()})
    assert max(errs.values()) <= 1e-9


def test_batch_member_with_external_source(gpu_lib):
    """A run with an external current source advances in a batch (eager steps: its source times
    are per step) exactly as alone."""
    import os

    from state_io import read_state

    golden = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
    cfgs = [h.configs.parity_p5(), h.configs.parity_p1()]
    inits = [read_state(os.path.join(golden, f"{c.name}.init.bin")) for c in cfgs]
    alone = []
    for c, st in zip(cfgs, inits):
        with h.Run(c, gpu_lib) as r:
            r.upload_state(st)
            r.advance(10)
            alone.append(r.state())
    runs = [h.Run(c, gpu_lib) for c in cfgs]
    try:
        for r, st in zip(runs, inits):
            r.upload_state(st)
        with h.abi.Batch(runs) as b:
            b.configure(sort_interval=4)
            b.advance(10)
            assert b.stats()["graph_launches"] == 0
            together = [r.state() for r in runs]
    finally:
        for r in runs:
            r.close()
    for c, a, t in zip(cfgs, alone, together):
        assert max(_field_errs(t, a, c).values()) <= 1e-12


@pytest.mark.parametrize("precision,tol", [(h.configs.PREC_FP64, 1e-10), (h.configs.PREC_MIXED, 1e-4)])
def test_batch_with_evolving_weights(gpu_lib, precision, tol):
    """Members whose weights evolve (delta-f over bi-Maxwellian, loss-cone and counter-beam
    equilibria, PSD refresh) beside a plain member: 20 batch steps (graph replays included) equal
    each run alone, weights and phase-space densities included."""
    import os

    from parity_util import with_reference_norms
    from state_io import read_state

    golden = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
    names = ["p7_psd_tsc_mirror_reflecting", "p9_losscone_psd_mirror", "p11_counterbeam_psd_mirror",
             "p2_tsc_mirror_reflecting"]
    states = [read_state(os.path.join(golden, f"{n}.init.bin")) for n in names]
    cfgs = [with_reference_norms(h.configs.PARITY[n](), st).replace(precision=precision) for n, st in zip(names, states)]
    alone = []
    for c, st in zip(cfgs, states):
        with h.Run(c, gpu_lib) as r:
            h.abi.configure(r, sort_interval=4)
            r.upload_state(st)
            r.advance(20)
            alone.append(r.state())
    runs = [h.Run(c, gpu_lib) for c in cfgs]
    try:
        for r, st in zip(runs, states):
            h.abi.configure(r, sort_interval=4)
            r.upload_state(st)
        with h.abi.Batch(runs) as b:
            b.configure(sort_interval=4)
            b.advance(20)
            assert b.stats()["steps"] == 20
            together = [r.state() for r in runs]
    finally:
        for r in runs:
            r.close()
    for c, a, t in zip(cfgs, alone, together):
        errs = state_errors(t, a, c)
        assert any(k.endswith("real_f") for k in errs) or not any(k.has_psd for k in c.kinetic)
        bad = {k: v for k, v in errs.items() if not v <= tol}
        assert not bad, (c.name, bad)


def _fixture_members(names, precision):
    import os

    from parity_util import with_reference_norms
    from state_io import read_state

    golden = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
    states = [read_state(os.path.join(golden, f"{n}.init.bin")) for n in names]
    return [with_reference_norms(h.configs.PARITY[n](), st).replace(precision=precision)
            for n, st in zip(names, states)], states


def _alone_and_together(gpu_lib, cfgs, states, steps, chunks=(3,)):
    alone = []
    for c, st in zip(cfgs, states):
        with h.Run(c, gpu_lib) as r:
            h.abi.configure(r, sort_interval=4)
            r.upload_state(st)
            r.advance(steps)
            alone.append(r.state())
    runs = [h.Run(c, gpu_lib) for c in cfgs]
    try:
        for r, st in zip(runs, states):
            h.abi.configure(r, sort_interval=4)
            r.upload_state(st)
        with h.abi.Batch(runs) as b:
            b.configure(sort_interval=4)
            done = 0
            for k in chunks:
                b.advance(k)
                done += k
            b.advance(steps - done)
            stats = b.stats()
            together = [r.state() for r in runs]
    finally:
        for r in runs:
            r.close()
    return alone, together, stats


@pytest.mark.parametrize("precision,tol", [(h.configs.PREC_FP64, 1e-10), (h.configs.PREC_MIXED, 1e-4)])
def test_pc_batch_members_match_runs_alone(gpu_lib, precision, tol):
    """Predictor-corrector members (TSC mirror reflecting, delta-f periodic, partial-shell delta-f):
    40 batch steps with CUDA-graph replays equal each run alone (Domain_PC::advance_by)."""
    names = ["p4_pc_tsc_mirror_reflecting", "p8_pc_psd_periodic", "p10_pc_shell_psd_mirror"]
    cfgs, states = _fixture_members(names, precision)
    alone, together, stats = _alone_and_together(gpu_lib, cfgs, states, 40)
    assert stats["steps"] == 40 and stats["graph_launches"] >= 2
    for c, a, t in zip(cfgs, alone, together):
        errs = state_errors(t, a, c)
        bad = {k: v for k, v in errs.items() if not v <= tol}
        assert not bad, (c.name, bad)


def test_pc_batch_with_external_source(gpu_lib):
    """A predictor-corrector member with an antenna current (its source times change every step,
    so the batch runs eagerly) beside a plain one."""
    names = ["p6_pc_source", "p4_pc_tsc_mirror_reflecting"]
    cfgs, states = _fixture_members(names, h.configs.PREC_FP64)
    alone, together, stats = _alone_and_together(gpu_lib, cfgs, states, 12)
    assert stats["graph_launches"] == 0
    for c, a, t in zip(cfgs, alone, together):
        errs = state_errors(t, a, c)
        bad = {k: v for k, v in errs.items() if not v <= 1e-10}
        assert not bad, (c.name, bad)


def test_batch_members_share_one_algorithm(gpu_lib):
    a = h.Run(h.configs.parity_p2(), gpu_lib)
    c = h.Run(h.configs.parity_p4(), gpu_lib)
    try:
        with pytest.raises(h.H1DError):
            h.abi.Batch([a, c])
    finally:
        a.close(), c.close()


def test_batch_sort_is_each_members_stable_cell_sort(gpu_lib):
    """The batch sorts every species of every member in one launch set (one histogram, scan and
    scatter launch per radix pass over all segments, with digits sized for the widest grid).  With
    a sort before every step, each species' device order after one step is exactly the CPU stable
    sort, by its own full-grid cell, of its uploaded particles: members of 64 to 4096 cells (keys
    of 7 and 13 bits, sorted together in two passes), with one and two species, FP64."""
    import os

    from hfemic_b200.loader import initial_state
    from parity_util import cell_keys
    from state_io import read_state

    golden = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
    p2 = h.configs.parity_p2()
    cfgs = [p2, h.configs.ensemble_member(0, precision=h.configs.PREC_FP64, ppc_scale=0.2),
            h.configs.ensemble_member(1, precision=h.configs.PREC_FP64, ppc_scale=0.2)]
    states = [read_state(os.path.join(golden, f"{p2.name}.init.bin"))]
    states += [initial_state(c, seed=i) for i, c in enumerate(cfgs[1:], 1)]
    runs = [h.Run(c, gpu_lib) for c in cfgs]
    try:
        for r, st in zip(runs, states):
            r.upload_state(st)
        with h.abi.Batch(runs) as b:
            b.configure(sort_interval=1, use_graphs=False)
            b.advance(1)
        for c, r, st in zip(cfgs, runs, states):
            for s in range(len(c.kinetic)):
                pid = r.particles(s)["pid"]
                keys = cell_keys(np.asarray(st["particles"][s]["q1"]), c.Nx)
                np.testing.assert_array_equal(pid, np.argsort(keys, kind="stable"), err_msg=f"{c.name} species {s}")
    finally:
        for r in runs:
            r.close()


def _alone(gpu_lib, cfgs, states, totals):
    out = []
    for c, st, n in zip(cfgs, states, totals):
        with h.Run(c, gpu_lib) as r:
            h.abi.configure(r, sort_interval=4)
            r.upload_state(st)
            if n:
                r.advance(n)
            out.append(r.state())
    return out


def _members_by_counts(gpu_lib, cfgs, states, counts, then):
    runs = [h.Run(c, gpu_lib) for c in cfgs]
    try:
        for r, st in zip(runs, states):
            h.abi.configure(r, sort_interval=4)
            r.upload_state(st)
        with h.abi.Batch(runs) as b:
            b.configure(sort_interval=4)
            b.advance_members(counts)  # each member by its own count, eager
            b.advance(then)            # then all together again, graph pairs included
            steps = [h.abi.step_count(r) for r in runs]
            together = [r.state() for r in runs]
    finally:
        for r in runs:
            r.close()
    return steps, together


@pytest.mark.parametrize("precision,tol", [(h.configs.PREC_FP64, 1e-10), (h.configs.PREC_MIXED, 1e-4)])
def test_batch_members_advance_by_their_own_counts(gpu_lib, precision, tol):
    """h1d_batch_advance_members_async: members advanced by 13, 40, 0 and 27 steps (the one with 0
    stays as it was), then all by 17 more, equal each run advanced alone by its total."""
    cfgs, states = _members(precision)
    counts, then = [13, 40, 0, 27], 17
    totals = [c + then for c in counts]
    steps, together = _members_by_counts(gpu_lib, cfgs, states, counts, then)
    assert steps == totals
    for c, a, t in zip(cfgs, _alone(gpu_lib, cfgs, states, totals), together):
        errs = _field_errs(t, a, c)
        assert max(errs.values()) <= tol, (c.name, errs)
        pa, pt = by_pid(a["particles"][0]), by_pid(t["particles"][0])
        assert rel_err(pt["vx"], pa["vx"]) <= tol


def test_pc_batch_members_advance_by_their_own_counts(gpu_lib):
    """The same for predictor-corrector members (TSC mirror reflecting; delta-f periodic)."""
    names = ["p4_pc_tsc_mirror_reflecting", "p8_pc_psd_periodic"]
    cfgs, states = _fixture_members(names, h.configs.PREC_FP64)
    counts, then = [7, 12], 5
    totals = [c + then for c in counts]
    steps, together = _members_by_counts(gpu_lib, cfgs, states, counts, then)
    assert steps == totals
    for c, a, t in zip(cfgs, _alone(gpu_lib, cfgs, states, totals), together):
        errs = state_errors(t, a, c)
        bad = {k: v for k, v in errs.items() if not v <= 1e-10}
        assert not bad, (c.name, bad)
