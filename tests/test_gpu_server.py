"""The serving loop (h1d_server_*): continuous batching under an HBM budget.

A request's results are the same whether it runs alone or among other requests that arrive,
join and leave while it is on the device: FP64 within 1e-10 and mixed precision within 1e-4
(max-norm relative over fields, energies and moments).  A request served equals the same run
built and advanced directly through h1d_create / h1d_populate / h1d_advance.
"""
import numpy as np
import pytest
from parity_util import rel_err

import hfemic_b200 as h

pytestmark = pytest.mark.gpu
GB = 1 << 30


def _cfg(seed, precision, ppc_scale=0.05):
    return h.configs.ensemble_member(seed, precision=precision, ppc_scale=ppc_scale)


def _drain(sv, ids, max_ticks=100000):
    for _ in range(max_ticks):
        a, q = sv.tick()
        if all(sv.poll(i)["state"] >= h.abi.REQ_DONE for i in ids):
            return
    raise AssertionError("requests did not finish")


def _errs(x, y):
    return {k: rel_err(x[k], y[k]) for k in ("B", "E", "dB2O2", "dE2O2", "KE", "n", "nV", "nvv")}


@pytest.mark.parametrize("precision,tol", [(h.configs.PREC_FP64, 1e-10), (h.configs.PREC_MIXED, 1e-4)])
def test_result_same_alone_and_in_mix(gpu_lib, precision, tol):
    x = _cfg(5, precision)
    with h.abi.Server(gpu_lib, 8 * GB, steps_per_tick=16, sort_interval=8) as sv:
        i = sv.submit(x, seed=5, n_steps=96)
        _drain(sv, [i])
        alone = sv.result(i)
    with h.abi.Server(gpu_lib, 8 * GB, steps_per_tick=16, sort_interval=8) as sv:
        early = [sv.submit(_cfg(s, precision), seed=s, n_steps=n) for s, n in ((1, 40), (2, 200))]
        sv.tick()
        i = sv.submit(x, seed=5, n_steps=96)  # joins a running batch
        sv.tick()
        late = [sv.submit(_cfg(s, h.configs.PREC_FP64), seed=s, n_steps=n) for s, n in ((3, 24), (4, 130))]
        _drain(sv, early + [i] + late)
        mixed = sv.result(i)
        st = sv.stats()
        assert st["completed"] == 5 and st["failed"] == 0
        assert st["batches_built"] >= 4
    errs = _errs(mixed, alone)
    print(precision, {k: f"{v:.1e}" for k, v in errs.items()})
    assert max(errs.values()) <= tol, errs


def test_served_equals_direct_run(gpu_lib):
    cfg = _cfg(6, h.configs.PREC_FP64)
    with h.abi.Server(gpu_lib, 8 * GB, steps_per_tick=32, sort_interval=16) as sv:
        i = sv.submit(cfg, seed=6, n_steps=64)
        _drain(sv, [i])
        res = sv.result(i)
    with h.Run(cfg.replace(sort_interval=16), gpu_lib) as r:
        h.abi.populate_state(r, seed=6)
        r.advance(64)
        B, E = r.fields()
        e = r.energy()
        n, nV, nvv = r.moments(0)
    assert rel_err(res["B"], B) <= 1e-10 and rel_err(res["E"], E) <= 1e-10
    assert rel_err(res["dB2O2"], e["dB2O2"]) <= 1e-10
    assert rel_err(res["n"][0], n) <= 1e-10 and rel_err(res["nvv"][0], nvv) <= 1e-10


def test_predictor_corrector_requests(gpu_lib):
    """Predictor-corrector requests are served beside CAM-CL ones (one batch per algorithm) and
    equal the same runs driven directly (Domain_PC::advance_by)."""
    pc = [_cfg(s, h.configs.PREC_FP64).replace(algorithm=h.configs.ALGO_PC) for s in (7, 8)]
    with h.abi.Server(gpu_lib, 8 * GB, steps_per_tick=16, sort_interval=16) as sv:
        ids = [sv.submit(c, seed=s, n_steps=n) for c, s, n in zip(pc, (7, 8), (48, 80))]
        ids.append(sv.submit(_cfg(9, h.configs.PREC_FP64), seed=9, n_steps=64))
        _drain(sv, ids)
        res = [sv.result(i) for i in ids[:2]]
        assert sv.stats()["completed"] == 3 and sv.stats()["failed"] == 0
    for c, s, n, got in zip(pc, (7, 8), (48, 80), res):
        with h.Run(c.replace(sort_interval=16), gpu_lib) as r:
            h.abi.populate_state(r, seed=s)
            r.advance(n)
            B, E = r.fields()
            nn, _, nvv = r.moments(0)
        assert rel_err(got["B"], B) <= 1e-10 and rel_err(got["E"], E) <= 1e-10
        assert rel_err(got["n"][0], nn) <= 1e-10 and rel_err(got["nvv"][0], nvv) <= 1e-10


def test_admission_respects_budget(gpu_lib):
    """A budget that holds the two largest requests but not three: the server never exceeds it,
    never runs all six together, and finishes them all."""
    cfgs = [_cfg(s, h.configs.PREC_MIXED) for s in range(6)]
    sizes = sorted((_estimate(c) for c in cfgs), reverse=True)
    budget = sizes[0] + sizes[1] + sizes[-1] // 2
    with h.abi.Server(gpu_lib, budget, steps_per_tick=16) as sv:
        ids = [sv.submit(c, seed=s, n_steps=48) for s, c in enumerate(cfgs)]
        peak_active = 0
        for _ in range(100000):
            a, q = sv.tick()
            peak_active = max(peak_active, a)
            assert sv.stats()["bytes_in_use"] <= budget
            if all(sv.poll(i)["state"] >= h.abi.REQ_DONE for i in ids):
                break
        st = sv.stats()
        assert st["completed"] == 6 and st["peak_bytes"] <= budget
        assert peak_active < 6


def _estimate(cfg):
    """The server's admission estimate, restated: particles in two buffer sets with ids and sort
    keys, sort histograms, grids."""
    M = cfg.Nx + 6
    per = 20 if cfg.precision == h.configs.PREC_MIXED else 40
    b = 0
    for k in cfg.kinetic:
        n = k.Nc * cfg.Nx + 64
        b += 2 * n * (per + 12) + (n // 2048 + 1) * 256 * 4 * 2
    b += 8 * M * (17 + 18 + 6 + 1 + 3 + 6 + 8 * 36 + 4 * 17)
    return b + (1 << 20)


def test_oversize_request_is_refused(gpu_lib):
    with h.abi.Server(gpu_lib, 1 << 20, steps_per_tick=16) as sv:
        with pytest.raises(h.H1DError):
            sv.submit(_cfg(0, h.configs.PREC_FP64), seed=0, n_steps=10)


def test_requests_the_device_loader_cannot_build_are_refused(gpu_lib):
    """Served runs are built by h1d_populate (bi-Maxwellian, full-f): a species of another
    distribution, or with evolving weights, is refused at submission."""
    import dataclasses
    base = _cfg(0, h.configs.PREC_FP64)
    with h.abi.Server(gpu_lib, 8 << 30, steps_per_tick=16) as sv:
        for change in (dict(vdf=h.configs.VDF_LOSSCONE, losscone_beta=0.3), dict(scheme=h.configs.DELTA_F)):
            cfg = base.replace(kinetic=[dataclasses.replace(base.kinetic[0], **change)] + base.kinetic[1:])
            with pytest.raises(h.H1DError):
                sv.submit(cfg, seed=0, n_steps=10)


def test_failing_member_fails_alone(gpu_lib):
    """A request whose particles move more than a cell per step (PartSpecies::update_pos's
    domain_error) fails with H1D_ERR_MOVED_TOO_FAR while the requests batched with it complete
    with the results they have alone."""
    good = [(_cfg(s, h.configs.PREC_FP64), s, n) for s, n in ((11, 48), (12, 80))]
    hot = _cfg(13, h.configs.PREC_FP64)
    hot.kinetic[0].beta1 = 500.0  # thermal speed of a few cells per step
    with h.abi.Server(gpu_lib, 8 * GB, steps_per_tick=16, sort_interval=8) as sv:
        ids = [sv.submit(c, seed=s, n_steps=n) for c, s, n in good]
        bad = sv.submit(hot, seed=13, n_steps=64)
        _drain(sv, ids + [bad])
        assert sv.poll(bad)["state"] == h.abi.REQ_FAILED and sv.poll(bad)["status"] == h.abi.ERR_MOVED_TOO_FAR
        assert all(sv.poll(i)["state"] == h.abi.REQ_DONE for i in ids)
        got = [sv.result(i) for i in ids]
        st = sv.stats()
        assert st["completed"] == 2 and st["failed"] == 1
    for (c, s, n), res in zip(good, got):
        with h.abi.Server(gpu_lib, 8 * GB, steps_per_tick=16, sort_interval=8) as sv:
            i = sv.submit(c, seed=s, n_steps=n)
            _drain(sv, [i])
            alone = sv.result(i)
        errs = _errs(res, alone)
        assert max(errs.values()) <= 1e-10, errs


def test_submit_and_poll_do_not_wait_for_a_tick(gpu_lib):
    """While one thread runs a long tick (a large request, a quantum of many steps), submit and
    poll from another thread return at once: the server's lock is not held while the GPU works."""
    import threading
    import time

    big = h.configs.ensemble_member(21, precision=h.configs.PREC_FP64, ppc_scale=1.0).replace(Nx=4096, xi=0.001)
    big.kinetic[0].Nc = 1000
    with h.abi.Server(gpu_lib, 40 * GB, steps_per_tick=1500, sort_interval=16) as sv:
        i = sv.submit(big, seed=21, n_steps=1500)
        sv.tick()  # admits and builds the run; it joins the batch at the next tick
        t = {}

        def long_tick():
            t0 = time.perf_counter()
            sv.tick()
            t["tick"] = time.perf_counter() - t0

        th = threading.Thread(target=long_tick)
        th.start()
        time.sleep(0.05)
        calls = []
        while th.is_alive():
            t0 = time.perf_counter()
            j = sv.submit(_cfg(22, h.configs.PREC_FP64), seed=22, n_steps=8)
            sv.poll(i)
            sv.poll(j)
            calls.append(time.perf_counter() - t0)
            time.sleep(0.01)
        th.join()
        print(f"tick {t['tick']:.3f} s, {len(calls)} submit+poll rounds, slowest {max(calls) * 1e3:.2f} ms")
        assert t["tick"] > 0.2 and len(calls) >= 5
        assert max(calls) < 0.05 * t["tick"]
