"""Evolving particle weights on the GPU (FP64): delta-f weights and phase-space density refresh
(PartSpecies::impl_update_weight, Core/PartSpecies.cc:178-208) with the delta-f equilibrium
moments (PartSpecies.cc:115-143), against the oracle and the reference's own fixtures.

p7 (CAM-CL, mirror, reflecting) holds a delta-f species with refresh beside a full-f species
loaded with hot markers (weights f0/g0) and refreshed; p8 is the predictor-corrector variant with
a delta-f species without refresh.  p9, p10 and p11 repeat p7 / p8 with the other equilibrium
distributions, loaded by the reference's own loaders: loss-cone, partial shell (PC, periodic) and
counter-beam.  Tolerances: as test_gpu_parity.py (1e-12 after one step, 1e-9 after ten), for the
weights, real_f and marker too; mixed precision within 1e-4 of FP64."""
import os

import numpy as np
import pytest
from parity_util import by_pid, rel_err, state_errors, with_reference_norms
from state_io import read_state

import hfemic_b200 as h

pytestmark = pytest.mark.gpu
GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
PSD = ["p7_psd_tsc_mirror_reflecting", "p8_pc_psd_periodic", "p9_losscone_psd_mirror", "p10_pc_shell_psd_mirror",
       "p11_counterbeam_psd_mirror"]


@pytest.mark.parametrize("name", PSD)
def test_weights_against_reference_fixture(name, gpu_lib):
    """Ten steps on the GPU against the reference's own output: fields, weights, real_f and the
    moments with the delta-f equilibrium added."""
    init = read_state(os.path.join(GOLDEN, f"{name}.init.bin"))
    cfg = with_reference_norms(h.configs.PARITY[name](), init)
    ref = read_state(os.path.join(GOLDEN, f"{name}.step10.bin"))
    with h.Run(cfg, gpu_lib) as g:
        g.upload_state(init)
        g.advance(10)
        st = g.state()
    for key in ("B", "E", "charge", "current"):
        assert rel_err(st[key], ref[key]) <= 1e-9, key
    for s in range(len(cfg.kinetic)):
        id0 = init["particles"][s]["id"]
        pg = by_pid(st["particles"][s])
        order = np.argsort(ref["particles"][s]["id"])  # reference order -> upload order (ids ascend with it)
        assert np.array_equal(id0, np.sort(id0))
        for key in ("q1", "w", "real_f", "marker"):
            assert rel_err(pg[key], ref["particles"][s][key][order]) <= 1e-9, (s, key)
        for key in ("n", "nV", "nvv"):
            assert rel_err(st["moments"][s][key], ref["moments"][s][key]) <= 1e-9, (s, key)
        # the weights did evolve
        assert rel_err(pg["w"], init["particles"][s]["w"]) > 1e-6


@pytest.mark.parametrize("name", PSD)
def test_mixed_precision_weights(name, gpu_lib):
    """The mixed-precision pass evolves the weights in FP32 (real_f and marker stored in FP32):
    weights and real_f within 1e-4 of the FP64 path after ten steps."""
    cfg = h.configs.PARITY[name]()
    init = read_state(os.path.join(GOLDEN, f"{name}.init.bin"))
    states = []
    for prec in (h.configs.PREC_FP64, h.configs.PREC_MIXED):
        with h.Run(cfg.replace(precision=prec), gpu_lib) as g:
            g.upload_state(init)
            g.advance(10)
            states.append(g.state())
    d, m = states
    for s in range(len(cfg.kinetic)):
        pd, pm = by_pid(d["particles"][s]), by_pid(m["particles"][s])
        for key in ("w", "real_f", "marker"):
            assert rel_err(pm[key], pd[key]) <= 1e-4, (s, key)
        assert rel_err(pm["w"], init["particles"][s]["w"]) > 1e-6  # the weights did evolve


def test_upload_psd_contract(gpu_lib):
    cfg = h.configs.parity_p7()
    init = read_state(os.path.join(GOLDEN, f"{cfg.name}.init.bin"))
    with h.Run(cfg, gpu_lib) as g:
        g.upload_state(init)
        p = init["particles"][0]
        with pytest.raises(ValueError):  # count differs from the uploaded particles
            g.upload_psd(0, p["real_f"][:-1], p["marker"][:-1])
        g.advance(1)
        with pytest.raises(ValueError):  # the particles were sorted since their upload
            g.upload_psd(0, p["real_f"], p["marker"])
    with h.Run(h.configs.parity_p2(), gpu_lib) as g:
        st = read_state(os.path.join(GOLDEN, "p2_tsc_mirror_reflecting.init.bin"))
        g.upload_state(st)
        with pytest.raises(ValueError):  # the weights of this species do not evolve
            g.upload_psd(0, st["particles"][0]["w"], np.ones(st["particles"][0]["w"].size))


@pytest.mark.parametrize("name", ["p7_psd_tsc_mirror_reflecting", "p11_counterbeam_psd_mirror"])
@pytest.mark.parametrize("precision,tol", [(h.configs.PREC_FP64, 1e-12), (h.configs.PREC_MIXED, 1e-5)])
def test_resume_with_evolving_weights(gpu_lib, name, precision, tol):
    cfg = h.configs.PARITY[name]().replace(precision=precision)
    init = read_state(os.path.join(GOLDEN, f"{cfg.name}.init.bin"))
    with h.Run(cfg, gpu_lib) as a:
        a.upload_state(init)
        a.advance(4)
        image = h.abi.checkpoint(a)
        a.advance(4)
        sa = a.state()
    with h.Run(cfg, gpu_lib) as b:
        h.abi.restore(b, image)
        b.advance(4)
        sb = b.state()
    errs = state_errors(sb, sa, cfg)
    assert "particles[0].real_f" in errs
    assert max(errs.values()) <= tol, errs


def test_vhistogram_psd_columns(gpu_lib, oracle_lib):
    """The recorder's third column is real_f / marker per particle."""
    cfg = h.configs.parity_p7()
    init = read_state(os.path.join(GOLDEN, f"{cfg.name}.init.bin"))
    specs = dict(extent=(cfg.q1min + cfg.Nx / 8, cfg.Nx * 0.75), v1=(-6.0, 12.0, 24), v2=(0.0, 8.0, 16))
    with h.Run(cfg, gpu_lib) as g, h.Run(cfg, oracle_lib, "orc_") as o:
        g.upload_state(init)
        o.upload_state(init)
        g.advance(3)
        o.advance(3)
        for s in range(len(cfg.kinetic)):
            hg, tg = h.abi.vhistogram(g, s, **specs)
            ho, to = h.abi.vhistogram(o, s, prefix="orc_", **specs)
            assert tg == to and to > 0
            assert np.abs(hg[..., 0] - ho[..., 0]).sum() * to <= 2
            same = hg[..., 0] == ho[..., 0]  # bins holding the same particles on both sides
            assert same.mean() > 0.95
            np.testing.assert_allclose(hg[..., 2][same], ho[..., 2][same], rtol=1e-9, atol=1e-14)
            if s == 1:  # full-f with hot markers: real_f / marker is the weight, not 1
                np.testing.assert_allclose(hg[..., 2][same], hg[..., 1][same], rtol=1e-9, atol=1e-14)


def test_device_loader_refuses_evolving_weights(gpu_lib):
    cfg = h.configs.parity_p7()
    with h.Run(cfg, gpu_lib) as r:
        with pytest.raises(ValueError):
            h.abi.populate(r, 0, seed=1, count=1000)
    # a full-f species of another distribution: the device loader draws bi-Maxwellians only
    import dataclasses
    cfg = h.configs.parity_p9()
    kin = [dataclasses.replace(k, scheme=h.configs.FULL_F, psd_refresh_frequency=0.0, marker_temp_ratio=1.0)
           for k in cfg.kinetic]
    with h.Run(cfg.replace(kinetic=kin), gpu_lib) as r:
        with pytest.raises(ValueError):
            h.abi.populate(r, 0, seed=1, count=1000)


@pytest.mark.parametrize("name", PSD[2:])
def test_loader_states_against_oracle(name, gpu_lib, oracle_lib):
    """States drawn by the host loader for each equilibrium distribution (128 and 96 particles per
    cell, real_f / marker included) advance on the GPU as in the oracle: ten steps within 1e-9."""
    from hfemic_b200.loader import initial_state

    cfg = h.configs.PARITY[name]()
    for k in cfg.kinetic:
        k.Nc *= 8
    init = initial_state(cfg, seed=17)
    with h.Run(cfg, gpu_lib, "h1d_") as g, h.Run(cfg, oracle_lib, "orc_") as c:
        g.upload_state(init)
        c.upload_state(init)
        g.advance(10)
        c.advance(10)
        errs = state_errors(g.state(), c.state(), cfg)
    bad = {k: v for k, v in errs.items() if not v <= 1e-9}
    assert not bad, bad


@pytest.mark.parametrize("name", PSD[:1] + PSD[2:])
def test_equilibrium_moments(name, gpu_lib):
    """The library's delta-f equilibrium moments (n0, nvv0 of every distribution, computed on the
    host at create) against the loader's independent evaluation: zero weights after
    advance_by(0) leave the equilibrium alone."""
    from test_vdf import _equilibrium_only, check_equilibrium_moments

    check_equilibrium_moments(*_equilibrium_only(gpu_lib, "h1d_", name))
