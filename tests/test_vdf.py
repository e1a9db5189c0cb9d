"""Host pieces of the equilibrium distributions of evolving weights (no GPU): Dawson's integral
that the counter-beam density B(nu) = 2 nu F(1/nu) needs (CounterBeamVDF.cc:14-17), and the
descriptors the C ABI receives for each distribution (h1d_kinetic_desc::vdf, vdf_param)."""
import math

import pytest

import hfemic_b200 as h


def test_dawson_against_scipy():
    special = pytest.importorskip("scipy.special")
    xs = [1e-6, 0.01, 0.1, 0.199, 0.2, 0.21, 0.5, 0.9, 1.0, 1.5, 2.0, 3.7, 5.0, 9.9, 20.0, 49.9, 50.1, 80.0, 1e3]
    for x in xs:
        ref = float(special.dawsn(x))
        assert abs(h.configs.dawson(x) - ref) <= 5e-15 * ref, x


def test_dawson_limits():
    # F(x) ~ x for small x, ~ 1/(2x) for large x; maximum 0.541044... at x = 0.924139
    assert h.configs.dawson(1e-8) == pytest.approx(1e-8, rel=1e-15)
    assert h.configs.dawson(1e4) == pytest.approx(0.5e-4, rel=1e-8)
    assert h.configs.dawson(0.9241388730) == pytest.approx(0.5410442246, rel=1e-9)


def test_vdf_descriptors():
    C = h.configs
    for name, kind in (("p9_losscone_psd_mirror", C.VDF_LOSSCONE), ("p10_pc_shell_psd_mirror", C.VDF_PARTIAL_SHELL),
                       ("p11_counterbeam_psd_mirror", C.VDF_COUNTER_BEAM)):
        cfg = C.PARITY[name]()
        p = h.abi.make_params(cfg)
        for s, k in enumerate(cfg.kinetic):
            d = p.kinetic[s]
            assert d.vdf == kind and k.has_psd
            assert tuple(d.vdf_param) == k.vdf_param()
            assert d.vth1 == math.sqrt(k.beta1) * cfg.c * abs(k.Oc) / k.op
    p9 = C.parity_p9()
    assert p9.kinetic[0].vdf_param() == (0.3, 0.0, 0.0)
    p10 = C.parity_p10()
    assert p10.kinetic[0].vdf_param()[0] == 2.0


def test_counter_beam_norm_override():
    """A caller-given PartSpecies::Nc replaces the computed one."""
    cfg = h.configs.parity_p11()
    k = cfg.kinetic[0]
    computed = cfg.moment_norm(k)
    k.norm = 123.0
    assert cfg.moment_norm(k) == 123.0 and computed != 123.0


# ---------------------------------------------------------------------------------------------
# the host loaders of every distribution (loader.load_other_species): statistics against the
# equilibrium moments, and against the particles of the reference's own loaders (golden fixtures)
# ---------------------------------------------------------------------------------------------

FAMILIES = ["p7_psd_tsc_mirror_reflecting", "p9_losscone_psd_mirror", "p10_pc_shell_psd_mirror",
            "p11_counterbeam_psd_mirror"]


def _physical(cfg, s):
    """species s as a full-f species with markers at the physical temperature"""
    import dataclasses
    kin = [dataclasses.replace(k, scheme=h.configs.FULL_F, marker_temp_ratio=1.0, psd_refresh_frequency=0.0)
           for k in cfg.kinetic]
    return cfg.replace(kinetic=kin)


@pytest.mark.parametrize("name", FAMILIES)
def test_loader_moments(name):
    """Positions follow n0(q1) and velocities the equilibrium's second moments (1 % on 2e5
    particles); full-f particles with physical markers have weight 1."""
    import numpy as np
    from hfemic_b200.loader import equilibrium, load_species
    base = h.configs.PARITY[name]()
    for s in range(len(base.kinetic)):
        cfg = _physical(base, s)
        k = cfg.kinetic[s]
        p = load_species(cfg, s, seed=11, count=200_000)
        np.testing.assert_allclose(p["w"], 1.0, rtol=1e-12)
        edges = np.linspace(cfg.q1min, cfg.q1max, cfg.Nx + 1)
        counts = np.histogram(p["q1"], edges)[0] / p["q1"].size
        fine = np.linspace(cfg.q1min, cfg.q1max, 64 * cfg.Nx + 1)
        n0 = equilibrium(cfg, k, 0.5 * (fine[1:] + fine[:-1]))[0]
        expect = n0.reshape(cfg.Nx, 64).sum(axis=1) / n0.sum()
        assert np.max(np.abs(counts / expect - 1)) < 0.01, name
        _, vpar2, vperp2 = equilibrium(cfg, k, p["q1"])
        assert abs(np.mean(p["vx"] ** 2 / vpar2) - 1) < 0.01, (name, s)
        assert abs(np.mean((p["vy"] ** 2 + p["vz"] ** 2) / (2 * vperp2)) - 1) < 0.01, (name, s)
        assert abs(np.mean(p["vy"] * p["vz"] / vperp2)) < 0.01


@pytest.mark.parametrize("name", FAMILIES)
def test_loader_hot_markers_and_delta_f(name):
    """Hot markers (marker_temp_ratio 2) carry weights f0/g0 whose weighted moments are the
    physical ones; delta-f particles carry real_f = f0 + w g0 with |w| <= initial_weight."""
    import dataclasses

    import numpy as np
    from hfemic_b200.loader import equilibrium, load_species, phase_space_density
    base = _physical(h.configs.PARITY[name](), 0)
    kin = [dataclasses.replace(k, marker_temp_ratio=2.0) for k in base.kinetic]
    cfg = base.replace(kinetic=kin)
    p = load_species(cfg, 0, seed=5, count=400_000)
    k = cfg.kinetic[0]
    f0 = phase_space_density(cfg, k, p["q1"], p["vx"], p["vy"], p["vz"])
    np.testing.assert_allclose(p["w"], f0 / p["marker"], rtol=1e-12)
    _, vpar2, vperp2 = equilibrium(cfg, k, p["q1"])
    assert abs(np.sum(p["w"] * p["vx"] ** 2 / vpar2) / np.sum(p["w"]) - 1) < 0.03, name
    assert abs(np.sum(p["w"] * (p["vy"] ** 2 + p["vz"] ** 2) / (2 * vperp2)) / np.sum(p["w"]) - 1) < 0.03, name
    assert abs(np.mean(p["w"]) - 1) < 0.03
    kd = dataclasses.replace(k, scheme=h.configs.DELTA_F, initial_weight=0.1)
    cd = cfg.replace(kinetic=[kd] + cfg.kinetic[1:])
    q = load_species(cd, 0, seed=5, count=10_000)
    assert np.all(np.abs(q["w"]) <= 0.1) and np.std(q["w"]) > 0.04
    f0 = phase_space_density(cd, kd, q["q1"], q["vx"], q["vy"], q["vz"])
    np.testing.assert_allclose(q["real_f"], f0 + q["w"] * q["marker"], rtol=1e-12)


@pytest.mark.parametrize("name", FAMILIES)
def test_loader_against_reference_loader(name):
    """The loader's particles against the reference loader's own (the fixture's initial state,
    1024 and 768 particles): the same position distribution (Kolmogorov-Smirnov distance) and
    the same second velocity moments and mean weights within the fixture's sampling error."""
    import os

    import numpy as np
    from state_io import read_state

    from hfemic_b200.loader import load_species
    cfg = h.configs.PARITY[name]()
    ref = read_state(os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", f"{name}.init.bin"))
    for s in range(len(cfg.kinetic)):
        r = ref["particles"][s]
        p = load_species(cfg, s, seed=3, count=100_000)
        a, b = np.sort(p["q1"]), np.sort(r["q1"])
        ks = np.max(np.abs(np.searchsorted(a, b, side="right") / a.size - np.arange(1, b.size + 1) / b.size))
        assert ks < 0.06, (name, s, ks)
        for key in ("vx", "vy"):
            m, mr = np.mean(p[key] ** 2), np.mean(r[key] ** 2)
            assert abs(m / mr - 1) < 0.25, (name, s, key, m, mr)
        if cfg.kinetic[s].scheme == h.configs.FULL_F:
            assert abs(np.mean(p["w"]) / np.mean(r["w"]) - 1) < 0.25, (name, s)
            assert abs(np.mean(p["marker"]) / np.mean(r["marker"]) - 1) < 0.25, (name, s)


def _equilibrium_only(lib, prefix, name):
    """moments of species 0 (delta-f) with every weight 0 after advance_by(0): the equilibrium
    n0, nvv0 times the moment weighting alone (PartSpecies.cc:129-143)"""
    import os

    import numpy as np
    from parity_util import with_reference_norms
    from state_io import read_state
    init = read_state(os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", f"{name}.init.bin"))
    cfg = with_reference_norms(h.configs.PARITY[name](), init)
    init["particles"][0]["w"][:] = 0.0
    with h.Run(cfg, lib, prefix) as r:
        r.upload_state(init)
        r.advance(0)
        return cfg, r.moments(0)


def check_equilibrium_moments(cfg, moments):
    import numpy as np

    from hfemic_b200.loader import equilibrium
    n, nV, nvv = moments
    P, Nx = 3, cfg.Nx
    n0, vpar2, vperp2 = equilibrium(cfg, cfg.kinetic[0], np.arange(Nx) + cfg.q1min + 0.5)
    np.testing.assert_allclose(n[P:P + Nx], n0, rtol=1e-13)
    np.testing.assert_allclose(nvv[P:P + Nx, 0], n0 * vpar2, rtol=1e-13)
    np.testing.assert_allclose(nvv[P:P + Nx, 1], n0 * vperp2, rtol=1e-13)
    np.testing.assert_allclose(nvv[P:P + Nx, 2], n0 * vperp2, rtol=1e-13)
    assert not np.any(nV) and not np.any(nvv[:, 3:]) and not np.any(n[:P]) and not np.any(n[P + Nx:])


@pytest.mark.parametrize("name", FAMILIES)
def test_oracle_equilibrium_moments(oracle_lib, name):
    """The oracle's delta-f equilibrium moments of every distribution against the loader's
    independent evaluation of the same formulas (agreement to rounding)."""
    check_equilibrium_moments(*_equilibrium_only(oracle_lib, "orc_", name))
