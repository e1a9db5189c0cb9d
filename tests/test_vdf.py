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
