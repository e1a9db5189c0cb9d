"""Pin the oracle's primitives against the known answers of the reference's own LibPIC unit
tests (src/LibPIC/test/*.cc of kyungguk1/hybrid_code-hfemic_wave), restated here."""
import ctypes as C
import math

import numpy as np
import pytest

dp = C.POINTER(C.c_double)
lp = C.POINTER(C.c_int64)


@pytest.fixture(scope="module")
def lib(oracle_cdll):
    L = oracle_cdll
    L.orc_shape.argtypes = [C.c_int, C.c_double, lp, dp]
    L.orc_boris.argtypes = [C.c_double] * 4 + [dp, dp, dp]
    L.orc_mask.argtypes = [C.c_int64, C.c_double, C.c_double]
    L.orc_mask.restype = C.c_double
    L.orc_geometry.argtypes = [C.c_double] * 5 + [dp]
    L.orc_grid_smooth.argtypes = [C.c_int64, dp, dp]
    L.orc_grid_deposit.argtypes = [C.c_int, C.c_double, C.c_double, dp]
    L.orc_grid_interp.argtypes = [C.c_int, C.c_double, dp]
    L.orc_grid_interp.restype = C.c_double
    return L


def shape(lib, order, x):
    i = np.zeros(4, dtype=np.int64)
    w = np.zeros(4)
    lib.orc_shape(order, x, i.ctypes.data_as(lp), w.ctypes.data_as(dp))
    return i[: order + 1], w[: order + 1]


def test_shape1_indices_and_weights(lib):  # test-Shape.cc:14-50
    for x in np.arange(0.0, 3.0, 0.1):
        i, w = shape(lib, 1, x)
        k = math.floor(x)
        assert list(i) == [k, k + 1]
        assert abs(w.sum() - 1) < 1e-10
        assert abs((x - k) - w[1]) < 1e-10


def test_shape2_indices_and_weights(lib):  # test-Shape.cc:52-84
    for x in np.arange(10.0, 11.0, 0.1):
        i, w = shape(lib, 2, x)
        k = int(math.floor(x + 0.5))  # std::round, half away from zero (x > 0)
        assert list(i) == [k - 1, k, k + 1]
        assert abs(w.sum() - 1) < 1e-10


def test_shape3_indices_and_weights(lib):  # test-Shape.cc:86-119
    for x in np.arange(10.0, 11.0, 0.1):
        i, w = shape(lib, 3, x)
        k = math.ceil(x)
        assert list(i) == [k - 2, k - 1, k, k + 1]
        assert abs(w.sum() - 1) < 1e-10


def test_shape_round_half_away_from_zero(lib):
    # Shape<2> uses std::round: -0.5 -> -1, 0.5 -> 1, 2.5 -> 3
    assert shape(lib, 2, -0.5)[0][1] == -1
    assert shape(lib, 2, 0.5)[0][1] == 1
    assert shape(lib, 2, 2.5)[0][1] == 3


def _push(lib, boris_args, v, B, E):
    v = np.asarray(v, dtype=float).copy()
    B = np.asarray(B, dtype=float)
    E = np.asarray(E, dtype=float)
    lib.orc_boris(*boris_args, v.ctypes.data_as(dp), B.ctypes.data_as(dp), E.ctypes.data_as(dp))
    return v


def test_boris_gyration_and_driven(lib):  # test-BorisPush.cc:36-72
    nt = 360
    args = (1.0, 1.0, 1.0, 2 * math.pi / nt)
    v = np.array([1.0, 0, 0])
    for _ in range(nt):
        v = _push(lib, args, v, [0, 0, 1], [0, 0, 0])
        assert abs(v @ v - 1) < 1e-15 and v[2] == 0
    vs = [np.zeros(3)]
    for t in range(nt):
        E = [0, 0, math.cos(2 * math.pi * (t + 0.5) / nt)]
        vs.append(_push(lib, args, vs[-1], [0, 0, 0], E))
    vs = vs[1:]
    assert all(v[0] == 0 and v[1] == 0 for v in vs)
    rms = sum(v @ v for v in vs) / len(vs)
    assert rms == pytest.approx(0.50001269258580949284, rel=1e-10)


def test_boris_harmonic_oscillator(lib):  # test-BorisPush.cc:74-106
    nt, w0 = 360, 2 * math.pi
    dt = 2 * math.pi / w0 / nt
    args = (dt, 1.0, 1.0, 1.0)
    xs, vs = [0.0], [np.array([1.0, 0, 0])]
    xs[-1] += 0.5 * dt * vs[-1][0]
    for _ in range(nt):
        F = [-w0 * w0 * xs[-1], 0, 0]
        vs.append(_push(lib, args, vs[-1], [0, 0, 0], F))
        xs.append(xs[-1] + dt * vs[-1][0])
    xs2 = sum(x * x for x in xs[1:]) * w0 * w0 / nt
    vs2 = sum(v @ v for v in vs[1:]) / nt
    assert xs2 == pytest.approx(0.5, rel=1e-4)
    assert vs2 == pytest.approx(0.5, rel=1e-4)


def geometry(lib, xi, D1, x, y=0.0, z=0.0):
    out = np.zeros(7)
    lib.orc_geometry(xi, D1, x, y, z, out.ctypes.data_as(dp))
    return out


def test_geometry_known_answers(lib):  # test-Geometry.cc:100-213
    g = geometry(lib, 1e-11, 0.1, 14.5, 10, 20)  # homogeneous
    assert g[0] * 0.1 == pytest.approx(14.5, rel=1e-10)
    assert g[1] == pytest.approx(14.5, rel=1e-10)
    assert g[2] == pytest.approx(1, rel=1e-15) and abs(g[3]) < 1e-15 and abs(g[4]) < 1e-15
    g = geometry(lib, 0.112, 2.0, 14.5, 10, 20)  # inhomogeneous
    assert g[0] * 2 == pytest.approx(9.09702270985558, rel=1e-10)
    assert g[1] == pytest.approx(14.5, rel=1e-10)
    assert g[2] == pytest.approx(3.637376, rel=1e-10)
    assert g[3] == pytest.approx(-1.8188800000000003, rel=1e-10)
    assert g[4] == pytest.approx(-3.6377600000000005, rel=1e-10)
    assert g[5] == pytest.approx(3.637376, rel=1e-10)  # |B|/B0 = 1 + xi^2 x^2
    # contravariant basis: v^1 = v_x cos^2 / D1 = v_x / (D1 * B/B0)
    assert g[6] == pytest.approx(1 / (2 * 3.637376), rel=1e-10)


def test_masking_function(lib):  # test-MaskingFunction.cc:12-51
    assert lib.orc_mask(0, 0.0, 0) == 1 and lib.orc_mask(0, 0.0, 1) == 1
    for off in (0, 1, 2):
        assert lib.orc_mask(0, 0.5, off) == pytest.approx(1, rel=1e-10)
        assert lib.orc_mask(10, 0.0, off) == pytest.approx(1, rel=1e-10)
    assert lib.orc_mask(10, 0.5, 0) == pytest.approx(1 - 0.25, rel=1e-10)
    for off in (10, -10, 11, -11):
        assert lib.orc_mask(10, 0.5, off) == pytest.approx(1, rel=1e-10)
    for i in range(-10, 11):
        exact = 1 - (0.5 * (abs(i) - 10) / 10) ** 2
        assert lib.orc_mask(10, 0.5, float(i)) == pytest.approx(exact, rel=1e-10)


def test_grid_smooth_deposit_interp(lib):  # test-GridArray.cc:246-316
    P, N = 3, 10
    src = np.zeros(N + 2 * P)
    src[4 + P] = 1
    dst = np.zeros_like(src)
    lib.orc_grid_smooth(N, src.ctypes.data_as(dp), dst.ctypes.data_as(dp))
    assert dst.sum() == pytest.approx(1, rel=1e-15)
    assert (dst[3 + P], dst[4 + P], dst[5 + P]) == (0.25, 0.5, 0.25)
    g = np.zeros(N + 2 * P)
    lib.orc_grid_deposit(1, -1.0, 10.0, g.ctypes.data_as(dp))
    assert g[-1 + P] == 10 and np.count_nonzero(g) == 1
    g[:] = 0
    lib.orc_grid_deposit(1, N - 1e-15, 10.0, g.ctypes.data_as(dp))
    assert g[N + P] == pytest.approx(10, rel=1e-10)
    g[:] = 0
    lib.orc_grid_deposit(1, 4.14, 10.0, g.ctypes.data_as(dp))
    _, w = shape(lib, 1, 4.14)
    assert g[4 + P] == 10 * w[0] and g[5 + P] == 10 * w[1]
    assert abs(10 - g.sum()) / 10 < 1e-15
    for order in (1, 2, 3):
        g[:] = 0
        lib.orc_grid_deposit(order, 4.3, 1.0, g.ctypes.data_as(dp))
        assert abs(g.sum() - 1) < 1e-15
    g[:] = 0
    g[4 + P] = 10
    for x, j in ((3.9, 1), (4.1, 0), (4.9, 0)):
        _, w = shape(lib, 1, x)
        assert lib.orc_grid_interp(1, x, g.ctypes.data_as(dp)) == 10 * w[j]
