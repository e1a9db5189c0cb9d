"""Seeded synthetic initial state for a run: kinetic species drawn from their equilibrium
distribution (bi-Maxwellian, loss-cone, partial shell or counter-beam), cold fluid at rest, zero
wave fields.

Follows the distributions of the reference loader MaxwellianVDF::load
(src/LibPIC/PIC/VDF/MaxwellianVDF.cc:115-134, with N_of_q1 / q1_of_N :44-65 and eta :33-43):
  - position: q1 = q1_of_N(u2 * N_len + N_loc) with u2 the base-2 radical inverse of the particle's
    sequence index;
  - v_par = sqrt(-log U1) sin(2 pi u3) vth1, v_perp = sqrt(-log U2 * T2/T1(q1)) (cos, sin)(2 pi u5)
    vth1 with u3, u5 base-3/base-5 radical inverses of the same index;
  - full-f weight 1 (marker distribution equal to the physical one).
The reference draws U1, U2 from std::mt19937 seeded with fixed constants and starts every sequence
at index 1.  Here a run's seed picks the sequences' starting index and U1, U2 are counter-based
draws (the splitmix64 finalizer of seed, species and particle index), so that runs with different
seeds are independent and the same draws can be made on the device: h1d_populate computes exactly
these particles (up to the last bit of the device's tan/atan/log/sin/cos).  Cold species start with
n = 1, nV = 0 (ColdSpecies.cc:18-29); B and E start at zero.

The other distributions follow their reference loaders with the same kind of draws
(load_other_species): positions from the inverse of N(q1) = int n0 dq1 at the base-2 radical
inverse (LossconeVDF.cc:154, PartialShellVDF.cc:177, CounterBeamVDF.cc:169-175; here the
inverse is a fine table of the integral of n0 instead of the reference's closed forms or its
stepped integration); loss-cone perpendicular speeds by the reference's rejection sampler against
a Gaussian of spread alpha = max(beta, 1) + 0.3 (LossconeVDF.cc:162, 171-213); partial-shell pitch
angles and shell speeds by inverting their cumulative distributions (PartialShellVDF.cc:94-124,
173-192); counter-beam pitch angles by rejection under exp(-sin^2 a / nu^2) sin a with a coin
flip into the second quadrant (CounterBeamVDF.cc:165-224).  Velocities are drawn from the marker
distribution g0 (the physical one heated by marker_temp_ratio); every species carries its
phase-space density real_f = f0, marker = g0 and the weight of its scheme: f0/g0 (full-f) or
initial_weight U(-1, 1) with real_f = f0 + w g0 (delta-f), as the reference's emit functions set
them (MaxwellianVDF.cc:96-114, LossconeVDF.cc:131-149).
"""
from __future__ import annotations

import math

import numpy as np

from .configs import (VDF_BIMAXWELLIAN, VDF_COUNTER_BEAM, VDF_LOSSCONE, VDF_PARTIAL_SHELL, DELTA_F, RunConfig,
                      _q1_of_n, _n_of_q1, dawson)

PAD = 3


M64 = (1 << 64) - 1
GOLDEN = 0x9E3779B97F4A7C15


def mix64(z):
    """splitmix64 finalizer on uint64 arrays (wrapping arithmetic)."""
    z = np.asarray(z, dtype=np.uint64)
    with np.errstate(over="ignore"):
        z = (z ^ (z >> np.uint64(30))) * np.uint64(0xBF58476D1CE4E5B9)
        z = (z ^ (z >> np.uint64(27))) * np.uint64(0x94D049BB133111EB)
    return z ^ (z >> np.uint64(31))


def species_key(seed: int, s: int) -> int:
    """Key of species s of a run with this seed; its sequence offset is 1 + key_offset(key)."""
    k0 = int(mix64(np.uint64((seed ^ 0x243F6A8885A308D3) & M64)))
    return int(mix64(np.uint64((k0 + s * GOLDEN) & M64)))


def sequence_offset(key: int) -> int:
    return 1 + (int(mix64(np.uint64(key ^ 0x13198A2E03707344))) >> 24)


def bit_reverse64(x: np.ndarray) -> np.ndarray:
    x = np.asarray(x, dtype=np.uint64).copy()
    for sh, m in ((1, 0x5555555555555555), (2, 0x3333333333333333), (4, 0x0F0F0F0F0F0F0F0F),
                  (8, 0x00FF00FF00FF00FF), (16, 0x0000FFFF0000FFFF)):
        sh, m = np.uint64(sh), np.uint64(m)
        x = ((x >> sh) & m) | ((x & m) << sh)
    return (x >> np.uint64(32)) | (x << np.uint64(32))


def radical_inverse(base: int, k: np.ndarray) -> np.ndarray:
    """Van der Corput sequence value of the integers k (< 2^53) in the given base, in [0, 1)."""
    k = np.asarray(k, dtype=np.uint64).copy()
    if base == 2:  # the reversed bits, exactly
        return (bit_reverse64(k) >> np.uint64(11)).astype(np.float64) * 2.0 ** -53
    out = np.zeros(k.shape, dtype=np.float64)
    f = 1.0 / base
    b = np.uint64(base)
    while np.any(k):
        out += (k % b).astype(np.float64) * f
        k //= b
        f /= base
    return out


def uniform(key: int, i: np.ndarray, j: int) -> np.ndarray:
    """Counter-based uniform draw j (1 or 2) of particle i, in [eps, 1 - eps]."""
    eps = 1e-15
    with np.errstate(over="ignore"):
        c = np.uint64(key) + (np.asarray(i, dtype=np.uint64) * np.uint64(2) + np.uint64(j)) * np.uint64(GOLDEN)
    u = (mix64(c) >> np.uint64(11)).astype(np.float64) * 2.0 ** -53
    return eps + (1 - 2 * eps) * u


def _q1_of_n_vec(cfg: RunConfig, k, N: np.ndarray) -> np.ndarray:
    T2OT1 = k.T2_T1
    if cfg.homogeneous:
        xiD1N = cfg.xi * cfg.Dx * N
        return N * (1 + (xiD1N * xiD1N) * (T2OT1 - 1) / 3)
    s = math.sqrt(T2OT1)
    return np.arctan(np.tan(s * cfg.Dx * cfg.xi * N) / s) / (cfg.xi * cfg.Dx)


def load_species(cfg: RunConfig, s: int, seed: int = 0, count: int | None = None):
    k = cfg.kinetic[s]
    if k.vdf != VDF_BIMAXWELLIAN or k.has_psd or k.marker_temp_ratio != 1.0:
        return load_other_species(cfg, s, seed, count)
    n = k.Nc * cfg.Nx if count is None else count
    key = species_key(seed, s)
    i = np.arange(n, dtype=np.uint64)
    idx = np.uint64(sequence_offset(key)) + i
    eps = 1e-15
    u2 = eps + (1 - 2 * eps) * radical_inverse(2, idx)
    u3 = eps + (1 - 2 * eps) * radical_inverse(3, idx)
    u5 = eps + (1 - 2 * eps) * radical_inverse(5, idx)
    N_loc = _n_of_q1(cfg, k, cfg.q1min)
    N_len = _n_of_q1(cfg, k, cfg.q1max) - N_loc
    q1 = _q1_of_n_vec(cfg, k, u2 * N_len + N_loc)
    q1 = np.clip(q1, cfg.q1min, np.nextafter(cfg.q1max, cfg.q1min))
    U1 = uniform(key, i, 1)
    U2 = uniform(key, i, 2)
    c = np.cos(cfg.xi * cfg.Dx * q1)
    eta = 1.0 / (k.T2_T1 + (1 - k.T2_T1) * c * c)
    T2OT1 = k.T2_T1 * eta
    vth1 = k.vth1(cfg.c)
    x1 = np.sqrt(-np.log(U1)) * np.sin(2 * math.pi * u3)
    tmp = np.sqrt(-np.log(U2) * T2OT1)
    x2 = np.cos(2 * math.pi * u5) * tmp
    x3 = np.sin(2 * math.pi * u5) * tmp
    return dict(q1=q1, vx=x1 * vth1, vy=x2 * vth1, vz=x3 * vth1, w=np.ones(n))


# ---------------------------------------------------------------------------------------------
# every equilibrium distribution, with its phase-space density
# ---------------------------------------------------------------------------------------------

def _losscone_beta_eq(k) -> float:
    b = k.losscone_beta
    if b < 1e-10:
        return 1e-10
    return b + math.copysign(1e-10, b - 1) if abs(b - 1) < 1e-10 else b


def _shell_speed_norm(xs: float):
    """A(xs) and T / vth^2 of the shell speed distribution x^2 exp(-(x - xs)^2)."""
    sqrt_pi = math.sqrt(math.pi)
    Ab = .5 * (xs * math.exp(-xs * xs) + sqrt_pi * (.5 + xs * xs) * math.erfc(-xs))
    T = .5 / Ab * (xs * (2.5 + xs * xs) * math.exp(-xs * xs) + sqrt_pi * (0.75 + xs * xs * (3 + xs * xs)) * math.erfc(-xs))
    return Ab, T


def equilibrium(cfg: RunConfig, k, q1):
    """n0(q1) and the field-aligned second moments <v_par^2>, <v_perp,1^2> (= <v_perp,2^2>) per
    particle of the species' equilibrium distribution (VDF::n0 / nvv0 divided by n0)."""
    q1 = np.asarray(q1, dtype=np.float64)
    c = np.cos(cfg.xi * cfg.Dx * q1)
    vth = k.vth1(cfg.c)
    if k.vdf == VDF_LOSSCONE:
        b = _losscone_beta_eq(k)
        X = k.T2_T1 / (1 + b)
        eta = 1 / (X + (1 - X) * c * c)
        eta_b = 1 / (b * X + (1 - b * X) * c * c)
        beta = b * eta_b / eta
        return (eta - b * eta_b) / (1 - b), np.full_like(q1, .5 * vth * vth), .5 * vth * vth * (1 + beta) * X * eta
    if k.vdf == VDF_PARTIAL_SHELL:
        _, T = _shell_speed_norm(k.vs / vth)
        T1 = T / (3 + k.zeta) * vth * vth
        n0 = np.ones_like(q1) if k.zeta == 0 else c ** k.zeta
        return n0, np.full_like(q1, T1), np.full_like(q1, T1 * (2 + k.zeta) / 2)
    if k.vdf == VDF_COUNTER_BEAM:
        _, T = _shell_speed_norm(k.vs / vth)
        nu = k.nu / c
        F = dawson(1 / nu)
        t1 = 0.5 * nu * (1 / F - nu)
        n0 = (2 * nu * F) / (2 * k.nu * dawson(1 / k.nu))
        return n0, t1 * T * vth * vth, 0.5 * (1 - t1) * T * vth * vth
    eta = 1 / (k.T2_T1 + (1 - k.T2_T1) * c * c)
    return eta, np.full_like(q1, .5 * vth * vth), .5 * vth * vth * k.T2_T1 * eta


def phase_space_density(cfg: RunConfig, k, q1, vx, vy, vz, temp_ratio: float = 1.0):
    """f0(v, q1) of the species' equilibrium (VDF::f0), or with temp_ratio = marker_temp_ratio the
    marker density g0 (the same distribution with vth scaled by sqrt(temp_ratio))."""
    q1 = np.asarray(q1, dtype=np.float64)
    vth = k.vth1(cfg.c) * math.sqrt(temp_ratio)
    c = np.cos(cfg.xi * cfg.Dx * q1)
    x1, x2, x3 = np.asarray(vx) / vth, np.asarray(vy) / vth, np.asarray(vz) / vth
    n0, _, _ = equilibrium(cfg, k, q1)
    if k.vdf == VDF_LOSSCONE:
        b = _losscone_beta_eq(k)
        X = k.T2_T1 / (1 + b)
        eta = 1 / (X + (1 - X) * c * c)
        eta_b = 1 / (b * X + (1 - b * X) * c * c)
        beta = b * eta_b / eta
        beta = np.where(np.abs(beta - 1) < 1e-10, beta + np.copysign(1e-10, beta - 1), beta)
        xth2 = X * eta
        y = (x2 * x2 + x3 * x3) / xth2
        f2 = (np.exp(-y) - np.exp(-y / beta)) / (math.pi * xth2 * (1 - beta))
        return n0 * (np.exp(-x1 * x1) / math.sqrt(math.pi) * f2 / vth ** 3)
    if k.vdf in (VDF_PARTIAL_SHELL, VDF_COUNTER_BEAM):
        xs = k.vs / vth
        Ab, _ = _shell_speed_norm(xs)
        x = np.sqrt(x1 * x1 + x2 * x2 + x3 * x3)
        fv = np.exp(-(x - xs) ** 2) / Ab
        u = x1 / x
        if k.vdf == VDF_PARTIAL_SHELL:
            Bz = math.sqrt(math.pi) * math.gamma(1 + .5 * k.zeta) / math.gamma(1.5 + .5 * k.zeta)
            fa = (1.0 if k.zeta == 0 else ((1 - u) * (1 + u)) ** (.5 * k.zeta)) / Bz
            return n0 * (.5 * fv * fa / (math.pi * vth ** 3))
        B0 = 2 * k.nu * dawson(1 / k.nu)
        return fv * np.exp(-((1 - u) * (1 + u)) * c * c / (k.nu * k.nu)) / B0 / (2 * math.pi * vth ** 3)
    T2OT1 = k.T2_T1 * n0
    return n0 * (np.exp(-x1 * x1) / math.sqrt(math.pi) * np.exp(-(x2 * x2 + x3 * x3) / T2OT1) / (math.pi * T2OT1) / vth ** 3)


def _inverse_cdf(density, lo: float, hi: float, u: np.ndarray, n: int = 1 << 16) -> np.ndarray:
    """x with int_lo^x density = u int_lo^hi density, from a trapezoid table of n intervals."""
    x = np.linspace(lo, hi, n + 1)
    d = density(x)
    F = np.concatenate([[0.0], np.cumsum(0.5 * (d[1:] + d[:-1]) * np.diff(x))])
    return np.interp(u * F[-1], F, x)


def _rejection(accept, key: int, n: int, propose):
    """Per-particle rejection sampling: rounds of counter-based draws (a fresh key per round) until
    every particle accepted a proposal; ``propose(u, idx)`` maps uniforms of the pending particles
    to proposals, ``accept(x, u, idx)`` votes on them."""
    out = np.empty(n)
    pending = np.arange(n, dtype=np.int64)
    for rnd in range(1000):
        if pending.size == 0:
            return out
        kr = int(mix64(np.uint64((key ^ (0xA5A5A5A5 + rnd * 0x9E3779B9)) & M64)))
        idx = pending.astype(np.uint64)
        x = propose(uniform(kr, idx, 1), pending)
        ok = accept(x, uniform(kr, idx, 2), pending)
        out[pending[ok]] = x[ok]
        pending = pending[~ok]
    raise RuntimeError("rejection sampling did not converge")


def load_other_species(cfg: RunConfig, s: int, seed: int = 0, count: int | None = None):
    """Particles of species s from its equilibrium distribution with their phase-space densities
    (module docstring); any distribution, any scheme and marker temperature."""
    k = cfg.kinetic[s]
    n = k.Nc * cfg.Nx if count is None else count
    key = species_key(seed, s)
    i = np.arange(n, dtype=np.uint64)
    idx = np.uint64(sequence_offset(key)) + i
    eps = 1e-15
    u2 = eps + (1 - 2 * eps) * radical_inverse(2, idx)
    u3 = eps + (1 - 2 * eps) * radical_inverse(3, idx)
    u5 = eps + (1 - 2 * eps) * radical_inverse(5, idx)
    U1 = uniform(key, i, 1)
    vth = k.vth1(cfg.c) * math.sqrt(k.marker_temp_ratio)  # marker thermal speed
    hi = np.nextafter(cfg.q1max, cfg.q1min)
    if k.vdf == VDF_BIMAXWELLIAN:
        N_loc = _n_of_q1(cfg, k, cfg.q1min)
        N_len = _n_of_q1(cfg, k, cfg.q1max) - N_loc
        q1 = np.clip(_q1_of_n_vec(cfg, k, u2 * N_len + N_loc), cfg.q1min, hi)
    else:
        q1 = np.clip(_inverse_cdf(lambda q: equilibrium(cfg, k, q)[0], cfg.q1min, cfg.q1max, u2), cfg.q1min, hi)
    c = np.cos(cfg.xi * cfg.Dx * q1)
    ph = 2 * math.pi * u5
    if k.vdf in (VDF_BIMAXWELLIAN, VDF_LOSSCONE):
        x1 = np.sqrt(-np.log(U1)) * np.sin(2 * math.pi * u3)
        if k.vdf == VDF_BIMAXWELLIAN:
            tmp = np.sqrt(-np.log(uniform(key, i, 2)) * (k.T2_T1 / (k.T2_T1 + (1 - k.T2_T1) * c * c)))
        else:  # LossconeVDF::RejectionSampler with beta(q1), then the perpendicular thermal spread
            b = _losscone_beta_eq(k)
            X = k.T2_T1 / (1 + b)
            eta = 1 / (X + (1 - X) * c * c)
            eta_b = 1 / (b * X + (1 - b * X) * c * c)
            beta = b * eta_b / eta
            beta = np.where(np.abs(beta - 1) < 1e-10, beta + np.copysign(1e-10, beta - 1), beta)
            alpha = np.where(beta < 1, 1.0, beta) + 0.3
            with np.errstate(divide="ignore", invalid="ignore"):
                det = -beta / (1 - beta) * np.log(((alpha - 1) * beta) / (alpha - beta))
            xpk = np.where(np.isfinite(det) & (det > 0), np.sqrt(np.where(det > 0, det, 0)), 0.0)

            def fOg(x, j):
                x2_ = x * x
                return ((np.exp(-x2_) - np.exp(-x2_ / beta[j])) / (1 - beta[j])) / (np.exp(-x2_ / alpha[j]) / alpha[j])
            M = fOg(xpk, np.arange(n))
            r = _rejection(lambda x, u, j: u * M[j] <= fOg(x, j), key, n,
                           lambda u, j: np.sqrt(-np.log(u) * alpha[j]))
            tmp = r * np.sqrt(X * eta)
        x2, x3 = np.cos(ph) * tmp, np.sin(ph) * tmp
    else:
        xs = k.vs / vth
        t_min = -min(xs, 5.0)
        x = _inverse_cdf(lambda v: v * v * np.exp(-(v - xs) ** 2), t_min + xs, 5.0 + xs, U1)
        if k.vdf == VDF_PARTIAL_SHELL:
            a = _inverse_cdf(lambda t: np.abs(np.sin(t)) ** (k.zeta + 1), 0.0, math.pi, u3)
        else:
            nu = k.nu / c
            a_max = np.arcsin(np.minimum(1.0, 4 * nu))

            def fa(t, j):
                st = np.sin(t)
                return np.exp(-st * st / (nu[j] * nu[j])) * st
            f_peak = fa(np.arcsin(np.minimum(1.0, nu * math.sqrt(0.5))), np.arange(n))
            a = _rejection(lambda t, u, j: u * f_peak[j] <= fa(t, j), key ^ 0x5151, n, lambda u, j: u * a_max[j])
            coin = uniform(key, i, 2) - 0.5
            a = np.where(coin > 0, math.pi - a, a)
        x1 = np.cos(a) * x
        x2, x3 = np.cos(ph) * np.sin(a) * x, np.sin(ph) * np.sin(a) * x
    vx, vy, vz = x1 * vth, x2 * vth, x3 * vth
    f0 = phase_space_density(cfg, k, q1, vx, vy, vz)
    g0 = phase_space_density(cfg, k, q1, vx, vy, vz, k.marker_temp_ratio)
    if k.scheme == DELTA_F:
        key_w = int(mix64(np.uint64(key ^ 0x7777)))
        w = k.initial_weight * (uniform(key_w, i, 1) * 2 - 1)
        real_f = f0 + w * g0
    else:
        w, real_f = f0 / g0, f0
    return dict(q1=q1, vx=vx, vy=vy, vz=vz, w=w, real_f=real_f, marker=g0)


def initial_state(cfg: RunConfig, seed: int = 0, fraction: float = 1.0):
    """State dict in the layout used by Run.upload_state.  ``fraction`` < 1 loads a subset
    of the particles (a bounded sample of the configuration)."""
    M = cfg.Nx + 2 * PAD
    parts = []
    for s, k in enumerate(cfg.kinetic):
        count = max(1, int(round(k.Nc * cfg.Nx * fraction)))
        parts.append(load_species(cfg, s, seed, count))
    cold = []
    for _ in cfg.cold:
        n_full = np.zeros(M)
        n_full[PAD:PAD + cfg.Nx] = 1.0
        cold.append(dict(n_full=n_full, nV_full=np.zeros((M, 3))))
    return dict(particles=parts, B=np.zeros((M, 3)), E=np.zeros((M, 3)), cold=cold)
