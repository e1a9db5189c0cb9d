"""Seeded synthetic initial state for a run: bi-Maxwellian kinetic species, cold fluid at rest,
zero wave fields.

Follows the distributions of the reference loader MaxwellianVDF::load
(src/LibPIC/PIC/VDF/MaxwellianVDF.cc:300-319, with N_of_q1 / q1_of_N :229-250 and eta :218-228):
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
n = 1, nV = 0 (ColdSpecies.cc:238-249); B and E start at zero.
"""
from __future__ import annotations

import math

import numpy as np

from .configs import RunConfig, _q1_of_n, _n_of_q1

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
