"""Seeded synthetic initial state for a run: bi-Maxwellian kinetic species, cold fluid at rest,
zero wave fields.

Follows the distributions of the reference loader MaxwellianVDF::load
(src/LibPIC/PIC/VDF/MaxwellianVDF.cc:300-319, with N_of_q1 / q1_of_N :229-250 and eta :218-228):
  - position: q1 = q1_of_N(u * N_len + N_loc) with u a base-2 radical-inverse sequence;
  - v_par = sqrt(-log U) sin(2 pi u3) vth1, v_perp = sqrt(-log U' * T2/T1(q1)) (cos, sin)(2 pi u5) vth1
    with u3, u5 base-3/base-5 radical-inverse sequences and U, U' uniform draws;
  - full-f weight 1 (marker distribution equal to the physical one).
The reference draws U, U' from std::mt19937 seeded with fixed constants; here they come from a
numpy PCG64 generator seeded per run, and the radical-inverse sequences start at a seeded offset,
so runs with different seeds are independent.  Cold species start with n = 1, nV = 0
(ColdSpecies.cc:238-249); B and E start at zero.
"""
from __future__ import annotations

import math

import numpy as np

from .configs import RunConfig, _q1_of_n, _n_of_q1

PAD = 3


def radical_inverse(base: int, k: np.ndarray) -> np.ndarray:
    """Van der Corput sequence value of the integers k in the given base, in [0, 1)."""
    k = np.asarray(k, dtype=np.uint64).copy()
    out = np.zeros(k.shape, dtype=np.float64)
    f = 1.0 / base
    b = np.uint64(base)
    while np.any(k):
        out += (k % b).astype(np.float64) * f
        k //= b
        f /= base
    return out


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
    rng = np.random.Generator(np.random.PCG64([seed, s, 0x9E3779B9]))
    offset = int(rng.integers(1, 1 << 40))
    idx = np.arange(offset, offset + n, dtype=np.uint64)
    eps = 1e-15
    u2 = eps + (1 - 2 * eps) * radical_inverse(2, idx)
    u3 = eps + (1 - 2 * eps) * radical_inverse(3, idx)
    u5 = eps + (1 - 2 * eps) * radical_inverse(5, idx)
    N_loc = _n_of_q1(cfg, k, cfg.q1min)
    N_len = _n_of_q1(cfg, k, cfg.q1max) - N_loc
    q1 = _q1_of_n_vec(cfg, k, u2 * N_len + N_loc)
    q1 = np.clip(q1, cfg.q1min, np.nextafter(cfg.q1max, cfg.q1min))
    U1 = rng.uniform(eps, 1 - eps, n)
    U2 = rng.uniform(eps, 1 - eps, n)
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
