"""The device loader (h1d_populate) against the host loader (loader.load_species).

Both evaluate the same radical-inverse sequences and counter-based uniforms with the same
arithmetic; they differ only in the last bits of tan/atan/cos/log/sin (CUDA's against the host's
C library).  Tolerances: positions within 1e-12 (absolute, in cells), velocities within 1e-13
(max-norm relative); in mixed precision the position is the host position rounded to the nearest
2^-F cell (F = configs.position_fraction_bits(Nx)), so the cell index of every particle equals
floor(q1 - q1min) of the host position except within half a step 2^-F of a cell boundary, where
rounding may carry it across (within half a step of q1max the position stays on the grid's last
position, up to one step away), and the velocities equal the host's FP32 rounding.
"""
import numpy as np
import pytest
from parity_util import rel_err

import hfemic_b200 as h
from hfemic_b200.loader import load_species

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("xi", [0.0, 0.002])
@pytest.mark.parametrize("precision", [h.configs.PREC_FP64, h.configs.PREC_MIXED])
def test_populate_matches_host_loader(gpu_lib, xi, precision):
    cfg = h.configs.ensemble_member(7, precision=precision, ppc_scale=0.2).replace(xi=xi)  # Nx = 4096 at most
    cfg.validate()
    host = load_species(cfg, 0, seed=123)
    with h.Run(cfg, gpu_lib) as r:
        h.abi.populate(r, 0, seed=123)
        dev = r.particles(0)
    np.testing.assert_array_equal(dev["pid"], np.arange(host["q1"].size))
    if precision == h.configs.PREC_FP64:
        assert np.max(np.abs(dev["q1"] - host["q1"])) <= 1e-12
        for key in ("vx", "vy", "vz"):
            assert rel_err(dev[key], host[key]) <= 1e-13, key
    else:
        step = 2.0 ** -h.configs.position_fraction_bits(cfg.Nx)
        x = host["q1"] - cfg.q1min
        tol = 0.5 * step + 1e-11  # half a fixed-point step, plus the loaders' last-bit differences
        near = np.abs(x - np.round(x)) <= tol
        cell_d = np.floor(dev["q1"] - cfg.q1min)
        assert np.array_equal(cell_d[~near], np.floor(x)[~near])
        # within half a step of q1max the position is kept on the grid's last position instead
        edge = x > cfg.Nx - tol
        assert np.max(np.abs(dev["q1"] - host["q1"])[~edge], initial=0.0) <= tol
        assert np.max(np.abs(dev["q1"] - host["q1"])[edge], initial=0.0) <= step + 1e-11
        assert np.all(dev["q1"] < cfg.q1max)
        for key in ("vx", "vy", "vz"):
            assert rel_err(dev[key], host[key].astype(np.float32)) <= 1e-6, key
    assert np.all(dev["w"] == 1.0)


def test_populated_run_matches_uploaded_run(gpu_lib):
    """A run populated on the device advances like the same run uploaded from the host loader."""
    from hfemic_b200.loader import initial_state

    cfg = h.configs.ensemble_member(3, precision=h.configs.PREC_FP64, ppc_scale=0.1)
    st = initial_state(cfg, seed=11)
    with h.Run(cfg, gpu_lib) as a, h.Run(cfg, gpu_lib) as b:
        a.upload_state(st)
        h.abi.populate_state(b, seed=11)
        a.advance(20)
        b.advance(20)
        ea, eb = a.energy(), b.energy()
        ma, mb = a.moments(0), b.moments(0)
    for key in ("dB2O2", "dE2O2", "KE_lab"):
        assert rel_err(eb[key], ea[key]) <= 1e-9, key
    for x, y in zip(mb, ma):
        assert rel_err(x, y) <= 1e-9
