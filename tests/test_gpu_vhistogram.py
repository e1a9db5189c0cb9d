"""On-device velocity histograms (VHistogramRecorder, Recorder/VHistogramRecorder.cc:222-306)
against the oracle's restatement on the same particles.

Both evaluate the recorder's arithmetic in the same rounded operations, so the particle total
is identical and a bin can differ only for a particle whose own state differs in its last bits
between the two runs after the steps taken: at most 2 particles' worth of bin mass in FP64, and
1 % of the particles for FP32 velocities, whose rounding moves bin edges.
"""
import os

import numpy as np
import pytest
from state_io import read_state

import hfemic_b200 as h

pytestmark = pytest.mark.gpu
GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


@pytest.mark.parametrize("name", ["p1_cic_periodic", "p2_tsc_mirror_reflecting"])
@pytest.mark.parametrize("precision", [h.configs.PREC_FP64, h.configs.PREC_MIXED])
def test_vhistogram_matches_oracle(gpu_lib, oracle_lib, name, precision):
    cfg = h.configs.PARITY[name]()
    init = read_state(os.path.join(GOLDEN, f"{name}.init.bin"))
    specs = dict(extent=(cfg.q1min + cfg.Nx / 8, cfg.Nx * 0.75), v1=(-6.0, 12.0, 24), v2=(0.0, 8.0, 16))
    steps = 1 if precision == h.configs.PREC_MIXED else 5
    with h.Run(cfg.replace(precision=precision), gpu_lib) as g, h.Run(cfg, oracle_lib, "orc_") as o:
        g.upload_state(init)
        o.upload_state(init)
        g.advance(steps)
        o.advance(steps)
        hg, tg = h.abi.vhistogram(g, 0, **specs)
        ho, to = h.abi.vhistogram(o, 0, prefix="orc_", **specs)
    assert tg == to and to > 0
    diff = np.abs(hg[..., 0] - ho[..., 0]).sum() * to
    limit = 2 if precision == h.configs.PREC_FP64 else 0.01 * to
    assert diff <= limit, diff
    assert ho[..., 0].sum() > 0.9  # the bins hold almost every particle of the extent
    np.testing.assert_allclose(hg[..., 2], hg[..., 0])  # full-f: real_f / marker = 1 per particle
