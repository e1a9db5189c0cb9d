"""Checkpoint / resume of device state (h1d_checkpoint_*), the reference's snapshot content.

A run saved after some steps and resumed in a fresh run continues as the original does: FP64
within 1e-12 (max-norm relative; the resumed run re-sorts its particles, which changes only the
order of deposit sums), mixed precision within 1e-5.  The grid arrays are compared on the
interior: a predictor-corrector run refreshes the ghost cells of the cold fluid's full moments
when it starts, from a checkpoint too, as the reference's Domain_PC::advance_by does after a
snapshot load (Domain_PC.cc:46), while the uninterrupted run keeps the ghosts it started with;
nothing reads those ghosts.  A save of a resumed run reproduces the
image byte for byte, and a checkpoint of other parameters is refused ("signature verification
failed", Recorder/Snapshot.cc:340-342).
"""
import os

import pytest
from parity_util import state_errors
from state_io import read_state

import hfemic_b200 as h

pytestmark = pytest.mark.gpu
GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


@pytest.mark.parametrize("name,precision,tol", [
    ("p2_tsc_mirror_reflecting", h.configs.PREC_FP64, 1e-12),
    ("p4_pc_tsc_mirror_reflecting", h.configs.PREC_FP64, 1e-12),
    ("p3_o3_adiabatic_periodic", h.configs.PREC_FP64, 1e-12),
    ("p2_tsc_mirror_reflecting", h.configs.PREC_MIXED, 1e-5),
])
def test_resume_continues_the_run(gpu_lib, name, precision, tol):
    cfg = h.configs.PARITY[name]().replace(precision=precision)
    init = read_state(os.path.join(GOLDEN, f"{name}.init.bin"))
    with h.Run(cfg, gpu_lib) as a:
        a.upload_state(init)
        a.advance(6)
        image = h.abi.checkpoint(a)
        a.advance(6)
        sa = a.state()
        assert h.abi.step_count(a) == 12
    with h.Run(cfg, gpu_lib) as b:
        h.abi.restore(b, image)
        assert h.abi.step_count(b) == 6
        b.advance(6)
        sb = b.state()
    errs = state_errors(sb, sa, cfg, interior_only=True)
    print(name, precision, {k: f"{v:.1e}" for k, v in errs.items()})
    assert max(errs.values()) <= tol, errs


def test_image_round_trip_is_exact(gpu_lib):
    cfg = h.configs.parity_p2().replace(precision=h.configs.PREC_MIXED)
    init = read_state(os.path.join(GOLDEN, f"{cfg.name}.init.bin"))
    with h.Run(cfg, gpu_lib) as a:
        a.upload_state(init)
        a.advance(3)
        image = h.abi.checkpoint(a)
    with h.Run(cfg, gpu_lib) as b:
        h.abi.restore(b, image)
        assert h.abi.checkpoint(b) == image


def test_signature_mismatch_is_refused(gpu_lib):
    cfg = h.configs.parity_p1()
    init = read_state(os.path.join(GOLDEN, f"{cfg.name}.init.bin"))
    with h.Run(cfg, gpu_lib) as a:
        a.upload_state(init)
        image = h.abi.checkpoint(a)
    with h.Run(cfg.replace(dt=cfg.dt * 0.5), gpu_lib) as b:
        with pytest.raises(ValueError, match="signature"):
            h.abi.restore(b, image)
        with pytest.raises(ValueError):
            h.abi.restore(b, image[:100])
