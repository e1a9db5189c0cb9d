"""A CUDA checkpoint resumed by the reference itself.

The reference restarts from a snapshot (Recorder/Snapshot.cc:330-375, Driver.cc:90-100): the
particles with their ids, B, E and the cold fluid's full moments come back, and the next
advance_by recomputes the sources.  Its hot path compiled from its sources
(oracle/_ref/<name>/ref_driver) restarts the same way from a state file (`run` mode).

Here a CUDA run advances 6 steps from the golden initial state and saves a checkpoint
(h1d_checkpoint_save); a fresh run restores it (h1d_checkpoint_load) and exports what it holds
as a state file: fields, particles in upload order with the reference's ids, phase-space
densities, and cold moments.  The reference binary advances that file by 1 and by 10 steps; the
restored CUDA run advances by the same steps.  Bars: FP64 within 1e-12 after one step with every
particle's cell index identical, and within 1e-9 after ten; mixed precision within 1e-4 in the
grid quantities.
"""
import os
import subprocess
import tempfile

import numpy as np
import pytest
from parity_util import attach_pid, cell_mismatches, state_errors
from state_io import read_state, write_state

import hfemic_b200 as h

pytestmark = pytest.mark.gpu
ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
GOLDEN = os.path.join(ROOT, "tests", "golden")


def _export(run, cfg, init, step):
    """The run's state in the reference's state-file layout, particles in upload order."""
    st = run.state()
    out = dict(Nx=init["Nx"], pad=init["pad"], step=step, moment_norm=init["moment_norm"],
               B=st["B"], E=st["E"], charge=st["charge"], current=st["current"], particles=[],
               moments=st["moments"], cold=st["cold"])
    for s, p in enumerate(st["particles"]):
        order = np.argsort(p["pid"], kind="stable")
        pid = np.asarray(p["pid"])[order]
        assert np.array_equal(pid, np.arange(pid.size))  # no particle was lost
        q = {k: np.asarray(p[k])[order] for k in ("q1", "vx", "vy", "vz", "w")}
        q["id"] = np.asarray(init["particles"][s]["id"])[pid]
        if cfg.kinetic[s].has_psd:  # evolving weights: the run's own real_f / marker
            q["real_f"], q["marker"] = np.asarray(p["real_f"])[order], np.asarray(p["marker"])[order]
        else:  # fixed weights: the phase-space density the particles were loaded with
            q["real_f"] = np.asarray(init["particles"][s]["real_f"])[pid]
            q["marker"] = np.asarray(init["particles"][s]["marker"])[pid]
        out["particles"].append(q)
    return out


@pytest.mark.parametrize("name, precision", [
    ("p1_cic_periodic", h.configs.PREC_FP64),
    ("p2_tsc_mirror_reflecting", h.configs.PREC_FP64),
    ("p4_pc_tsc_mirror_reflecting", h.configs.PREC_FP64),
    ("p7_psd_tsc_mirror_reflecting", h.configs.PREC_FP64),
    ("p2_tsc_mirror_reflecting", h.configs.PREC_MIXED),
])
def test_reference_resumes_a_cuda_checkpoint(gpu_lib, name, precision):
    drv = os.path.join(ROOT, "oracle", "_ref", name, "ref_driver")
    if not os.path.exists(drv):
        pytest.fail(f"{drv} is not built (make -C oracle ref REF=<reference tree>)")
    cfg = h.configs.PARITY[name]().replace(precision=precision)
    init = read_state(os.path.join(GOLDEN, f"{name}.init.bin"))
    with h.Run(cfg, gpu_lib) as a:
        a.upload_state(init)
        a.advance(6)
        image = h.abi.checkpoint(a)
    with tempfile.TemporaryDirectory() as tmp, h.Run(cfg, gpu_lib) as b:
        h.abi.restore(b, image)
        assert h.abi.step_count(b) == 6
        path = os.path.join(tmp, "resume.bin")
        write_state(path, _export(b, cfg, init, 6))
        for steps in (1, 10):
            subprocess.run([drv, "run", path, str(steps), "1", os.path.join(tmp, f"r{steps}_")], check=True,
                           timeout=600, capture_output=True)
        refs = {s: attach_pid(read_state(os.path.join(tmp, f"r{s}_1.bin")), init) for s in (1, 10)}
        done = 0
        for steps, tol in ((1, 1e-12), (10, 1e-9)):
            b.advance(steps - done)
            done = steps
            st = b.state()
            errs = state_errors(st, refs[steps], cfg)
            if precision == h.configs.PREC_MIXED:
                errs = {k: v for k, v in errs.items() if "particles" not in k}
                tol = 1e-4
            inner = max(state_errors(st, refs[steps], cfg, interior_only=True).values())
            print(name, "mixed" if precision else "fp64", steps, f"max {max(errs.values()):.2e}",
                  f"(interior cells {inner:.2e})")
            bad = {k: v for k, v in errs.items() if not v <= tol}
            assert not bad, (steps, bad)
            if precision == h.configs.PREC_FP64 and steps == 1:
                assert all(d < 1e-12 for _, _, d in cell_mismatches(st, refs[steps], cfg))
