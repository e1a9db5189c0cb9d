"""The drop-in GPU Domain (hybrid_code-hfemic_wave_b200/adapter/Domain_GPU.h) inside the reference.

oracle/_ref/<config>/ref_driver_gpu is the reference's own hot path compiled from its sources, with
Domain_CAMCL_GPU / Domain_PC_GPU constructed in place of Domain_CAMCL / Domain_PC (oracle/Makefile
target `gpu`).  From the same initial state (the reference loader's particles, committed as
tests/golden/<name>.init.bin) it runs advance_by on the GPU and writes what the reference's
recorders would read -- bfield, efield, charge, current, every species' moment<0..2>() and the cold
fluid, downloaded by the adapter into the reference's own GridArrays -- and the particles it copied
back into PartSpecies::bucket.  These are compared with the reference's CPU Domain after the same
steps (the golden fixtures <name>.step1.bin / .step10.bin, written by the same driver without the
GPU Domain), at the parity bars of the other FP64 tests: 1e-12 (max-norm relative) after one step
with every particle's cell index identical, 1e-9 after ten steps taken as two advance_by(5) calls.
The mixed-precision Domain is held to 1e-4.  A particle that moves too far surfaces as the
reference's std::domain_error.
"""
import os
import subprocess
import tempfile

import pytest
from parity_util import attach_pid, cell_mismatches, state_errors
from state_io import read_state, write_state

import hfemic_b200 as h

pytestmark = pytest.mark.gpu
ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
GOLDEN = os.path.join(ROOT, "tests", "golden")
NAMES = sorted(h.configs.PARITY)


def _driver(name):
    path = os.path.join(ROOT, "oracle", "_ref", name, "ref_driver_gpu")
    if not os.path.exists(path):
        pytest.fail(f"{path} is not built (make -C oracle gpu REF=<reference tree>)")
    return path


def _gpu_run(name, init_path, steps, chunks, precision="fp64"):
    with tempfile.TemporaryDirectory() as tmp:
        prefix = os.path.join(tmp, "g")
        out = subprocess.run([_driver(name), "gpu_run", init_path, str(steps), str(chunks), prefix, precision],
                             capture_output=True, text=True, timeout=600)
        assert out.returncode == 0, out.stderr
        return read_state(f"{prefix}{chunks}.bin")


@pytest.mark.parametrize("name", NAMES)
def test_adapter_one_and_ten_steps(name):
    cfg = h.configs.PARITY[name]()
    init_path = os.path.join(GOLDEN, f"{name}.init.bin")
    init = read_state(init_path)
    for steps, chunks, fixture, tol in ((1, 1, "step1", 1e-12), (5, 2, "step10", 1e-9)):
        ref = attach_pid(read_state(os.path.join(GOLDEN, f"{name}.{fixture}.bin")), init)
        gpu = attach_pid(_gpu_run(name, init_path, steps, chunks), init)
        assert gpu["step"] == ref["step"] == steps * chunks
        errs = state_errors(gpu, ref, cfg)
        print(name, fixture, {k: f"{v:.2e}" for k, v in errs.items()})
        bad = {k: v for k, v in errs.items() if not v <= tol}
        assert not bad, bad
        assert not [m for m in cell_mismatches(gpu, ref, cfg) if m[2] >= tol]


@pytest.mark.parametrize("name", ["p2_tsc_mirror_reflecting", "p4_pc_tsc_mirror_reflecting"])
def test_adapter_mixed_precision(name):
    cfg = h.configs.PARITY[name]()
    init_path = os.path.join(GOLDEN, f"{name}.init.bin")
    init = read_state(init_path)
    ref = attach_pid(read_state(os.path.join(GOLDEN, f"{name}.step10.bin")), init)
    gpu = attach_pid(_gpu_run(name, init_path, 10, 1, "mixed"), init)
    errs = {k: v for k, v in state_errors(gpu, ref, cfg).items() if "particles" not in k}
    print(name, "mixed", {k: f"{v:.2e}" for k, v in errs.items()})
    assert max(errs.values()) <= 1e-4, errs


def test_adapter_moved_too_far_is_the_references_domain_error():
    name = "p1_cic_periodic"
    cfg = h.configs.PARITY[name]()
    st = read_state(os.path.join(GOLDEN, f"{name}.init.bin"))
    st["particles"][0]["vx"][7] = 2.0 * cfg.Dx / cfg.dt  # two cells in one step
    with tempfile.TemporaryDirectory() as tmp:
        path = os.path.join(tmp, "bad.bin")
        write_state(path, st)
        cpu = subprocess.run([os.path.join(ROOT, "oracle", "_ref", name, "ref_driver"), "run", path, "1", "1",
                              os.path.join(tmp, "c")], capture_output=True, text=True, timeout=600)
        gpu = subprocess.run([_driver(name), "gpu_run", path, "1", "1", os.path.join(tmp, "g"), "fp64"],
                             capture_output=True, text=True, timeout=600)
    for out in (cpu, gpu):
        assert out.returncode == 1 and "std::domain_error" in out.stderr and "moved too far" in out.stderr, out.stderr
