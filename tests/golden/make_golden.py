"""Regenerate the golden state fixtures from the reference itself.

Builds the reference hot path (oracle/Makefile ``ref`` target: the unmodified
src/hybrid_1d/Core and src/LibPIC sources of kyungguk1/hybrid_code-hfemic_wave compiled in
place, one binary per configuration) and, for every parity configuration, writes
    <name>.init.bin    particles from the reference's own loader (PartSpecies::populate with
                       the species' VDF: Maxwellian, loss-cone, partial shell or counter-beam)
                       and the initial fields
    <name>.step1.bin   after Domain::advance_by(1)
    <name>.step10.bin  after Domain::advance_by(10) from the same initial state
into tests/golden/.  Needs the reference tree, given as the argument or as $H1D_REFERENCE.

usage: python tests/golden/make_golden.py [<reference tree>]
"""
import os
import shutil
import subprocess
import sys
import tempfile

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
NAMES = ["p1_cic_periodic", "p2_tsc_mirror_reflecting", "p3_o3_adiabatic_periodic",
         "p4_pc_tsc_mirror_reflecting", "p5_tsc_mirror_source", "p6_pc_source", "p7_psd_tsc_mirror_reflecting",
         "p8_pc_psd_periodic", "p9_losscone_psd_mirror", "p10_pc_shell_psd_mirror", "p11_counterbeam_psd_mirror"]


def main():
    ref = sys.argv[1] if len(sys.argv) > 1 else os.environ.get("H1D_REFERENCE")
    if not ref or not os.path.isdir(ref):
        sys.exit("make_golden.py: give the reference tree as the argument or as $H1D_REFERENCE")
    subprocess.check_call(["make", "-C", os.path.join(ROOT, "oracle"), "ref", f"REF={ref}",
                           f"PYTHON={sys.executable}", "-j8"])
    with tempfile.TemporaryDirectory() as tmp:
        for name in NAMES:
            drv = os.path.join(ROOT, "oracle", "_ref", name, "ref_driver")
            init = os.path.join(HERE, f"{name}.init.bin")
            subprocess.check_call([drv, "init", init])
            subprocess.check_call([drv, "run", init, "1", "1", os.path.join(tmp, "a")])
            shutil.copy(os.path.join(tmp, "a1.bin"), os.path.join(HERE, f"{name}.step1.bin"))
            subprocess.check_call([drv, "run", init, "10", "1", os.path.join(tmp, "b")])
            shutil.copy(os.path.join(tmp, "b1.bin"), os.path.join(HERE, f"{name}.step10.bin"))
            print("wrote", name)


if __name__ == "__main__":
    main()
