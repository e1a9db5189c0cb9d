"""Benchmark of the hybrid_1d hot path on B200: particle-steps/s of the plain FP64 GPU drop-in.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference] [--config NAME]

Workload (default): the FP64 drop-in configuration -- mirror field xi=0.002, Nx=2048, masking
over 128 cells at each end, reflecting particles, hot H+ and hot He+ with 1000 particles per
cell each (TSC, 4.1M particles), dt=0.01, CAM-CL with 10 B subcycles.  One bench step is one
CAM-CL cycle of every particle (push, two deposits, move, boundary, field cycle), cell sorts
included.  Synthetic seeded bi-Maxwellian particles; 197 MB of particle state per GPU, larger
than L2, so no flush is needed between steps.

Multi-GPU: every rank runs an independent replica of the workload (the path does not shard;
no collective is used); value = particle-steps of all ranks / max-over-ranks device time.

--impl reference times the reference's own CPU implementation of the same workload
(oracle/_ref, compiled from the reference sources) with one process per host core, each
holding 1/P of the particles (PartSpecies::populate(color, divisor)); rank 0 only.
"""
from __future__ import annotations

import argparse
import importlib.util
import json
import os
import statistics
import subprocess
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
PKG_DIR = os.path.join(ROOT, "hybrid_code-hfemic_wave_b200")


def _package():
    if "hfemic_b200" in sys.modules:
        return sys.modules["hfemic_b200"]
    spec = importlib.util.spec_from_file_location("hfemic_b200", os.path.join(PKG_DIR, "__init__.py"),
                                                  submodule_search_locations=[PKG_DIR])
    mod = importlib.util.module_from_spec(spec)
    sys.modules["hfemic_b200"] = mod
    spec.loader.exec_module(mod)
    return mod


METRIC = "particle-steps/s"
BYTES_PER_PARTICLE_STEP = 72  # FP64: read q1, vx, vy, vz, w (40 B), write q1, vx, vy, vz (32 B)


def measured_peak():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(path) as f:
            return float(json.load(f)["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


class ClockSampler:
    """nvidia-smi samples of SM clock and throttle reasons while the timed region runs."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
         "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
         "clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.proc = None
        self.lines = []

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.index}", f"--query-gpu={self.Q}",
                                          "--format=csv,noheader,nounits", "-lms", "100"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except Exception:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self):
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            f = [x.strip() for x in ln.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                mx = float(f[2])
            except ValueError:
                continue
            for n, v in zip(names, f[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(n)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(sm)}


def workload(h, name):
    table = {**h.configs.PRESETS, **h.configs.PARITY}
    return table[name]()


def cpu_baseline_reference(cfg, budget_s=20.0):
    """The reference binary (oracle/_ref) on one core for a bounded number of steps."""
    drv = os.path.join(ROOT, "oracle", "_ref", cfg.name, "ref_driver")
    if not os.path.exists(drv):
        return None
    steps = 2
    out = subprocess.run([drv, "bench", str(steps)], capture_output=True, text=True, timeout=600)
    r = json.loads(out.stdout.strip().splitlines()[-1])
    per_step = r["advance_s"] / steps
    steps = max(2, min(60, int(budget_s / max(per_step, 1e-6))))
    if steps > 2:
        out = subprocess.run([drv, "bench", str(steps)], capture_output=True, text=True, timeout=600)
        r = json.loads(out.stdout.strip().splitlines()[-1])
    return {"value": r["particle_steps_per_s"], "unit": METRIC, "cores": 1, "kind": "reference",
            "sample": f"{cfg.name}: {r['particles']} particles x {r['steps']} steps of Domain_CAMCL::advance_by "
                      f"({r['advance_s']:.1f} s, loader excluded), one core"}


def cpu_baseline_port(h, cfg, budget_s=15.0):
    """The C oracle on one core on a particle subsample, when the reference binary is absent."""
    from hfemic_b200.loader import initial_state

    frac = 1 / 16
    st = initial_state(cfg, seed=1, fraction=frac)
    lib = os.path.join(ROOT, "oracle", "liboracle.so")
    with h.Run(cfg, lib, "orc_") as r:
        r.upload_state(st)
        n = sum(p["q1"].size for p in st["particles"])
        t0 = time.perf_counter()
        steps = 0
        while time.perf_counter() - t0 < budget_s and steps < 200:
            r.advance(1)
            steps += 1
        dt = time.perf_counter() - t0
    return {"value": n * steps / dt, "unit": METRIC, "cores": 1, "kind": "port",
            "sample": f"{cfg.name} with 1/16 of the particles ({n}) x {steps} steps, one core"}


def run_reference_arm(args, h, rank):
    if rank != 0:
        return
    cfg = workload(h, args.config)
    drv = os.path.join(ROOT, "oracle", "_ref", cfg.name, "ref_driver")
    if not os.path.exists(drv):
        print(json.dumps({"impl": "reference", "unavailable": f"reference binary for {cfg.name} was not built"}))
        return
    P = max(1, min(os.cpu_count() or 1, 64))
    # each process holds 1/P of the particles; steps sized so the arm ends within minutes
    probe = subprocess.run([drv, "bench", "1", "0", str(P)], capture_output=True, text=True, timeout=900)
    r0 = json.loads(probe.stdout.strip().splitlines()[-1])
    per_step = max(r0["advance_s"], 1e-4)
    steps = max(1, min(args.steps + args.warmup, int(60.0 / per_step)))
    procs = [subprocess.Popen([drv, "bench", str(steps), str(c), str(P)], stdout=subprocess.PIPE, text=True)
             for c in range(P)]
    outs = [json.loads(p.communicate(timeout=1800)[0].strip().splitlines()[-1]) for p in procs]
    total = sum(o["particles"] for o in outs) * steps
    wall = max(o["advance_s"] for o in outs)
    value = total / wall
    line = {"impl": "reference", "metric": METRIC, "value": value, "unit": METRIC, "n_gpus": args.gpus,
            "steps": steps, "warmup": 0, "ms_per_step": 1e3 * wall / steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic (reference loader)",
            "config": {"workload": cfg.name, "Nx": cfg.Nx, "particles": sum(o["particles"] for o in outs),
                       "note": f"{P} independent processes x 1/{P} of the particles, no moment all-reduce "
                               "(upper bound of the reference's particle decomposition)"},
            "cpu_baseline": {"value": value, "unit": METRIC, "cores": P, "kind": "reference",
                             "sample": f"{steps} steps of Domain_CAMCL::advance_by on {P} processes"},
            "e2e": {"value": value, "unit": METRIC, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line))


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=300)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--config", default="config2_tsc_mirror_nx2048")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-e2e", action="store_true")
    args = ap.parse_args()
    assert args.warmup >= 3 or args.impl == "reference", "at least 3 warm-up steps"

    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    h = _package()
    if args.impl == "reference":
        run_reference_arm(args, h, rank)
        return

    import ctypes

    import numpy as np
    import torch
    import torch.distributed as dist

    torch.cuda.set_device(local)
    if world > 1:
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=120), device_id=torch.device("cuda", local))
    cfg = workload(h, args.config)
    from hfemic_b200.loader import initial_state

    st = initial_state(cfg, seed=1000 + rank)
    n_particles = sum(p["q1"].size for p in st["particles"])

    run = h.open_run(cfg)
    lib = run.lib
    lib.h1d_advance_async.argtypes = [ctypes.c_void_p, ctypes.c_uint32]
    lib.h1d_synchronize.argtypes = [ctypes.c_void_p]
    lib.h1d_get_stream.argtypes = [ctypes.c_void_p, ctypes.POINTER(ctypes.c_void_p)]
    lib.h1d_profile_enable.argtypes = [ctypes.c_void_p, ctypes.c_int]
    lib.h1d_profile_read.argtypes = [ctypes.c_void_p, ctypes.POINTER(h.abi.Profile)]
    run.upload_state(st)
    sp = ctypes.c_void_p()
    run._check(lib.h1d_get_stream(run.h, ctypes.byref(sp)))
    stream = torch.cuda.ExternalStream(sp.value)

    # warm-up
    run._check(lib.h1d_advance_async(run.h, args.warmup))
    run._check(lib.h1d_synchronize(run.h))

    # timed region: K steps, events on the run's stream, profiling events around each kernel group
    run._check(lib.h1d_profile_enable(run.h, 1))
    start, end = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize()
    with ClockSampler(local) as clk:
        start.record(stream)
        run._check(lib.h1d_advance_async(run.h, args.steps))
        end.record(stream)
        run._check(lib.h1d_synchronize(run.h))
        torch.cuda.synchronize()
    ms = start.elapsed_time(end)
    prof = h.abi.Profile()
    run._check(lib.h1d_profile_read(run.h, ctypes.byref(prof)))
    run._check(lib.h1d_profile_enable(run.h, 0))
    if world > 1:
        t = torch.tensor([ms], device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        ms = float(t.item())
        dist.barrier()
    value = n_particles * args.steps * world / (ms / 1e3)

    # roofline of the dominant kernel (fused push/deposit): algorithmic bytes per launch / avg launch time
    peak, peak_kind = measured_peak()
    push_avg_ms = prof.push_ms / max(prof.push_launches, 1)
    bytes_per_launch = BYTES_PER_PARTICLE_STEP * prof.particles_pushed / max(prof.push_launches, 1)
    achieved = bytes_per_launch / (push_avg_ms / 1e3) / 1e9
    roofline = {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                "traffic": None, "kernel": "push_kernel (fused push + 2 deposits + move + BC, FP64)",
                "peak_kind": peak_kind,
                "bytes_per_launch": bytes_per_launch,
                "window_miss_rate": prof.window_misses / max(2 * prof.particles_pushed, 1),
                "phase_ms_per_step": {"push": prof.push_ms / args.steps, "sort": prof.sort_ms / args.steps,
                                      "field": prof.field_ms / args.steps}}
    traffic_path = os.path.join(ROOT, "profiles", "push_kernel_traffic.json")
    if os.path.exists(traffic_path):
        try:
            with open(traffic_path) as f:
                tr = json.load(f)
            roofline["traffic"] = tr["bytes_per_particle"] * bytes_per_launch / BYTES_PER_PARTICLE_STEP
        except Exception:
            pass

    # e2e through the C-ABI with host buffers: upload from pinned memory, inner_Nt-step chunks
    # with the recorder downloads (fields, sources, moments) after each, particles back at the end
    e2e = None
    if not args.no_e2e:
        K = args.steps
        inner = cfg.inner_Nt
        pinned = []
        for p in st["particles"]:
            d = {}
            for key in ("q1", "vx", "vy", "vz", "w"):
                t = torch.empty(p[key].size, dtype=torch.float64, pin_memory=True)
                t.numpy()[:] = p[key]
                d[key] = t.numpy()
            pinned.append(d)
        M = cfg.Nx + 6
        bufB = torch.empty((M, 3), dtype=torch.float64, pin_memory=True).numpy()
        bufE = torch.empty((M, 3), dtype=torch.float64, pin_memory=True).numpy()
        outs = [{k: torch.empty(p["q1"].size, dtype=torch.float64, pin_memory=True).numpy()
                 for k in ("q1", "vx", "vy", "vz", "w")} for p in st["particles"]]
        with h.open_run(cfg) as r2:
            if world > 1:
                dist.barrier()
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            for s, d in enumerate(pinned):
                r2.upload_particles(s, d["q1"], d["vx"], d["vy"], d["vz"], d["w"])
            r2.upload_fields(st["B"], st["E"])
            for i, c in enumerate(st["cold"]):
                r2.upload_cold(i, c["n_full"], c["nV_full"])
            done = 0
            d2h = 0
            while done < K:
                k = min(inner, K - done)
                r2.advance(k)
                done += k
                run_B, run_E = r2.fields()
                rho, J = r2.sources()
                d2h += (run_B.nbytes + run_E.nbytes + rho.nbytes + J.nbytes)
                for s in range(len(cfg.kinetic)):
                    m = r2.moments(s)
                    d2h += sum(a.nbytes for a in m)
            for s in range(len(cfg.kinetic)):
                p = r2.particles(s)
                d2h += sum(p[k].nbytes for k in ("q1", "vx", "vy", "vz", "w"))
            torch.cuda.synchronize()
            e2e_s = time.perf_counter() - t0
        if world > 1:
            t = torch.tensor([e2e_s], device="cuda")
            dist.all_reduce(t, op=dist.ReduceOp.MAX)
            e2e_s = float(t.item())
        h2d = sum(p["q1"].nbytes * 5 for p in st["particles"]) + st["B"].nbytes + st["E"].nbytes
        e2e = {"value": n_particles * K * world / e2e_s, "unit": METRIC, "h2d_bytes_per_step": h2d / K,
               "d2h_bytes_per_step": d2h / K,
               "note": f"upload, {K} steps as advance_by({inner}) chunks with field/source/moment downloads "
                       "after each chunk, particle download at the end"}

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        cpu = cpu_baseline_reference(cfg) or cpu_baseline_port(h, cfg)

    run.close()
    if world > 1:
        dist.destroy_process_group()
    if rank != 0:
        return
    line = {
        "metric": METRIC, "value": value, "unit": METRIC, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms / args.steps, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded bi-Maxwellian loader)",
        "config": {"workload": cfg.name, "Nx": cfg.Nx, "particles_per_gpu": n_particles,
                   "species": len(cfg.kinetic), "ppc": [k.Nc for k in cfg.kinetic],
                   "shape_order": [k.shape_order for k in cfg.kinetic], "xi": cfg.xi,
                   "algorithm": "CAM-CL", "n_subcycles": cfg.n_subcycles, "precision": "fp64",
                   "l2": "particle state (197 MB per GPU) larger than L2; no flush",
                   "parallelism": f"replicas x{world}"},
        "roofline": roofline, "cpu_baseline": cpu, "e2e": e2e, "clocks": clk.summary(),
        "gpu_launches": int(prof.kernel_launches),
    }
    print(json.dumps(line))


if __name__ == "__main__":
    main()
