"""Benchmark of the hybrid_1d hot path on B200: particle-steps/s, mixed precision against plain FP64.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference] [--config NAME]
                    [--precision auto|fp64|mixed]

Workload (default): the config-1 plasma at Nx=4096 with 4000 particles per cell -- uniform B0,
periodic, one kinetic H+ species (beta_par 0.1, T_perp/T_par 3, CIC; 16.4M particles) plus a
cold H+ background, isothermal electrons, dt=0.02, CAM-CL with 10 B subcycles -- run with the
mixed-precision particle pass (int32 fixed-point position, FP32 velocity / interpolation / push,
FP32 warp deposits summed into FP64 cells; FP64 field cycle).  One bench step is one CAM-CL
cycle of every particle (push, two deposits, move, boundary, field cycle), cell sorts included.
Beside it the same workload in plain FP64 (`fp64`), the mixed run's error against FP64 after
100 steps from the same state (`error_vs_fp64`, wave energy, particle energy and moments), and
the FP64 drop-in configuration (mirror field, Nx=2048, two TSC species, 4.1M particles,
`drop_in_fp64`).  Synthetic seeded bi-Maxwellian particles; the particle state (393 MB mixed,
722 MB FP64) is larger than L2, so no flush is needed between steps.

Multi-GPU: every rank runs an independent replica of the workload (the path does not shard;
no collective is used); value = particle-steps of all ranks / max-over-ranks device time.

--impl reference times the reference's own CPU implementation of the same workload
(oracle/_ref, compiled from the reference sources, FP64) with one process per host core, each
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
# algorithmic HBM bytes per particle-step of the particle pass
BYTES_PER_PARTICLE_STEP = {
    "fp64": 72,   # read q1, vx, vy, vz, w (40 B), write q1, vx, vy, vz (32 B)
    "mixed": 36,  # read position (int32 fixed point), vx, vy, vz, w (20 B), write position, vx, vy, vz (16 B)
}
STATE_BYTES = {"fp64": 44, "mixed": 24}  # stored bytes per particle, id included
KERNEL = {"fp64": "push_kernel (fused push + 2 deposits + move + BC, FP64)",
          "mixed": "push_kernel_mixed (fused push + 2 deposits + move + BC, FP32 with int32 fixed-point position)"}


def measured_peak():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(path) as f:
            return float(json.load(f)["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


class ClockSampler:
    """SM clock and clock-event reasons while the timed region runs, read (never set) through NVML:
    one sample when the region opens, samples about every millisecond while it runs, and one when
    it closes, so that even a region of a few milliseconds carries its own clock record.  Falls
    back to an nvidia-smi polling loop when NVML cannot be loaded."""

    REASONS = (("hw_slowdown", "nvmlClocksEventReasonHwSlowdown"),
               ("hw_thermal_slowdown", "nvmlClocksEventReasonHwThermalSlowdown"),
               ("sw_thermal_slowdown", "nvmlClocksEventReasonSwThermalSlowdown"),
               ("sw_power_cap", "nvmlClocksEventReasonSwPowerCap"))
    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
         "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
         "clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.samples = []  # (sm_mhz, max_mhz, reasons)
        self.nvml = None
        self.proc = None
        self.stop = threading.Event()
        self.thread = None

    def _sample_nvml(self):
        nv = self.nvml
        sm = nv.nvmlDeviceGetClockInfo(self.handle, nv.NVML_CLOCK_SM)
        mask = nv.nvmlDeviceGetCurrentClocksEventReasons(self.handle)
        reasons = [name for name, const in self.REASONS if mask & getattr(nv, const)]
        self.samples.append((float(sm), self.max_mhz, reasons))

    def _loop_nvml(self):
        while not self.stop.wait(0.001):
            try:
                self._sample_nvml()
            except Exception:
                return

    def _loop_smi(self):
        for line in self.proc.stdout:
            f = [x.strip() for x in line.split(",")]
            try:
                reasons = [n for n, v in zip([r[0] for r in self.REASONS], f[5:9]) if v.lower().startswith("active")]
                self.samples.append((float(f[1]), float(f[2]), reasons))
            except (ValueError, IndexError):
                continue

    def __enter__(self):
        try:
            import pynvml

            pynvml.nvmlInit()
            self.nvml = pynvml
            self.handle = pynvml.nvmlDeviceGetHandleByIndex(self.index)
            self.max_mhz = float(pynvml.nvmlDeviceGetMaxClockInfo(self.handle, pynvml.NVML_CLOCK_SM))
            self._sample_nvml()
            self.thread = threading.Thread(target=self._loop_nvml, daemon=True)
            self.thread.start()
        except Exception:
            self.nvml = None
            try:
                self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.index}", f"--query-gpu={self.Q}",
                                              "--format=csv,noheader,nounits", "-lms", "50"],
                                             stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
                self.thread = threading.Thread(target=self._loop_smi, daemon=True)
                self.thread.start()
            except Exception:
                self.proc = None
        return self

    def __exit__(self, *a):
        self.stop.set()
        if self.nvml is not None:
            if self.thread:
                self.thread.join(timeout=1)
            try:
                self._sample_nvml()
                self.nvml.nvmlShutdown()
            except Exception:
                pass
        elif self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self):
        sm = [s[0] for s in self.samples]
        reasons = sorted({r for s in self.samples for r in s[2]})
        return {"sm_mhz": statistics.median(sm) if sm else None,
                "sm_max_mhz": self.samples[-1][1] if self.samples else None, "reasons": reasons,
                "samples": len(sm), "source": "nvml" if self.nvml is not None else "nvidia-smi"}


def workload(h, name):
    table = {**h.configs.PRESETS, **h.configs.PARITY}
    return table[name]()


def cpu_baseline_reference(cfg, budget_s=20.0):
    """The reference binary (oracle/_ref) on one core for a bounded number of steps, holding
    1/divisor of the particles (PartSpecies::populate(0, divisor)) so that loading stays short."""
    drv = os.path.join(ROOT, "oracle", "_ref", cfg.name, "ref_driver")
    if not os.path.exists(drv):
        return None
    div = max(1, cfg.n_particles // 1_000_000)
    args = [] if div == 1 else ["0", str(div)]
    steps = 2
    out = subprocess.run([drv, "bench", str(steps), *args], capture_output=True, text=True, timeout=600)
    r = json.loads(out.stdout.strip().splitlines()[-1])
    per_step = r["advance_s"] / steps
    steps = max(2, min(200, int(budget_s / max(per_step, 1e-6))))
    if steps > 2:
        out = subprocess.run([drv, "bench", str(steps), *args], capture_output=True, text=True, timeout=600)
        r = json.loads(out.stdout.strip().splitlines()[-1])
    return {"value": r["particle_steps_per_s"], "unit": METRIC, "cores": 1, "kind": "reference",
            "sample": f"{cfg.name} with 1/{div} of the particles: {r['particles']} particles x {r['steps']} steps of "
                      f"Domain_CAMCL::advance_by ({r['advance_s']:.1f} s, loader excluded), one core, FP64"}


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


def _cpu_member_rate(job):
    """Worker: particle-steps/s of the C oracle (the reference's step restated in C, pinned bit for
    bit to the reference build; one core) on a bounded sample of one run of the ensemble
    distribution -- at most `target` of its particles, a few steps -- and its full particle count."""
    seed, target = job
    h = _package()
    from hfemic_b200.loader import initial_state

    cfg = h.configs.ensemble_member(seed, precision=h.configs.PREC_FP64)
    full = cfg.n_particles
    st = initial_state(cfg, seed=seed, fraction=min(1.0, target / full))
    n = sum(p["q1"].size for p in st["particles"])
    with h.Run(cfg, os.path.join(ROOT, "oracle", "liboracle.so"), "orc_") as r:
        r.upload_state(st)
        r.advance(1)
        k = max(2, int(2e6 / max(n, 1)))
        t0 = time.perf_counter()
        r.advance(k)
        dt = time.perf_counter() - t0
    return full, n * k / dt, n, k


def cpu_ensemble_serving_baselines(h, members=64, steps=500, n_requests=48, rate=4.0, seed=2024, target=100_000):
    """CPU baselines of the ensemble and the serving workloads on all host cores (P processes).
    Every run's CPU rate is measured on a bounded sample (<= `target` particles, a few steps, one
    core each, C oracle); the ensemble's time is the makespan of its runs' full work
    (particles x steps / rate) on P cores (longest first onto the least loaded core), and the
    serving stream -- the same seeded Poisson arrivals and step counts as serving_measure -- is
    replayed on a P-core first-come-first-served pool with those service times."""
    import heapq
    import multiprocessing as mp

    import numpy as np

    P = max(1, os.cpu_count() or 1)
    ens_seeds = list(range(members))
    srv_seeds = [1000 + i for i in range(n_requests)]
    t0 = time.perf_counter()
    with mp.get_context("spawn").Pool(min(P, len(ens_seeds) + len(srv_seeds))) as pool:
        res = pool.map(_cpu_member_rate, [(sd, target) for sd in ens_seeds + srv_seeds], chunksize=1)
    wall = time.perf_counter() - t0
    ens, srv = res[:members], res[members:]
    work = sorted((full * steps / r for full, r, _, _ in ens), reverse=True)
    loads = [0.0] * P
    for w in work:
        i = loads.index(min(loads))
        loads[i] += w
    makespan = max(loads)
    sample = (f"each run on <= {target} of its particles for a few steps (C oracle, one core per run), "
              f"scaled to its full particles x steps; {P} host cores; sampling took {wall:.1f} s")
    ens_line = {"runs_per_s": members / makespan, "value": sum(f for f, _, _, _ in ens) * steps / makespan,
                "unit": METRIC, "cores": P, "kind": "port", "makespan_s": makespan,
                "sample": f"{members} runs x {steps} steps scheduled longest-first on {P} cores; " + sample}
    rng = np.random.default_rng(seed)
    arrivals = np.cumsum(rng.exponential(1.0 / rate, n_requests))
    req_steps = rng.integers(200, 2001, n_requests)
    free = [0.0] * P
    heapq.heapify(free)
    lat, done = [], []
    for a, (full, r, _, _), k in zip(arrivals, srv, req_steps):
        start = max(a, heapq.heappop(free))
        end = start + full * int(k) / r
        heapq.heappush(free, end)
        lat.append(end - a)
        done.append(end)
    lat = np.array(lat)
    srv_line = {"runs_per_s": n_requests / (max(done) - arrivals[0]), "p50_s": float(np.percentile(lat, 50)),
                "p99_s": float(np.percentile(lat, 99)), "mean_s": float(lat.mean()), "cores": P, "kind": "port",
                "sample": f"the serving stream (Poisson, mean {rate}/s, {n_requests} requests, steps U[200, 2000], "
                          f"seed {seed}) replayed first-come-first-served on {P} cores with service times "
                          "particles x steps / rate; " + sample}
    return ens_line, srv_line


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


def reduce_over_ranks(seconds, units, device="cuda"):
    """Whole-job figures of a replicated measurement: the time is the max over ranks and the
    work the sum over ranks (torch.distributed, any backend; the identity on one process)."""
    import torch
    import torch.distributed as dist

    if not (dist.is_available() and dist.is_initialized()) or dist.get_world_size() == 1:
        return float(seconds), float(units)
    t = torch.tensor([float(seconds)], dtype=torch.float64, device=device)
    u = torch.tensor([float(units)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    dist.all_reduce(u, op=dist.ReduceOp.SUM)
    return float(t.item()), float(u.item())


def precision_name(cfg, h):
    return "mixed" if cfg.precision == h.configs.PREC_MIXED else "fp64"


class TimedRun:
    """A run behind the C-ABI with its stream, for device-timed advances."""

    def __init__(self, h, cfg, st, populate_seed=None):
        """From the host state `st`, or (st None) from the device loader with `populate_seed`."""
        import ctypes

        import torch

        self.h, self.cfg = h, cfg
        self.run = h.open_run(cfg)
        lib = self.lib = self.run.lib
        lib.h1d_advance_async.argtypes = [ctypes.c_void_p, ctypes.c_uint32]
        lib.h1d_synchronize.argtypes = [ctypes.c_void_p]
        lib.h1d_get_stream.argtypes = [ctypes.c_void_p, ctypes.POINTER(ctypes.c_void_p)]
        lib.h1d_profile_enable.argtypes = [ctypes.c_void_p, ctypes.c_int]
        lib.h1d_profile_read.argtypes = [ctypes.c_void_p, ctypes.POINTER(h.abi.Profile)]
        if st is None:
            h.abi.populate_state(self.run, populate_seed)
        else:
            self.run.upload_state(st)
        sp = ctypes.c_void_p()
        self.run._check(lib.h1d_get_stream(self.run.h, ctypes.byref(sp)))
        self.stream = torch.cuda.ExternalStream(sp.value)
        self.n_particles = cfg.n_particles if st is None else sum(p["q1"].size for p in st["particles"])

    def advance(self, n):
        self.run._check(self.lib.h1d_advance_async(self.run.h, n))
        self.run._check(self.lib.h1d_synchronize(self.run.h))

    def warm(self, n, autotune=True):
        """n plain warm-up steps, then (CAM-CL runs) the library's autotuner, which advances the run
        by real steps while it picks the sort interval and CTA count kept for the timed steps."""
        self.advance(n)
        self.tuned = None
        if autotune and self.cfg.algorithm == self.h.configs.ALGO_CAMCL:
            steps, k, c = self.h.abi.autotune(self.run)
            self.tuned = {"steps": steps, "sort_interval": k, "ctas_per_sm": c}
        return self.tuned

    def timed(self, steps, world=1, clocks_index=None, profile=False):
        """Device time (ms) of `steps` steps, max over ranks.  With `profile`, the library records
        events around every phase (push, sort, field) and the phase profile is returned too; the
        events cost time between the kernels, so the headline is timed without them."""
        import ctypes

        import torch
        import torch.distributed as dist

        r, lib = self.run, self.lib
        r._check(lib.h1d_profile_enable(r.h, 1 if profile else 0))
        start, end = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        if world > 1:
            dist.barrier()
        torch.cuda.synchronize()
        clk = ClockSampler(clocks_index) if clocks_index is not None else None
        if clk:
            clk.__enter__()
        try:
            start.record(self.stream)
            r._check(lib.h1d_advance_async(r.h, steps))
            end.record(self.stream)
            r._check(lib.h1d_synchronize(r.h))
            torch.cuda.synchronize()
        finally:
            if clk:
                clk.__exit__(None, None, None)
        ms = start.elapsed_time(end)
        prof = None
        if profile:
            prof = self.h.abi.Profile()
            r._check(lib.h1d_profile_read(r.h, ctypes.byref(prof)))
            r._check(lib.h1d_profile_enable(r.h, 0))
        if world > 1:
            ms, _ = reduce_over_ranks(ms, 0.0)
            dist.barrier()
        return ms, prof, (clk.summary() if clk else None)

    def close(self):
        self.run.close()


def roofline_of(prof, precision, steps, traffic_table, workload=None):
    """Roofline of the dominant kernel (the particle pass): algorithmic bytes per launch over its
    average launch time (CUDA events on the run's stream around every launch).  `traffic` is the
    DRAM bytes per particle of an ncu capture of the same kernel (profiles/push_kernel_traffic.json,
    keyed by precision, or by precision and workload), scaled to this launch's particles."""
    peak, peak_kind = measured_peak()
    B = BYTES_PER_PARTICLE_STEP[precision]
    push_avg_ms = prof.push_ms / max(prof.push_launches, 1)
    bytes_per_launch = B * prof.particles_pushed / max(prof.push_launches, 1)
    achieved = bytes_per_launch / (push_avg_ms / 1e3) / 1e9
    traffic = None
    tr = traffic_table.get(f"{precision}:{workload}") or traffic_table.get(precision)
    if tr:
        traffic = tr["bytes_per_particle"] * bytes_per_launch / B
    return {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
            "traffic": traffic, "kernel": KERNEL[precision], "peak_kind": peak_kind,
            "bytes_per_particle_step": B, "bytes_per_launch": bytes_per_launch, "launch_ms": push_avg_ms,
            "window_miss_rate": prof.window_misses / max(2 * prof.particles_pushed, 1),
            "phase_ms_per_step": {"push": prof.push_ms / steps, "sort": prof.sort_ms / steps,
                                  "field": prof.field_ms / steps}}


def load_traffic():
    path = os.path.join(ROOT, "profiles", "push_kernel_traffic.json")
    try:
        with open(path) as f:
            return json.load(f)
    except Exception:
        return {}


def error_vs_fp64(h, cfg, st, steps=100):
    """Max-norm relative error of the mixed run against the FP64 CUDA run after `steps` steps from
    the same full-size state: wave energy (dB^2/2, dE^2/2 per component), particle energies and
    the moments."""
    import numpy as np

    out = {}
    for prec in (h.configs.PREC_FP64, h.configs.PREC_MIXED):
        with h.open_run(cfg.replace(precision=prec)) as r:
            r.upload_state(st)
            r.advance(steps)
            e = r.energy()
            mom = [r.moments(s) for s in range(len(cfg.kinetic))]
            out[prec] = (e, mom)
    (e0, m0), (e1, m1) = out[h.configs.PREC_FP64], out[h.configs.PREC_MIXED]

    def rel(a, b):
        a, b = np.asarray(a), np.asarray(b)
        sc = np.max(np.abs(b))
        return float(np.max(np.abs(a - b)) / sc) if sc else float(np.max(np.abs(a - b)))

    errs = {"dB2O2": rel(e1["dB2O2"], e0["dB2O2"]), "dE2O2": rel(e1["dE2O2"], e0["dE2O2"]),
            "KE_lab": rel(e1["KE_lab"], e0["KE_lab"]), "KE_pla": rel(e1["KE_pla"], e0["KE_pla"])}
    for s in range(len(cfg.kinetic)):
        for k, key in enumerate(("n", "nV", "nvv")):
            errs[f"moments[{s}].{key}"] = rel(m1[s][k], m0[s][k])
    return {"comparator": "the FP64 CUDA path, same full-size state", "steps": steps, "max": max(errs.values()),
            "tolerance": 1e-4, "within_tolerance": max(errs.values()) <= 1e-4, "errors": errs}


def error_vs_reference(h, cfg, divisor=64, every=10):
    """The CUDA path, mixed precision and FP64, against the reference itself over the
    configuration's whole length.  The reference binary (oracle/_ref/<name>/ref_driver: the
    reference's Domain_CAMCL compiled from its sources, FP64 on one host core) loads 1/divisor of
    the particles with its own loader (PartSpecies::populate(0, divisor)) and records the
    EnergyRecorder sums (dB^2/2, dE^2/2, and per species KE_lab and KE_pla) every `every` steps
    for cfg.steps steps; the CUDA path starts from the same state file and records the same sums
    through h1d_energy.  Errors: the largest |W - W_ref| over the run relative to the largest
    W_ref, for the wave energy (sum of the six components) and for each particle-energy component
    (the worst one is reported).  Returns None when the reference binary is absent."""
    import tempfile

    import numpy as np

    drv = os.path.join(ROOT, "oracle", "_ref", cfg.name, "ref_driver")
    if not os.path.exists(drv):
        return None
    sys.path[:0] = [os.path.join(ROOT, "tests", "golden"), os.path.join(ROOT, "tests")]
    from parity_util import with_reference_norms
    from state_io import read_state

    chunks = cfg.steps // every
    with tempfile.TemporaryDirectory(prefix="h1d_bench_") as tmp:
        init, series = os.path.join(tmp, "init.bin"), os.path.join(tmp, "series.bin")
        subprocess.run([drv, "init", init, "0", str(divisor)], check=True, timeout=600, capture_output=True)
        t0 = time.perf_counter()
        subprocess.run([drv, "series", init, str(every), str(chunks), series], check=True, timeout=1200,
                       capture_output=True)
        ref_s = time.perf_counter() - t0
        st = read_state(init)
        ref = np.fromfile(series).reshape(chunks, -1)
    n = sum(p["q1"].size for p in st["particles"])
    wave_ref = ref[:, :6].sum(axis=1)
    kin_ref = ref[:, 6:]
    kin_scale = np.abs(kin_ref).max(axis=0)
    cols = kin_scale > 0
    res = {"comparator": "reference binary (oracle/_ref ref_driver: Domain_CAMCL from the reference sources, "
                         "FP64, one host core), EnergyRecorder sums",
           "workload": f"{cfg.name} with 1/{divisor} of the particles ({n}), the reference loader's state",
           "steps": chunks * every, "every": every, "reference_s": ref_s}
    for prec, key in ((h.configs.PREC_MIXED, "mixed"), (h.configs.PREC_FP64, "fp64")):
        rows = []
        with h.open_run(with_reference_norms(cfg, st).replace(precision=prec)) as r:
            r.upload_state(st)
            for _ in range(chunks):
                r.advance(every)
                e = r.energy()
                per_species = [np.concatenate([lab, pla]) for lab, pla in zip(e["KE_lab"], e["KE_pla"])]
                rows.append(np.concatenate([e["dB2O2"], e["dE2O2"], *per_species]))
        rows = np.array(rows)
        wave = np.abs(rows[:, :6].sum(axis=1) - wave_ref) / wave_ref.max()
        kin = (np.abs(rows[:, 6:] - kin_ref)[:, cols] / kin_scale[cols]).max(axis=1)
        res[key] = {"wave_energy": float(wave.max()), "particle_energy": float(kin.max()),
                    "wave_energy_at": {str((i + 1) * every): float(wave[i]) for i in
                                       sorted({0, chunks // 10, chunks // 2, chunks - 1})}}
    res["wave_energy_range"] = [float(wave_ref.min()), float(wave_ref.max())]
    return res


def e2e_measure(h, cfg, st, K, world, tuned=None):
    """The same metric through the C-ABI with host buffers: upload from pinned memory, K steps as
    advance_by(inner_Nt) chunks with the recorder downloads (fields, sources, moments) after each,
    particles back at the end, all host buffers pinned and owned by the caller; wall clock, max over
    ranks.  The run is configured (h1d_configure) with the sort interval and CTAs the autotuner
    chose for the device-timed run (`tuned`), as a caller would after tuning once."""
    import numpy as np
    import torch
    import torch.distributed as dist

    n_particles = sum(p["q1"].size for p in st["particles"])
    keys = ("q1", "vx", "vy", "vz", "w")

    def pinned_like(p, copy):
        d = {}
        for key in keys:
            t = torch.empty(p[key].size, dtype=torch.float64, pin_memory=True)
            if copy:
                t.numpy()[:] = p[key]
            d[key] = t.numpy()
        return d

    # the caller's host buffers, in pinned memory and allocated before the timed region: the
    # particles to upload, and the arrays the particles and the recorder grids come back into
    pinned = [pinned_like(p, True) for p in st["particles"]]
    back = [pinned_like(p, False) for p in st["particles"]]
    M = st["B"].shape[0]

    def pinned_grid(*shape):
        return torch.zeros(*shape, dtype=torch.float64, pin_memory=True).numpy()

    grids = dict(B=pinned_grid(M, 3), E=pinned_grid(M, 3), rho=pinned_grid(M), J=pinned_grid(M, 3),
                 n=pinned_grid(M), nV=pinned_grid(M, 3), nvv=pinned_grid(M, 6))
    inner = cfg.inner_Nt
    with h.open_run(cfg) as r2:
        if tuned:
            h.abi.configure(r2, sort_interval=tuned["sort_interval"], push_ctas_per_sm=tuned["ctas_per_sm"])
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
            r2.fields(out=(grids["B"], grids["E"]))
            r2.sources(out=(grids["rho"], grids["J"]))
            d2h += sum(grids[k].nbytes for k in ("B", "E", "rho", "J"))
            for s in range(len(cfg.kinetic)):
                d2h += sum(a.nbytes for a in r2.moments(s, out=(grids["n"], grids["nV"], grids["nvv"])))
        for s in range(len(cfg.kinetic)):
            p = r2.particles(s, out=back[s], with_pid=False)
            d2h += sum(p[k].nbytes for k in keys)
        torch.cuda.synchronize()
        e2e_s = time.perf_counter() - t0
    if world > 1:
        e2e_s, _ = reduce_over_ranks(e2e_s, 0.0)
    h2d = sum(p["q1"].nbytes * 5 for p in st["particles"]) + st["B"].nbytes + st["E"].nbytes
    return {"value": n_particles * K * world / e2e_s, "unit": METRIC, "h2d_bytes_per_step": h2d / K,
            "d2h_bytes_per_step": d2h / K,
            "note": f"FP64 host buffers in pinned memory; upload, {K} steps as advance_by({inner}) chunks with "
                    "field/source/moment downloads after each chunk, particle download at the end; sort interval "
                    "and CTAs as the autotuner chose for the device-timed run"}


def ensemble_measure(h, precision, steps=500, members=64):
    """The ensemble workload: `members` runs drawn with seeds 0..members-1 (Nx uniform over
    256..4096, particles per cell log-uniform in [100, 2000], T_perp/T_par, beta_par and xi drawn,
    TSC), loaded on the device, advanced together by `steps` steps in one batch (one particle-pass
    launch and one field launch per step, pairs of sort blocks replayed as CUDA graphs) after the
    autotuner chose the sort interval and CTA count.  Returns runs/s and particle-steps/s."""
    import torch

    cfgs = [h.configs.ensemble_member(seed, precision=precision, steps=steps) for seed in range(members)]
    runs = []
    try:
        for seed, c in enumerate(cfgs):
            r = h.open_run(c)
            h.abi.populate_state(r, seed)
            runs.append(r)
        n_particles = sum(c.n_particles for c in cfgs)
        with h.abi.Batch(runs) as b:
            tuned_steps, k, ctas = b.autotune()
            stream = torch.cuda.ExternalStream(b.stream())
            b.advance(4 * k)  # warm-up: builds and replays the graph of the chosen interval
            s0 = b.stats()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            torch.cuda.synchronize()
            e0.record(stream)
            b.advance_async(steps)
            e1.record(stream)
            b.synchronize()
            torch.cuda.synchronize()
            ms = e0.elapsed_time(e1)
            s1 = b.stats()
    finally:
        for r in runs:
            r.close()
    # the same members one after another, each alone (their own stream, the library's default
    # sort interval and CTAs): what the batch replaces
    alone_ms = 0.0
    for seed, c in enumerate(cfgs):
        tr = TimedRun(h, c, None, populate_seed=seed)
        try:
            tr.advance(4)
            m, _, _ = tr.timed(steps)
            alone_ms += m
        finally:
            tr.close()
    alone = {"workload": f"the {members} members one after another, each alone", "runs_per_s": members / (alone_ms / 1e3),
             "value": n_particles * steps / (alone_ms / 1e3)}

    # the same plasma as one dense run: the first Nx=4096 member's plasma holding as many particles
    # as the whole ensemble (about 20 000 per cell, where a sorted warp's particles share a cell),
    # advanced alone with its own autotuned sort interval and CTAs
    import dataclasses

    base = next(c for c in cfgs if c.Nx == max(x.Nx for x in cfgs))
    one = base.replace(kinetic=[dataclasses.replace(base.kinetic[0], Nc=max(1, n_particles // base.Nx))])
    tr = TimedRun(h, one, None, populate_seed=0)
    try:
        tr.warm(4)
        ms1, _, _ = tr.timed(steps)
        single = {"workload": f"{base.name} plasma at Nx {base.Nx} with {one.kinetic[0].Nc} particles per cell "
                              f"({tr.n_particles} particles), alone", "value": tr.n_particles * steps / (ms1 / 1e3),
                  "autotune": tr.tuned}
    finally:
        tr.close()
    value = n_particles * steps / (ms / 1e3)
    return {"workload": f"ensemble of {members} runs (seeds 0..{members - 1}), {steps} steps each, TSC",
            "precision": "mixed" if precision == h.configs.PREC_MIXED else "fp64",
            "runs_per_s": members / (ms / 1e3), "value": value, "unit": METRIC,
            "members_alone": alone, "over_members_alone": value / alone["value"],
            "dense_single_run": single, "over_dense_single_run": value / single["value"],
            "ms": ms, "particles": n_particles, "Nx": [c.Nx for c in cfgs][:8] + ["..."],
            "autotune": {"steps": tuned_steps, "sort_interval": k, "ctas_per_sm": ctas},
            "gpu_launches": s1["kernel_launches"] - s0["kernel_launches"],
            "graph_launches": s1["graph_launches"] - s0["graph_launches"]}


def serving_measure(h, precision, n_requests=48, rate=4.0, budget_gb=150, seed=2024):
    """The serving workload: a seeded Poisson stream (mean `rate` per second) of `n_requests`
    requests drawn like the ensemble members with steps uniform in [200, 2000], served in real time
    by the continuous-batching server under a `budget_gb` HBM budget.  Latency = completion time -
    submission time; throughput = completed runs / (last completion - first submission)."""
    import numpy as np

    rng = np.random.default_rng(seed)
    arrivals = np.cumsum(rng.exponential(1.0 / rate, n_requests)) if rate else np.zeros(n_requests)
    steps = rng.integers(200, 2001, n_requests)
    lib = h.library_path()
    sv = h.abi.Server(lib, int(budget_gb * (1 << 30)), steps_per_tick=64, sort_interval=16)
    ids = []
    try:
        # warm-up outside the measurement: two short requests load the kernels a served run uses
        warm = [sv.submit(h.configs.ensemble_member(seed, precision=precision), seed=seed, n_steps=64)
                for seed in (7, 11)]
        while any(sv.poll(i)["state"] < h.abi.REQ_DONE for i in warm):
            sv.tick()
        for i in warm:
            sv.release(i)
        t0 = time.perf_counter()
        nxt = 0
        done = set()
        while len(done) < n_requests:
            now = time.perf_counter() - t0
            while nxt < n_requests and arrivals[nxt] <= now:
                cfg = h.configs.ensemble_member(1000 + nxt, precision=precision)
                ids.append(sv.submit(cfg, seed=1000 + nxt, n_steps=int(steps[nxt])))
                nxt += 1
            active, queued = sv.tick()
            for i in ids:
                if i not in done and sv.poll(i)["state"] >= h.abi.REQ_DONE:
                    done.add(i)
            if active == 0 and queued == 0 and nxt < n_requests:
                time.sleep(max(0.0, min(0.05, arrivals[nxt] - (time.perf_counter() - t0))))
        polls = [sv.poll(i) for i in ids]
        st = sv.stats()
    finally:
        sv.close()
    # the yardstick of the tail: the largest request (particles x steps) served alone
    work = [h.configs.ensemble_member(1000 + i, precision=precision).n_particles * int(steps[i])
            for i in range(n_requests)]
    big = int(np.argmax(work))
    sv = h.abi.Server(lib, int(budget_gb * (1 << 30)), steps_per_tick=64, sort_interval=16)
    try:
        i = sv.submit(h.configs.ensemble_member(1000 + big, precision=precision), seed=1000 + big,
                      n_steps=int(steps[big]))
        while sv.poll(i)["state"] < h.abi.REQ_DONE:
            sv.tick()
        p1 = sv.poll(i)
        alone = p1["t_done"] - p1["t_submit"]
    finally:
        sv.close()
    lat = np.array([p["t_done"] - p["t_submit"] for p in polls])
    span = max(p["t_done"] for p in polls) - min(p["t_submit"] for p in polls)
    failed = sum(p["state"] != h.abi.REQ_DONE for p in polls)
    stream = f"Poisson stream, mean {rate}/s" if rate else "all submitted at once (saturated)"
    return {"workload": f"{stream}, {n_requests} requests (ensemble draws, steps U[200, 2000]), {budget_gb} GB HBM budget",
            "precision": "mixed" if precision == h.configs.PREC_MIXED else "fp64",
            "runs_per_s": (n_requests - failed) / span, "p50_s": float(np.percentile(lat, 50)),
            "p99_s": float(np.percentile(lat, 99)), "mean_s": float(lat.mean()), "failed": int(failed),
            "largest_alone_s": alone, "p99_over_largest_alone": float(np.percentile(lat, 99)) / alone,
            "peak_hbm_gb": st["peak_bytes"] / (1 << 30), "batches_built": st["batches_built"],
            "gpu_launches": st["kernel_launches"], "graph_launches": st["graph_launches"]}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=2000)  # the configuration's run length
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--config", default="config3_cic_periodic_nx4096")
    ap.add_argument("--precision", default="auto", choices=["auto", "fp64", "mixed"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-extras", action="store_true", help="skip the fp64 / error / drop-in side measurements")
    ap.add_argument("--no-ensemble", action="store_true", help="skip the ensemble and serving measurements")
    ap.add_argument("--no-autotune", action="store_true", help="keep the library's default sort interval and CTAs")
    args = ap.parse_args()
    assert args.warmup >= 3 or args.impl == "reference", "at least 3 warm-up steps"
    if int(os.environ.get("WORLD_SIZE", "1")) > 1:  # replicas: each rank measures the headline only
        args.no_extras = args.no_ensemble = True

    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    h = _package()
    if args.impl == "reference":
        run_reference_arm(args, h, rank)
        return

    import torch
    import torch.distributed as dist

    torch.cuda.set_device(local)
    if world > 1:
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=120), device_id=torch.device("cuda", local))
    cfg = workload(h, args.config)
    if args.precision != "auto":
        cfg = cfg.replace(precision=h.configs.PREC_MIXED if args.precision == "mixed" else h.configs.PREC_FP64)
    prec = precision_name(cfg, h)
    from hfemic_b200.loader import initial_state

    st = initial_state(cfg, seed=1000 + rank)
    traffic = load_traffic()

    tr = TimedRun(h, cfg, st)
    tuned = tr.warm(args.warmup, autotune=not args.no_autotune)
    ms, _, clocks = tr.timed(args.steps, world, clocks_index=local)  # the headline: no phase events
    ms_p, prof, _ = tr.timed(args.steps, world, profile=True)       # the same steps again, per phase
    n_particles = tr.n_particles
    tr.close()
    value = n_particles * args.steps * world / (ms / 1e3)
    roofline = roofline_of(prof, prec, args.steps, traffic)
    roofline["profiled_ms_per_step"] = ms_p / args.steps

    # side measurements on the same state: the plain FP64 pass, the mixed pass's error against it,
    # and the FP64 drop-in configuration
    extras = {}
    if not args.no_extras:
        if prec == "mixed":
            t64 = TimedRun(h, cfg.replace(precision=h.configs.PREC_FP64), st)
            tuned64 = t64.warm(args.warmup, autotune=not args.no_autotune)
            ms64, _, _ = t64.timed(args.steps, world)
            _, prof64, _ = t64.timed(args.steps, world, profile=True)
            t64.close()
            v64 = n_particles * args.steps * world / (ms64 / 1e3)
            extras["fp64"] = {"value": v64, "unit": METRIC, "ms_per_step": ms64 / args.steps, "autotune": tuned64,
                              "roofline": roofline_of(prof64, "fp64", args.steps, traffic)}
            extras["mixed_over_fp64"] = value / v64
            extras["error_vs_fp64"] = error_vs_fp64(h, cfg, st)
            extras["error_vs_reference"] = error_vs_reference(h, cfg)
        if cfg.name != "config2_tsc_mirror_nx2048":
            # the FP64 drop-in configuration with the reference's reflecting walls (the parity form)
            # and with the particle-absorbing walls the configuration names (an extension: the
            # reference has periodic and reflecting particle boundaries only)
            c2 = h.configs.config2()
            st2 = initial_state(c2, seed=2000 + rank)
            for key, bc in (("drop_in_fp64", h.configs.BC_REFLECTING), ("drop_in_fp64_absorbing", h.configs.BC_ABSORBING)):
                cb = c2.replace(particle_bc=bc)
                t2 = TimedRun(h, cb, st2)
                tuned2 = t2.warm(args.warmup, autotune=not args.no_autotune)
                k2 = max(args.steps, 100)
                ms2, _, _ = t2.timed(k2, world)
                _, prof2, _ = t2.timed(k2, world, profile=True)
                v2 = t2.n_particles * k2 * world / (ms2 / 1e3)
                t2.close()
                extras[key] = {"workload": c2.name, "particle_bc": "reflecting" if bc == h.configs.BC_REFLECTING else
                               "absorbing (extension; the reference has no absorbing boundary)",
                               "particles_per_gpu": t2.n_particles, "value": v2, "autotune": tuned2,
                               "unit": METRIC, "ms_per_step": ms2 / k2,
                               "roofline": roofline_of(prof2, "fp64", k2, traffic, c2.name)}
            del st2

    e2e = None if args.no_e2e else e2e_measure(h, cfg, st, args.steps, world, tuned)
    del st

    if not args.no_ensemble:
        extras["ensemble"] = {p: ensemble_measure(h, getattr(h.configs, "PREC_" + p.upper())) for p in ("mixed", "fp64")}
        extras["serving"] = {p: serving_measure(h, getattr(h.configs, "PREC_" + p.upper())) for p in ("mixed", "fp64")}
        extras["serving"]["mixed_saturated"] = serving_measure(h, h.configs.PREC_MIXED, rate=None)

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        cpu = cpu_baseline_reference(cfg) or cpu_baseline_port(h, cfg)
        if not args.no_ensemble:
            ens_cpu, srv_cpu = cpu_ensemble_serving_baselines(h)
            extras["ensemble"]["cpu_baseline"] = ens_cpu
            extras["serving"]["cpu_baseline"] = srv_cpu

    if world > 1:
        dist.destroy_process_group()
    if rank != 0:
        return
    state_mb = n_particles * STATE_BYTES[prec] / 1e6
    head = {}  # the headline comparisons first, so that a truncated line still carries them
    if "fp64" in extras:
        head = {"mixed_over_fp64": extras.pop("mixed_over_fp64"), "fp64_value": extras["fp64"]["value"],
                "frac": roofline["frac"], "fp64_frac": extras["fp64"]["roofline"]["frac"]}
    if "drop_in_fp64" in extras:
        head["drop_in_fp64_frac"] = extras["drop_in_fp64"]["roofline"]["frac"]
        head["field_ms"] = roofline.get("phase_ms_per_step", {}).get("field")
        head["drop_in_field_ms"] = extras["drop_in_fp64"]["roofline"].get("phase_ms_per_step", {}).get("field")
    line = {
        "metric": METRIC, "value": value, **head, "unit": METRIC, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms / args.steps, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32+i32 particles, f64 fields" if prec == "mixed" else "f64",
        "data": "synthetic (seeded bi-Maxwellian loader)",
        "config": {"workload": cfg.name, "Nx": cfg.Nx, "particles_per_gpu": n_particles,
                   "species": len(cfg.kinetic), "ppc": [k.Nc for k in cfg.kinetic],
                   "shape_order": [k.shape_order for k in cfg.kinetic], "xi": cfg.xi,
                   "algorithm": "CAM-CL" if cfg.algorithm == h.configs.ALGO_CAMCL else "PC",
                   "n_subcycles": cfg.n_subcycles, "precision": prec,
                   "l2": f"particle state ({state_mb:.0f} MB per GPU, one buffer set) larger than L2; no flush",
                   "parallelism": f"replicas x{world}",
                   "autotune": tuned,
                   "warmup_note": "W plain warm-up steps, then the autotuner's own (real) steps, both untimed"},
        "roofline": roofline, "cpu_baseline": cpu, "e2e": e2e, "clocks": clocks,
        "gpu_launches": int(prof.kernel_launches),
        **extras,
    }
    print(json.dumps(line))


if __name__ == "__main__":
    main()
