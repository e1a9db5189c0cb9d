"""ctypes mirror of include/h1d_gpu.h.

:class:`Run` drives one run through any library exporting the h1d C-ABI (the entry
points are looked up with a name prefix, ``h1d_`` for the CUDA library).  Errors come back
as the exceptions the reference raises for the same condition: ``H1D_ERR_MOVED_TOO_FAR``
is ``std::domain_error`` "particle(s) moved too far" in PartSpecies::update_pos
(src/hybrid_1d/Core/PartSpecies.cc:113) and becomes :class:`MovedTooFar`;
``H1D_ERR_INVALID_ARG`` (std::invalid_argument) becomes :class:`ValueError`.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

from . import configs as _cfg

PAD = 3
MAX_KINETIC = 8
MAX_COLD = 4
ABI_VERSION = 4

OK, ERR_INVALID_ARG, ERR_MOVED_TOO_FAR, ERR_OOM, ERR_CUDA, ERR_TIMEOUT, ERR_NAN, ERR_STATE, \
    ERR_NO_DEVICE = range(9)


class H1DError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__(f"h1d error {code}: {msg}")
        self.code = code


class MovedTooFar(H1DError):
    """std::domain_error("... - particle(s) moved too far") of PartSpecies::update_pos."""


class KineticDesc(C.Structure):
    _fields_ = [("Oc", C.c_double), ("op", C.c_double), ("n_smooth", C.c_int64), ("Nc", C.c_int64),
                ("shape_order", C.c_int64), ("moment_norm", C.c_double), ("scheme", C.c_int32),
                ("vdf", C.c_int32), ("psd_refresh_frequency", C.c_double), ("vth1", C.c_double),
                ("T2_T1", C.c_double), ("vdf_param", C.c_double * 3)]


class ColdDesc(C.Structure):
    _fields_ = [("Oc", C.c_double), ("op", C.c_double), ("n_smooth", C.c_int64)]


class EFluidDesc(C.Structure):
    _fields_ = [("Oc", C.c_double), ("op", C.c_double), ("beta", C.c_double), ("gamma", C.c_double)]


MAX_SOURCES, MAX_SOURCE_POINTS = 2, 16


class SourceDesc(C.Structure):
    _fields_ = [("omega", C.c_double), ("start", C.c_double), ("duration", C.c_double),
                ("ease_in", C.c_double), ("ease_out", C.c_double), ("n_smooth", C.c_int64),
                ("n_points", C.c_int64), ("pos", C.c_double * MAX_SOURCE_POINTS),
                ("J0re", (C.c_double * 3) * MAX_SOURCE_POINTS), ("J0im", (C.c_double * 3) * MAX_SOURCE_POINTS)]


class Params(C.Structure):
    _fields_ = [
        ("Nx", C.c_int64), ("Dx", C.c_double), ("xi", C.c_double), ("O0", C.c_double),
        ("c", C.c_double), ("dt", C.c_double), ("n_subcycles", C.c_int64),
        ("algorithm", C.c_int32), ("particle_bc", C.c_int32), ("randomize_gyrophase", C.c_int32),
        ("precision", C.c_int32), ("gyrophase_seed", C.c_uint64),
        ("phase_retardation_inset", C.c_int64), ("phase_retardation_factor", C.c_double),
        ("amplitude_damping_inset", C.c_int64), ("amplitude_damping_factor", C.c_double),
        ("moment_weighting", C.c_double), ("sort_interval", C.c_int32), ("n_kinetic", C.c_int32),
        ("n_cold", C.c_int32), ("n_sources", C.c_int32), ("efluid", EFluidDesc),
        ("kinetic", KineticDesc * MAX_KINETIC), ("cold", ColdDesc * MAX_COLD),
        ("sources", SourceDesc * MAX_SOURCES),
    ]


def make_params(cfg: "_cfg.RunConfig") -> Params:
    cfg.validate()
    p = Params()
    p.Nx, p.Dx, p.xi, p.O0, p.c, p.dt = cfg.Nx, cfg.Dx, cfg.xi, cfg.O0, cfg.c, cfg.dt
    p.n_subcycles = cfg.n_subcycles
    p.algorithm, p.particle_bc = cfg.algorithm, cfg.particle_bc
    p.randomize_gyrophase, p.gyrophase_seed = int(cfg.randomize_gyrophase), cfg.gyrophase_seed
    p.precision = cfg.precision
    p.phase_retardation_inset, p.phase_retardation_factor = cfg.phase_retardation
    p.amplitude_damping_inset, p.amplitude_damping_factor = cfg.amplitude_damping
    p.moment_weighting = 1.0
    p.sort_interval = cfg.sort_interval
    p.n_kinetic, p.n_cold = len(cfg.kinetic), len(cfg.cold)
    if p.n_kinetic > MAX_KINETIC or p.n_cold > MAX_COLD:
        raise ValueError("too many species")
    ef = cfg.efluid
    p.efluid = EFluidDesc(ef.Oc, ef.op, ef.beta, ef.gamma)
    for i, k in enumerate(cfg.kinetic):
        p.kinetic[i] = KineticDesc(k.Oc, k.op, k.n_smooth, k.Nc, k.shape_order, cfg.moment_norm(k), k.scheme, k.vdf,
                                   k.psd_refresh_frequency, k.vth1(cfg.c), k.T2_T1, (C.c_double * 3)(*k.vdf_param()))
    for i, c in enumerate(cfg.cold):
        p.cold[i] = ColdDesc(c.Oc, c.op, c.n_smooth)
    if len(cfg.sources) > MAX_SOURCES:
        raise ValueError("too many external sources")
    p.n_sources = len(cfg.sources)
    for i, src in enumerate(cfg.sources):
        d = p.sources[i]
        d.omega, d.start, d.duration = src.omega, src.start, src.duration
        d.ease_in, d.ease_out, d.n_smooth = src.ease_in, src.ease_out, src.n_smooth
        if len(src.points) > MAX_SOURCE_POINTS:
            raise ValueError("too many source points")
        d.n_points = len(src.points)
        for j, (q1, J0) in enumerate(src.points):
            d.pos[j] = q1
            for c in range(3):
                d.J0re[j][c], d.J0im[j][c] = complex(J0[c]).real, complex(J0[c]).imag
    return p


class Profile(C.Structure):
    _fields_ = [("push_ms", C.c_double), ("sort_ms", C.c_double), ("field_ms", C.c_double),
                ("push_launches", C.c_int64), ("sort_calls", C.c_int64), ("field_launches", C.c_int64),
                ("kernel_launches", C.c_int64), ("particles_pushed", C.c_int64),
                ("window_misses", C.c_int64)]


_dp = C.POINTER(C.c_double)
_lp = C.POINTER(C.c_int64)


def _declare(lib, prefix):
    def f(name, *args, res=C.c_int):
        fn = getattr(lib, prefix + name)
        fn.argtypes = list(args)
        fn.restype = res
        return fn

    v = C.c_void_p
    return dict(
        create=f("create", C.POINTER(Params), C.POINTER(C.c_void_p)),
        destroy=f("destroy", v),
        upload_particles=f("upload_particles", v, C.c_int, C.c_int64, _dp, _dp, _dp, _dp, _dp),
        upload_fields=f("upload_fields", v, _dp, _dp),
        upload_cold=f("upload_cold", v, C.c_int, _dp, _dp),
        advance=f("advance", v, C.c_uint32),
        particle_count=f("particle_count", v, C.c_int, _lp),
        download_particles=f("download_particles", v, C.c_int, _dp, _dp, _dp, _dp, _dp, _lp),
        upload_psd=f("upload_psd", v, C.c_int, C.c_int64, _dp, _dp),
        download_psd=f("download_psd", v, C.c_int, _dp, _dp),
        download_fields=f("download_fields", v, _dp, _dp),
        download_sources=f("download_sources", v, _dp, _dp),
        download_moments=f("download_moments", v, C.c_int, _dp, _dp, _dp),
        download_cold=f("download_cold", v, C.c_int, _dp, _dp, _dp, _dp, _dp),
        energy=f("energy", v, _dp, _dp, _dp, _dp),
        status_string=f("status_string", v, res=C.c_char_p),
    )


def _ptr(a, ctype=C.c_double):
    if a is None:
        return None
    return a.ctypes.data_as(C.POINTER(ctype))


_LIBS = {}


def load_library(path: str, prefix: str):
    key = (os.path.abspath(path), prefix)
    if key not in _LIBS:
        lib = C.CDLL(key[0])
        _LIBS[key] = (lib, _declare(lib, prefix))
    return _LIBS[key]


class Run:
    """One run (a Domain) behind the h1d C-ABI of library ``path`` with symbol ``prefix``."""

    def __init__(self, cfg: "_cfg.RunConfig", path: str, prefix: str = "h1d_"):
        self.cfg = cfg
        self.lib, self.fn = load_library(path, prefix)
        self.params = make_params(cfg)
        self.M = cfg.Nx + 2 * PAD
        h = C.c_void_p()
        self._check(self.fn["create"](C.byref(self.params), C.byref(h)), h=None)
        self.h = h

    # ----- plumbing -----
    def _check(self, st, h="self"):
        if st == OK:
            return
        hh = self.h if h == "self" else h
        msg = self.fn["status_string"](hh).decode() if hh else ""
        if st == ERR_MOVED_TOO_FAR:
            raise MovedTooFar(st, msg or "particle(s) moved too far")
        if st == ERR_INVALID_ARG:
            raise ValueError(msg or "invalid argument")
        raise H1DError(st, msg)

    def close(self):
        if getattr(self, "h", None):
            self.fn["destroy"](self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    # ----- uploads -----
    def upload_particles(self, s, q1, vx, vy, vz, w):
        arrs = [np.ascontiguousarray(a, dtype=np.float64) for a in (q1, vx, vy, vz, w)]
        n = arrs[0].size
        self._check(self.fn["upload_particles"](self.h, s, n, *[_ptr(a) for a in arrs]))

    def upload_fields(self, B, E):
        B = np.ascontiguousarray(B, dtype=np.float64).reshape(-1)
        E = np.ascontiguousarray(E, dtype=np.float64).reshape(-1)
        assert B.size == 3 * self.M and E.size == 3 * self.M
        self._check(self.fn["upload_fields"](self.h, _ptr(B), _ptr(E)))

    def upload_cold(self, i, n_full, nV_full):
        n = np.ascontiguousarray(n_full, dtype=np.float64).reshape(-1)
        v = np.ascontiguousarray(nV_full, dtype=np.float64).reshape(-1)
        self._check(self.fn["upload_cold"](self.h, i, _ptr(n), _ptr(v)))

    def upload_psd(self, s, real_f, marker):
        """Particle::PSD of species s (real_f, marker), in upload order."""
        arrs = [np.ascontiguousarray(a, dtype=np.float64) for a in (real_f, marker)]
        self._check(self.fn["upload_psd"](self.h, s, arrs[0].size, *[_ptr(a) for a in arrs]))

    def psd(self, s):
        """(real_f, marker) of species s, in the order of particles(s)."""
        n = self.particle_count(s)
        real_f, marker = np.empty(n), np.empty(n)
        self._check(self.fn["download_psd"](self.h, s, _ptr(real_f), _ptr(marker)))
        return real_f, marker

    def upload_state(self, st):
        """Upload a state dict as read by tests/golden/state_io.read_state (the phase-space
        densities too, for the species whose weights evolve)."""
        for s, p in enumerate(st["particles"]):
            self.upload_particles(s, p["q1"], p["vx"], p["vy"], p["vz"], p["w"])
            if self.cfg.kinetic[s].has_psd:
                self.upload_psd(s, p["real_f"], p["marker"])
        self.upload_fields(st["B"], st["E"])
        for i, c in enumerate(st["cold"]):
            self.upload_cold(i, c["n_full"], c["nV_full"])

    # ----- stepping -----
    def advance(self, n_steps: int):
        self._check(self.fn["advance"](self.h, n_steps))

    # ----- downloads -----
    def particle_count(self, s) -> int:
        n = C.c_int64()
        self._check(self.fn["particle_count"](self.h, s, C.byref(n)))
        return n.value

    def particles(self, s, out=None, with_pid=True):
        """The particles of species s as FP64 arrays q1, vx, vy, vz, w (+ pid).  `out` may hold
        caller-owned arrays (for instance in pinned memory) of at least particle_count(s) elements;
        they are filled and returned as views of that length."""
        n = self.particle_count(s)
        keys = ("q1", "vx", "vy", "vz", "w")
        if out is None:
            out = {k: np.empty(n) for k in keys}
        else:
            for k in keys:
                a = out[k]
                if a.dtype != np.float64 or a.ndim != 1 or a.size < n or not a.flags.c_contiguous:
                    raise ValueError(f"particles: out[{k!r}] must be a contiguous float64 array of >= {n} elements")
            out = {k: out[k][:n] for k in keys}
        pid = np.empty(n, dtype=np.int64) if with_pid else None
        self._check(self.fn["download_particles"](self.h, s, *[_ptr(out[k]) for k in keys],
                                                  _ptr(pid, C.c_int64) if with_pid else None))
        if with_pid:
            out["pid"] = pid
        return out

    def _grids(self, out, shapes):
        """Caller-owned output grids (checked), or new ones."""
        if out is None:
            return [np.empty(sh) for sh in shapes]
        for a, sh in zip(out, shapes):
            if a.dtype != np.float64 or a.shape != sh or not a.flags.c_contiguous:
                raise ValueError(f"output grid must be a contiguous float64 array of shape {sh}")
        return list(out)

    def fields(self, out=None):
        B, E = self._grids(out, [(self.M, 3), (self.M, 3)])
        self._check(self.fn["download_fields"](self.h, _ptr(B), _ptr(E)))
        return B, E

    def sources(self, out=None):
        rho, J = self._grids(out, [(self.M,), (self.M, 3)])
        self._check(self.fn["download_sources"](self.h, _ptr(rho), _ptr(J)))
        return rho, J

    def moments(self, s, out=None):
        n, nV, nvv = self._grids(out, [(self.M,), (self.M, 3), (self.M, 6)])
        self._check(self.fn["download_moments"](self.h, s, _ptr(n), _ptr(nV), _ptr(nvv)))
        return n, nV, nvv

    def cold(self, i):
        n, nV, nvv = np.empty(self.M), np.empty((self.M, 3)), np.empty((self.M, 6))
        nf, nVf = np.empty(self.M), np.empty((self.M, 3))
        self._check(self.fn["download_cold"](self.h, i, _ptr(n), _ptr(nV), _ptr(nvv), _ptr(nf), _ptr(nVf)))
        return dict(n=n, nV=nV, nvv=nvv, n_full=nf, nV_full=nVf)

    def energy(self):
        ns = len(self.cfg.kinetic) + len(self.cfg.cold)
        b, e = np.empty(3), np.empty(3)
        lab, pla = np.empty((ns, 3)), np.empty((ns, 3))
        self._check(self.fn["energy"](self.h, _ptr(b), _ptr(e), _ptr(lab), _ptr(pla)))
        return dict(dB2O2=b, dE2O2=e, KE_lab=lab, KE_pla=pla)

    def state(self):
        """Everything, in the layout of tests/golden/state_io.read_state."""
        B, E = self.fields()
        rho, J = self.sources()
        st = dict(B=B, E=E, charge=rho, current=J, particles=[], moments=[], cold=[])
        for s in range(len(self.cfg.kinetic)):
            st["particles"].append(self.particles(s))
            if self.cfg.kinetic[s].has_psd:
                st["particles"][-1]["real_f"], st["particles"][-1]["marker"] = self.psd(s)
            n, nV, nvv = self.moments(s)
            st["moments"].append(dict(n=n, nV=nV, nvv=nvv))
        for i in range(len(self.cfg.cold)):
            st["cold"].append(self.cold(i))
        return st


# ---------------------------------------------------------------------------------------------
# ensembles and tuning (CUDA library only; no counterpart in the reference or the oracle)
# ---------------------------------------------------------------------------------------------

class BatchStats(C.Structure):
    _fields_ = [("steps", C.c_int64), ("kernel_launches", C.c_int64), ("graph_launches", C.c_int64),
                ("graphs_built", C.c_int64)]


def _declare_batch(lib):
    v, u = C.c_void_p, C.POINTER(C.c_uint32)
    ip = C.POINTER(C.c_int)
    spec = {
        "h1d_batch_create": ([C.POINTER(C.c_void_p), C.c_int, C.POINTER(C.c_void_p)], C.c_int),
        "h1d_batch_destroy": ([v], C.c_int),
        "h1d_batch_advance": ([v, C.c_uint32], C.c_int),
        "h1d_batch_advance_async": ([v, C.c_uint32], C.c_int),
        "h1d_batch_advance_members_async": ([v, C.POINTER(C.c_uint32)], C.c_int),
        "h1d_batch_synchronize": ([v], C.c_int),
        "h1d_batch_get_stream": ([v, C.POINTER(C.c_void_p)], C.c_int),
        "h1d_batch_configure": ([v, C.c_int, C.c_int, C.c_int], C.c_int),
        "h1d_batch_autotune": ([v, u, ip, ip], C.c_int),
        "h1d_batch_stats_read": ([v, C.POINTER(BatchStats)], C.c_int),
        "h1d_batch_status_string": ([v], C.c_char_p),
        "h1d_configure": ([v, C.c_int, C.c_int], C.c_int),
        "h1d_autotune": ([v, u, ip, ip], C.c_int),
    }
    for name, (args, res) in spec.items():
        fn = getattr(lib, name)
        fn.argtypes, fn.restype = args, res
    return lib


def configure(run: Run, sort_interval: int = 0, push_ctas_per_sm: int = 0):
    """Sort interval and CTAs per SM of the particle pass of one run (h1d_configure)."""
    lib = _declare_batch(run.lib)
    run._check(lib.h1d_configure(run.h, sort_interval, push_ctas_per_sm))


def autotune(run: Run):
    """h1d_autotune: advances the run by real steps while choosing its sort interval and CTA count.
    Returns (steps_taken, sort_interval, ctas_per_sm)."""
    lib = _declare_batch(run.lib)
    n, k, c = C.c_uint32(), C.c_int(), C.c_int()
    run._check(lib.h1d_autotune(run.h, C.byref(n), C.byref(k), C.byref(c)))
    return n.value, k.value, c.value


class Batch:
    """Many CAM-CL runs advanced together (h1d_batch_*); the runs stay owned by the caller."""

    def __init__(self, runs):
        self.runs = list(runs)
        self.lib = _declare_batch(self.runs[0].lib)
        arr = (C.c_void_p * len(self.runs))(*[r.h.value for r in self.runs])
        h = C.c_void_p()
        st = self.lib.h1d_batch_create(arr, len(self.runs), C.byref(h))
        if st != OK:
            raise H1DError(st, "h1d_batch_create failed")
        self.h = h

    def _check(self, st):
        if st == OK:
            return
        msg = self.lib.h1d_batch_status_string(self.h).decode()
        if st == ERR_MOVED_TOO_FAR or "moved too far" in msg:
            raise MovedTooFar(st, msg)
        raise H1DError(st, msg)

    def configure(self, sort_interval=0, push_ctas_per_sm=0, use_graphs=True):
        self._check(self.lib.h1d_batch_configure(self.h, sort_interval, push_ctas_per_sm, int(use_graphs)))

    def advance(self, n_steps: int):
        self._check(self.lib.h1d_batch_advance(self.h, n_steps))

    def advance_async(self, n_steps: int):
        self._check(self.lib.h1d_batch_advance_async(self.h, n_steps))

    def synchronize(self):
        self._check(self.lib.h1d_batch_synchronize(self.h))

    def advance_members(self, n_steps):
        """Member i advances by n_steps[i] (h1d_batch_advance_members_async), then the batch
        synchronises."""
        if len(n_steps) != len(self.runs):
            raise ValueError("advance_members: one step count per member")
        arr = (C.c_uint32 * len(n_steps))(*[int(x) for x in n_steps])
        self._check(self.lib.h1d_batch_advance_members_async(self.h, arr))
        self.synchronize()

    def stream(self):
        s = C.c_void_p()
        self._check(self.lib.h1d_batch_get_stream(self.h, C.byref(s)))
        return s.value

    def autotune(self):
        n, k, c = C.c_uint32(), C.c_int(), C.c_int()
        self._check(self.lib.h1d_batch_autotune(self.h, C.byref(n), C.byref(k), C.byref(c)))
        return n.value, k.value, c.value

    def stats(self):
        s = BatchStats()
        self._check(self.lib.h1d_batch_stats_read(self.h, C.byref(s)))
        return dict(steps=s.steps, kernel_launches=s.kernel_launches, graph_launches=s.graph_launches,
                    graphs_built=s.graphs_built)

    def close(self):
        if getattr(self, "h", None):
            self.lib.h1d_batch_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()


def populate(run: Run, s: int, seed: int, count: int | None = None):
    """h1d_populate: load kinetic species s of the run's configuration on the device (the particles
    loader.load_species computes on the host for the same seed)."""
    lib = run.lib
    fn = lib.h1d_populate
    fn.argtypes = [C.c_void_p, C.c_int, C.c_int64, C.c_uint64, C.c_double, C.c_double]
    fn.restype = C.c_int
    k = run.cfg.kinetic[s]
    n = k.Nc * run.cfg.Nx if count is None else count
    run._check(fn(run.h, s, n, seed, k.beta1, k.T2_T1))


def populate_state(run: Run, seed: int):
    """The state of loader.initial_state(cfg, seed) built on the device: every kinetic species by
    h1d_populate, the cold species at rest with unit density, zero fields."""
    cfg = run.cfg
    for s in range(len(cfg.kinetic)):
        populate(run, s, seed)
    M = cfg.Nx + 2 * PAD
    for i in range(len(cfg.cold)):
        n_full = np.zeros(M)
        n_full[PAD:PAD + cfg.Nx] = 1.0
        run.upload_cold(i, n_full, np.zeros((M, 3)))


# ---------------------------------------------------------------------------------------------
# serving loop (h1d_server_*)
# ---------------------------------------------------------------------------------------------

MAXK = 8
REQ_QUEUED, REQ_ACTIVE, REQ_DONE, REQ_FAILED = 0, 1, 2, 3


class Request(C.Structure):
    _fields_ = [("params", Params), ("beta1", C.c_double * MAXK), ("T2_T1", C.c_double * MAXK),
                ("n_particles", C.c_int64 * MAXK), ("seed", C.c_uint64), ("n_steps", C.c_uint32),
                ("reserved0", C.c_uint32)]


class ServerStats(C.Structure):
    _fields_ = [(k, C.c_int64) for k in ("submitted", "admitted", "completed", "failed", "steps", "kernel_launches",
                                         "graph_launches", "batches_built", "bytes_in_use", "peak_bytes")]


def make_request(cfg: "_cfg.RunConfig", seed: int, n_steps: int) -> Request:
    rq = Request()
    rq.params = make_params(cfg)
    for s, k in enumerate(cfg.kinetic):
        rq.beta1[s], rq.T2_T1[s], rq.n_particles[s] = k.beta1, k.T2_T1, k.Nc * cfg.Nx
    rq.seed, rq.n_steps = seed, n_steps
    return rq


class Server:
    """Continuous-batching serving loop over the CUDA library (h1d_server_*)."""

    def __init__(self, path: str, hbm_budget_bytes: int, steps_per_tick: int = 64, sort_interval: int = 16):
        lib = self.lib = C.CDLL(os.path.abspath(path))
        v, u64 = C.c_void_p, C.c_uint64
        dp = C.POINTER(C.c_double)
        spec = {
            "h1d_server_create": ([C.c_size_t, C.c_int, C.POINTER(C.c_void_p)], C.c_int),
            "h1d_server_configure": ([v, C.c_int], C.c_int),
            "h1d_server_submit": ([v, C.POINTER(Request), C.POINTER(u64)], C.c_int),
            "h1d_server_tick": ([v, C.POINTER(C.c_int), C.POINTER(C.c_int)], C.c_int),
            "h1d_server_poll": ([v, u64, C.POINTER(C.c_int), dp, dp, dp], C.c_int),
            "h1d_server_result": ([v, u64, dp, dp, dp, dp, dp, dp], C.c_int),
            "h1d_server_release": ([v, u64], C.c_int),
            "h1d_server_stats_read": ([v, C.POINTER(ServerStats)], C.c_int),
            "h1d_server_destroy": ([v], C.c_int),
        }
        for name, (args, res) in spec.items():
            fn = getattr(lib, name)
            fn.argtypes, fn.restype = args, res
        h = C.c_void_p()
        st = lib.h1d_server_create(hbm_budget_bytes, steps_per_tick, C.byref(h))
        if st != OK:
            raise H1DError(st, "h1d_server_create failed")
        self.h = h
        self.cfgs = {}
        self._chk(lib.h1d_server_configure(h, sort_interval))

    def _chk(self, st, what="server call"):
        if st != OK:
            raise H1DError(st, what)

    def submit(self, cfg, seed: int, n_steps: int) -> int:
        rq = make_request(cfg, seed, n_steps)
        i = C.c_uint64()
        self._chk(self.lib.h1d_server_submit(self.h, C.byref(rq), C.byref(i)), "h1d_server_submit")
        self.cfgs[i.value] = cfg
        return i.value

    def tick(self):
        a, q = C.c_int(), C.c_int()
        self._chk(self.lib.h1d_server_tick(self.h, C.byref(a), C.byref(q)), "h1d_server_tick")
        return a.value, q.value

    def poll(self, rid: int):
        st, t0, t1, t2 = C.c_int(), C.c_double(), C.c_double(), C.c_double()
        rc = self.lib.h1d_server_poll(self.h, rid, C.byref(st), C.byref(t0), C.byref(t1), C.byref(t2))
        return dict(state=st.value, status=rc, t_submit=t0.value, t_admit=t1.value, t_done=t2.value)

    def result(self, rid: int):
        cfg = self.cfgs[rid]
        M = cfg.Nx + 2 * PAD
        nk, ns = len(cfg.kinetic), len(cfg.kinetic) + len(cfg.cold)
        B, E, en = np.empty((M, 3)), np.empty((M, 3)), np.empty(6 + 6 * ns)
        n, nV, nvv = np.empty((nk, M)), np.empty((nk, M, 3)), np.empty((nk, M, 6))
        self._chk(self.lib.h1d_server_result(self.h, rid, *[_ptr(a) for a in (B, E, en, n, nV, nvv)]),
                  "h1d_server_result")
        return dict(B=B, E=E, dB2O2=en[0:3], dE2O2=en[3:6], KE=en[6:].reshape(ns, 2, 3), n=n, nV=nV, nvv=nvv)

    def release(self, rid: int):
        self._chk(self.lib.h1d_server_release(self.h, rid), "h1d_server_release")
        self.cfgs.pop(rid, None)

    def stats(self):
        s = ServerStats()
        self._chk(self.lib.h1d_server_stats_read(self.h, C.byref(s)))
        return {k: getattr(s, k) for k, _ in ServerStats._fields_}

    def close(self):
        if getattr(self, "h", None):
            self.lib.h1d_server_destroy(self.h)
            self.h = None

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


# ---------------------------------------------------------------------------------------------
# checkpoint / resume (h1d_checkpoint_*) and velocity histograms (h1d_vhistogram)
# ---------------------------------------------------------------------------------------------

def _declare_ckpt(lib):
    v, sz = C.c_void_p, C.c_size_t
    spec = {
        "h1d_checkpoint_size": ([v, C.POINTER(sz)], C.c_int),
        "h1d_checkpoint_save": ([v, v, sz, C.POINTER(sz)], C.c_int),
        "h1d_checkpoint_load": ([v, v, sz], C.c_int),
        "h1d_step_count": ([v, C.POINTER(C.c_int64)], C.c_int),
    }
    for name, (args, res) in spec.items():
        fn = getattr(lib, name)
        fn.argtypes, fn.restype = args, res
    return lib


def checkpoint(run: Run) -> bytes:
    """The run's state as a byte image (h1d_checkpoint_save)."""
    lib = _declare_ckpt(run.lib)
    n = C.c_size_t()
    run._check(lib.h1d_checkpoint_size(run.h, C.byref(n)))
    buf = C.create_string_buffer(n.value)
    w = C.c_size_t()
    run._check(lib.h1d_checkpoint_save(run.h, buf, n.value, C.byref(w)))
    return buf.raw[:w.value]


def restore(run: Run, image: bytes):
    """Resume the run from a byte image of a run with the same parameters (h1d_checkpoint_load)."""
    lib = _declare_ckpt(run.lib)
    run._check(lib.h1d_checkpoint_load(run.h, image, len(image)))


def step_count(run: Run) -> int:
    lib = _declare_ckpt(run.lib)
    n = C.c_int64()
    run._check(lib.h1d_step_count(run.h, C.byref(n)))
    return n.value


def trim_device_memory(path: str, keep_bytes: int = 0) -> int:
    """Return the library's unused pooled device memory on the current device to the driver,
    keeping at most `keep_bytes` (h1d_trim_device_memory); returns the bytes the pool still holds."""
    lib = C.CDLL(path)
    fn = lib.h1d_trim_device_memory
    fn.argtypes, fn.restype = [C.c_size_t, C.POINTER(C.c_size_t)], C.c_int
    held = C.c_size_t()
    rc = fn(keep_bytes, C.byref(held))
    if rc != 0:
        raise H1DError(rc, "h1d_trim_device_memory failed")
    return held.value


def vhistogram(run: Run, s: int, extent, v1, v2, prefix: str = "h1d_"):
    """VHistogramRecorder of kinetic species s: extent = (loc, len) in q1, v1 = (min, len, bins)
    for the parallel and v2 = (min, len, bins) for the perpendicular speed.  Returns (hist, total)
    with hist[i1, i2] = (marker count, weight, real_f/marker) / total.  Works on either library
    (h1d_ or the oracle's orc_ prefix)."""
    fn = getattr(run.lib, prefix + "vhistogram")
    fn.argtypes = [C.c_void_p, C.c_int, C.c_double, C.c_double, C.c_double, C.c_double, C.c_int64, C.c_double,
                   C.c_double, C.c_int64, _dp, C.POINTER(C.c_int64)]
    fn.restype = C.c_int
    out = np.empty((int(v1[2]), int(v2[2]), 3))
    tot = C.c_int64()
    run._check(fn(run.h, s, extent[0], extent[1], v1[0], v1[1], int(v1[2]), v2[0], v2[1], int(v2[2]), _ptr(out),
                  C.byref(tot)))
    return out, tot.value
