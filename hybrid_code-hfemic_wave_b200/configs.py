"""Run descriptions for the hybrid_1d hot path.

The reference fixes every parameter at compile time in ``struct Input``
(src/hybrid_1d/Include/Inputs.h:13-241).  Here a run is described at runtime by
:class:`RunConfig`, which maps field-for-field onto that struct and onto the C struct
``h1d_params`` of include/h1d_gpu.h.

Species are given in physical terms (density fraction ``f``, charge number ``Z``, mass
number ``A``) and converted with the reference's own normalisation: O0 = 1 (proton
cyclotron frequency), ``c`` = c/vA, so a species has ``Oc = Z/A`` and
``op = c*sqrt(f*Z**2/A)``; the electron fluid is ``eFluidDesc({-1836, c*sqrt(1836*ne)}, beta_e,
closure)`` with ``ne = sum(f*Z)``.  The thermal speed of a bi-Maxwellian is
``vth1 = sqrt(beta1)*c*|Oc|/op`` (src/LibPIC/PIC/VDF/MaxwellianVDF.cc:24).
"""
from __future__ import annotations

import dataclasses
import math
from dataclasses import dataclass, field
from typing import List

ALGO_PC, ALGO_CAMCL = 0, 1
BC_PERIODIC, BC_REFLECTING, BC_ABSORBING = 0, 1, 2
PREC_FP64, PREC_MIXED = 0, 1
ISOTHERMAL, ADIABATIC = 11, 53  # Closure (src/LibPIC/PIC/Predefined.h:42-45)
FULL_F, DELTA_F = 0, 1  # ParticleScheme (src/LibPIC/PIC/Predefined.h)
# the equilibrium distribution of a kinetic species (VDFVariant, src/LibPIC/PIC/VDFVariant.h)
VDF_BIMAXWELLIAN, VDF_LOSSCONE, VDF_PARTIAL_SHELL, VDF_COUNTER_BEAM = 0, 1, 2, 3


@dataclass
class Kinetic:
    """A kinetic species (KineticPlasmaDesc, PlasmaDesc.h:118-177) with its equilibrium
    distribution: bi-Maxwellian (BiMaxPlasmaDesc, :207-236, the default), loss-cone
    (LossconePlasmaDesc, :244-284: ``losscone_beta``; ``T2_T1`` is the BiMaxPlasmaDesc value),
    partial shell (PartialShellPlasmaDesc, :290-320: thermal spread ``beta1``, ``zeta``, ``vs``) or
    counter-beam (CounterBeamPlasmaDesc, :326-345: thermal spread ``beta1``, ``nu``, ``vs``)."""

    Oc: float
    op: float
    Nc: int  # particles per cell
    shape_order: int = 2
    n_smooth: int = 2
    beta1: float = 0.1  # parallel beta
    T2_T1: float = 1.0  # perpendicular / parallel temperature
    # phase-space density weighting (KineticPlasmaDesc, PlasmaDesc.h:118-160)
    scheme: int = FULL_F
    initial_weight: float = 0.0  # delta-f only: initial weights are initial_weight * U(-1, 1)
    marker_temp_ratio: float = 1.0  # marker temperature / physical temperature
    psd_refresh_frequency: float = 0.0  # nu: weights relax toward the equilibrium at this rate
    vdf: int = VDF_BIMAXWELLIAN
    losscone_beta: float = 0.0
    zeta: int = 0  # partial shell: sin^zeta pitch-angle exponent
    vs: float = 0.0  # partial shell, counter-beam: shell speed
    nu: float = 0.0  # counter-beam: pitch-angle width at the equator
    norm: float | None = None  # PartSpecies::Nc when given by the caller (else computed)

    def vdf_param(self):
        """h1d_kinetic_desc::vdf_param of this distribution."""
        if self.vdf == VDF_LOSSCONE:
            return (self.losscone_beta, 0.0, 0.0)
        if self.vdf == VDF_PARTIAL_SHELL:
            return (float(self.zeta), self.vs, 0.0)
        if self.vdf == VDF_COUNTER_BEAM:
            return (self.nu, self.vs, 0.0)
        return (0.0, 0.0, 0.0)

    def vth1(self, c: float) -> float:
        return math.sqrt(self.beta1) * c * abs(self.Oc) / self.op

    @property
    def has_psd(self) -> bool:
        """Whether the particles carry a phase-space density that changes in time (delta-f, or
        full-f with PSD refresh): their weights are then updated every step."""
        return self.scheme == DELTA_F or self.psd_refresh_frequency != 0.0


@dataclass
class Cold:
    """A cold fluid species (ColdPlasmaDesc, PlasmaDesc.h:92-114)."""

    Oc: float
    op: float
    n_smooth: int = 2


@dataclass
class EFluid:
    """Charge-neutralising massless electron fluid (eFluidDesc, PlasmaDesc.h:66-88)."""

    Oc: float
    op: float
    beta: float = 0.0
    closure: int = ISOTHERMAL

    @property
    def gamma(self) -> float:
        # gamma(closure / 10) with integer division, then gamma /= closure % 10
        return float(self.closure // 10) / float(self.closure % 10)


@dataclass
class Source:
    """An external current source (ExternalSourceDesc<N>, PlasmaDesc.h:363-437): angular frequency,
    time extent (start, duration) without the ease phases, ease-in/-out durations, smoothing count,
    and source points (q1, (J0x, J0y, J0z)) with complex field-aligned amplitudes."""

    omega: float
    start: float
    duration: float
    ease_in: float
    ease_out: float
    points: list
    n_smooth: int = 0


@dataclass
class RunConfig:
    name: str
    Nx: int
    Dx: float
    xi: float
    c: float
    dt: float
    efluid: EFluid
    kinetic: List[Kinetic] = field(default_factory=list)
    cold: List[Cold] = field(default_factory=list)
    sources: List[Source] = field(default_factory=list)
    O0: float = 1.0
    n_subcycles: int = 10
    algorithm: int = ALGO_CAMCL
    particle_bc: int = BC_PERIODIC
    randomize_gyrophase: bool = False
    gyrophase_seed: int = 0
    phase_retardation: tuple = (0, 0.0)
    amplitude_damping: tuple = (0, 0.0)
    precision: int = PREC_FP64
    sort_interval: int = 0
    steps: int = 1  # run length the preset is quoted on
    inner_Nt: int = 10  # Input::inner_Nt

    def replace(self, **kw) -> "RunConfig":
        return dataclasses.replace(self, **kw)

    @property
    def has_psd(self) -> bool:
        return any(k.has_psd for k in self.kinetic)

    @property
    def n_particles(self) -> int:
        return sum(k.Nc * self.Nx for k in self.kinetic)

    # ----- extents (ParamSet.cc:20-23) -----
    @property
    def q1min(self) -> float:
        return -0.5 * self.Nx

    @property
    def q1max(self) -> float:
        return -0.5 * self.Nx + self.Nx

    @property
    def homogeneous(self) -> bool:
        return self.xi < 1e-10  # MirrorGeometry.h:19, MirrorGeometry.cc:20

    def moment_norm(self, k: Kinetic) -> float:
        """PartSpecies::Nc = Nx*Nc*Nrefcell_div_Ntotal (PartSpecies.cc:45-49), with the
        distribution's N_of_q1 (MaxwellianVDF.cc:28-30, 44-54, LossconeVDF.cc:37-39, 71-88,
        PartialShellVDF.cc:84-93); ``k.norm`` when the caller gives it."""
        if k.norm is not None:
            return k.norm
        if self.Nx * k.Nc == 0:
            return 1.0
        return self.Nx * k.Nc * nrefcell_div_ntotal(self, k)

    def validate(self) -> None:
        """The static checks of InputWrapper.h:132-155 and ParamSet.cc:25-29."""
        if self.Nx < 6:
            raise ValueError("Nx must be at least 2*number_of_ghost_cells")
        if self.n_subcycles < 2:
            raise ValueError("number of subcyclings should be at least 2")
        for inset, _ in (self.phase_retardation, self.amplitude_damping):
            if inset > self.Nx // 2:
                raise ValueError("masking inset is greater than half the domain length")
        if self.xi > 0:
            for q1 in (self.q1min, self.q1max, self.q1min + 0.5, self.q1max + 0.5):
                if not abs(self.xi * self.Dx * q1) < math.pi / 2:
                    raise ValueError("invalid domain extent: |xi*D1*q1| >= pi/2")


def position_fraction_bits(Nx: int) -> int:
    """Fraction bits F of the mixed-precision fixed-point position (an int32 holding
    (q1 - q1min) 2^F): the most bits, at most FP32's 24, that keep (Nx + 2) 2^F within 2^31.  A
    position is stored to the nearest 2^-F cell."""
    f = 24
    while f > 0 and (Nx + 2) << f > 1 << 31:
        f -= 1
    return f


def _int_cos_zeta(zeta: int, a: float, x: float, small_a: bool) -> float:
    """int_0^x cos^zeta(a t) dt by the recurrence of VDFHelper.h:125-147 (zeta - 2 -> zeta)."""
    ax = a * x
    if zeta == 0:
        return x
    if zeta == 1:
        return (1 - ax * ax * 0.1666666666666666666666666666666666666667) * x if small_a else math.sin(ax) / a
    addendum = _int_cos_zeta(zeta - 2, a, x, small_a) * float(zeta - 1) / zeta
    if small_a:
        return (1 + ax * ax * 0.1666666666666666666666666666666666666667 * (2 - 3 * float(zeta))) * (x / zeta) + addendum
    return math.cos(ax) ** (zeta - 1) * math.sin(ax) / (zeta * a) + addendum


def _losscone_beta(k: Kinetic) -> float:
    b = k.losscone_beta
    if b < 1e-10:
        return 1e-10
    if abs(b - 1) < 1e-10:
        return b + math.copysign(1e-10, b - 1)
    return b


def _n_of_q1(cfg: RunConfig, k: Kinetic, q1: float) -> float:
    """N_of_q1 of the species' distribution: MaxwellianVDF.cc:44-54, LossconeVDF.cc:71-88,
    PartialShellVDF.cc:84-93; counter-beam: the integral of n0 by Gauss-Legendre quadrature
    (the reference integrates it numerically to about 1e-8, VDFHelper.h:47-70)."""
    if k.vdf == VDF_LOSSCONE:
        b = _losscone_beta(k)
        X = k.T2_T1 / (1 + b)
        if cfg.homogeneous:
            xiD1q1 = cfg.xi * cfg.Dx * q1
            t1 = 1 - (X - 1) / 3 * xiD1q1 * xiD1q1
            t2 = 1 - (b * X - 1) / 3 * xiD1q1 * xiD1q1
            return q1 * (t1 - b * t2) / (1 - b)
        sb, sx = math.sqrt(b), math.sqrt(X)
        tan = math.tan(cfg.xi * cfg.Dx * q1)
        t1 = math.atan(sx * tan) / (sx * cfg.Dx * cfg.xi)
        t2 = math.atan(sb * sx * tan) / (sb * sx * cfg.Dx * cfg.xi)
        return (t1 - b * t2) / (1 - b)
    if k.vdf == VDF_PARTIAL_SHELL:
        return _int_cos_zeta(k.zeta, cfg.xi, cfg.Dx * q1, cfg.homogeneous)
    if k.vdf == VDF_COUNTER_BEAM:
        import numpy as np
        t, w = np.polynomial.legendre.leggauss(64)
        q = 0.5 * q1 * (t + 1)
        nu = k.nu / np.cos(cfg.xi * cfg.Dx * q)
        bnu = 2 * nu * dawson(1 / nu)
        return float(0.5 * q1 * np.sum(w * bnu)) / (2 * k.nu * dawson(1 / k.nu))
    T2OT1 = k.T2_T1
    if cfg.homogeneous:
        xiD1q1 = cfg.xi * cfg.Dx * q1
        return q1 * (1 - (xiD1q1 * xiD1q1) * (T2OT1 - 1) / 3)
    s = math.sqrt(T2OT1)
    return math.atan(s * math.tan(cfg.xi * cfg.Dx * q1)) / (s * cfg.Dx * cfg.xi)


def _q1_of_n(cfg: RunConfig, k: Kinetic, N: float) -> float:
    """MaxwellianVDF::q1_of_N (MaxwellianVDF.cc:55-65)."""
    T2OT1 = k.T2_T1
    if cfg.homogeneous:
        xiD1N = cfg.xi * cfg.Dx * N
        return N * (1 + (xiD1N * xiD1N) * (T2OT1 - 1) / 3)
    s = math.sqrt(T2OT1)
    return math.atan(math.tan(s * cfg.Dx * cfg.xi * N) / s) / (cfg.xi * cfg.Dx)


def dawson(x):
    """Dawson's integral F(x) = exp(-x^2) int_0^x exp(t^2) dt of positive x (a float or an array):
    Maclaurin series below 0.2, Rybicki's sampling-theorem sum pi^-1/2 sum_{n odd}
    exp(-(x - 0.2 n)^2)/n up to 50 (G. B. Rybicki, Computers in Physics 3(2), 85 (1989)), the
    asymptotic series (1/2x) sum_k (2k-1)!!/(2x^2)^k beyond; relative error below 5e-15."""
    import numpy as np
    scalar = np.ndim(x) == 0
    x = np.atleast_1d(np.asarray(x, dtype=np.float64))
    out = np.empty_like(x)
    small, large = x < 0.2, x > 50
    mid = ~(small | large)
    if small.any():
        xs = x[small]
        t, acc = xs.copy(), xs.copy()
        for j in range(1, 40):
            t = t * (-2 * xs * xs / (2 * j + 1))
            acc += t
        out[small] = acc
    if large.any():
        xl = x[large]
        r = 1 / (2 * xl * xl)
        t, acc = np.ones_like(xl), np.ones_like(xl)
        for j in range(1, 12):
            t = t * ((2 * j - 1) * r)
            acc += t
        out[large] = acc / (2 * xl)
    if mid.any():
        xm = x[mid]
        lo = np.floor((xm - 7) / 0.2).astype(np.int64) | 1
        hi = np.ceil((xm + 7) / 0.2).astype(np.int64)
        acc = np.zeros_like(xm)
        for j in range(0, 80, 2):
            nn = lo + j
            acc += np.where(nn <= hi, np.exp(-(xm - nn * 0.2) ** 2) / nn, 0.0)
        out[mid] = acc / math.sqrt(math.pi)
    return float(out[0]) if scalar else out


def nrefcell_div_ntotal(cfg: RunConfig, k: Kinetic) -> float:
    loc = _n_of_q1(cfg, k, cfg.q1min)
    length = _n_of_q1(cfg, k, cfg.q1max) - loc
    return (_n_of_q1(cfg, k, +0.5) - _n_of_q1(cfg, k, -0.5)) / length


def plasma(c: float, species, cold_fraction: float, beta_e: float, closure=ISOTHERMAL,
           cold_smooth: int = 2):
    """Build (efluid, kinetic, cold) from physical fractions.

    ``species`` is a list of dicts with keys f, Z, A, Nc, shape_order, beta1, T2_T1, n_smooth.
    """
    kin = []
    ne = 0.0
    for s in species:
        Z, A, f = s.get("Z", 1.0), s.get("A", 1.0), s["f"]
        ne += f * Z
        kin.append(Kinetic(Oc=Z / A, op=c * math.sqrt(f * Z * Z / A), Nc=s["Nc"],
                           shape_order=s.get("shape_order", 2), n_smooth=s.get("n_smooth", 2),
                           beta1=s["beta1"], T2_T1=s.get("T2_T1", 1.0), scheme=s.get("scheme", FULL_F),
                           initial_weight=s.get("initial_weight", 0.0),
                           marker_temp_ratio=s.get("marker_temp_ratio", 1.0),
                           psd_refresh_frequency=s.get("psd_refresh_frequency", 0.0),
                           vdf=s.get("vdf", VDF_BIMAXWELLIAN), losscone_beta=s.get("losscone_beta", 0.0),
                           zeta=s.get("zeta", 0), vs=s.get("vs", 0.0), nu=s.get("nu", 0.0)))
    cold = []
    if cold_fraction > 0:
        ne += cold_fraction
        cold.append(Cold(Oc=1.0, op=c * math.sqrt(cold_fraction), n_smooth=cold_smooth))
    ef = EFluid(Oc=-1836.0, op=c * math.sqrt(1836.0 * ne), beta=beta_e, closure=closure)
    return ef, kin, cold


# ---------------------------------------------------------------------------------------------
# presets
# ---------------------------------------------------------------------------------------------

def config1() -> RunConfig:
    """Plain FP64, CPU-runnable: uniform B0, periodic, Nx=256, Dx=0.3, dt=0.02, 1000 steps,
    hot H+ (f=0.1, beta_par=0.1, T_perp/T_par=3, 100 ppc, CIC) + cold H+, beta_e=0.1, c/vA=100."""
    ef, kin, cold = plasma(100.0, [dict(f=0.1, Nc=100, shape_order=1, beta1=0.1, T2_T1=3.0)],
                           0.9, 0.1)
    return RunConfig("config1_cic_periodic_nx256", Nx=256, Dx=0.3, xi=0.0, c=100.0, dt=0.02,
                     efluid=ef, kinetic=kin, cold=cold, steps=1000)


def config2() -> RunConfig:
    """Plain FP64 GPU drop-in: mirror xi=0.002, Nx=2048, masking over 128 cells each end,
    hot H+ (beta 0.2, A 4, 10%) + hot He+ (beta 0.05, A 2, 5%), 1000 ppc each, TSC,
    dt=0.01, 5000 steps.  Particle boundary: reflecting (the reference has no absorbing BC)."""
    ef, kin, cold = plasma(100.0, [
        dict(f=0.10, Z=1, A=1, Nc=1000, shape_order=2, beta1=0.2, T2_T1=4.0),
        dict(f=0.05, Z=1, A=4, Nc=1000, shape_order=2, beta1=0.05, T2_T1=2.0),
    ], 0.85, 0.1)
    return RunConfig("config2_tsc_mirror_nx2048", Nx=2048, Dx=0.3, xi=0.002, c=100.0, dt=0.01,
                     efluid=ef, kinetic=kin, cold=cold, particle_bc=BC_REFLECTING,
                     phase_retardation=(128, 1.0), amplitude_damping=(128, 0.2), steps=5000)


def config3(precision=PREC_MIXED) -> RunConfig:
    """Config-1 plasma at Nx=4096 with 4000 particles per cell (one kinetic species:
    16.4M particles), 2000 steps."""
    ef, kin, cold = plasma(100.0, [dict(f=0.1, Nc=4000, shape_order=1, beta1=0.1, T2_T1=3.0)],
                           0.9, 0.1)
    return RunConfig("config3_cic_periodic_nx4096", Nx=4096, Dx=0.3, xi=0.0, c=100.0, dt=0.02,
                     efluid=ef, kinetic=kin, cold=cold, precision=precision, steps=2000)


# small cases the oracle finishes in seconds; each is also built against the reference
def parity_p1() -> RunConfig:
    ef, kin, cold = plasma(100.0, [dict(f=0.1, Nc=16, shape_order=1, beta1=0.1, T2_T1=3.0)], 0.9, 0.1)
    return RunConfig("p1_cic_periodic", Nx=32, Dx=0.3, xi=0.0, c=100.0, dt=0.02, efluid=ef,
                     kinetic=kin, cold=cold, steps=10)


def parity_p2() -> RunConfig:
    ef, kin, cold = plasma(100.0, [
        dict(f=0.10, Z=1, A=1, Nc=16, shape_order=2, beta1=0.2, T2_T1=4.0),
        dict(f=0.05, Z=1, A=4, Nc=12, shape_order=2, beta1=0.05, T2_T1=2.0),
    ], 0.85, 0.1)
    return RunConfig("p2_tsc_mirror_reflecting", Nx=64, Dx=0.3, xi=0.05, c=100.0, dt=0.01,
                     efluid=ef, kinetic=kin, cold=cold, particle_bc=BC_REFLECTING,
                     phase_retardation=(8, 1.0), amplitude_damping=(8, 0.2), steps=10)


def parity_p3() -> RunConfig:
    ef, kin, cold = plasma(100.0, [dict(f=0.2, Nc=20, shape_order=3, beta1=0.3, T2_T1=2.0,
                                        n_smooth=1)], 0.8, 0.2, closure=ADIABATIC, cold_smooth=1)
    return RunConfig("p3_o3_adiabatic_periodic", Nx=48, Dx=0.25, xi=0.0, c=50.0, dt=0.02,
                     efluid=ef, kinetic=kin, cold=cold, n_subcycles=4, steps=10)


def parity_p4() -> RunConfig:
    ef, kin, cold = plasma(100.0, [dict(f=0.1, Nc=16, shape_order=2, beta1=0.2, T2_T1=3.0)], 0.9, 0.1)
    return RunConfig("p4_pc_tsc_mirror_reflecting", Nx=64, Dx=0.3, xi=0.03, c=100.0, dt=0.01,
                     efluid=ef, kinetic=kin, cold=cold, algorithm=ALGO_PC,
                     particle_bc=BC_REFLECTING, phase_retardation=(6, 1.0),
                     amplitude_damping=(6, 0.2), steps=10)


def parity_p5() -> RunConfig:
    """The p2 plasma with an external current source whose ramps and flat top all fall within ten
    steps (t = 0.005 .. 0.095), at three points, one depositing into the last ghost cell (folded by the reflecting boundary)."""
    cfg = parity_p2()
    src = Source(omega=3.0, start=0.03, duration=0.03, ease_in=0.02, ease_out=0.025, n_smooth=1,
                 points=[(0.3, (0.5, 0.5j, 0.0)), (-20.25, (0.2 + 0.1j, -0.3j, 0.1)), (31.7, (0.0, 1.0, 1.0j))])
    return cfg.replace(name="p5_tsc_mirror_source", sources=[src])


def parity_p6() -> RunConfig:
    """The predictor-corrector case p4 with an external current source active from the first step."""
    cfg = parity_p4()
    src = Source(omega=2.0, start=0.0, duration=0.05, ease_in=0.0, ease_out=0.03, n_smooth=2,
                 points=[(1.7, (0.4j, 0.6, 0.0)), (30.9, (0.0, 0.3, -0.2j))])
    return cfg.replace(name="p6_pc_source", sources=[src])


def parity_p7() -> RunConfig:
    """Phase-space density weights in a mirror field (CAM-CL, reflecting): a delta-f H+ species
    (initial weights 0.1 U(-1, 1), PSD refresh at nu = 2) beside a full-f He+ species loaded with
    markers twice as hot as the plasma (weights f0/g0) and refreshed at nu = 5."""
    ef, kin, cold = plasma(100.0, [
        dict(f=0.10, Z=1, A=1, Nc=16, shape_order=2, beta1=0.2, T2_T1=4.0, scheme=DELTA_F, initial_weight=0.1,
             psd_refresh_frequency=2.0),
        dict(f=0.05, Z=1, A=4, Nc=12, shape_order=1, beta1=0.05, T2_T1=2.0, marker_temp_ratio=2.0,
             psd_refresh_frequency=5.0),
    ], 0.85, 0.1)
    return RunConfig("p7_psd_tsc_mirror_reflecting", Nx=64, Dx=0.3, xi=0.05, c=100.0, dt=0.01,
                     efluid=ef, kinetic=kin, cold=cold, particle_bc=BC_REFLECTING,
                     phase_retardation=(8, 1.0), amplitude_damping=(8, 0.2), steps=10)


def parity_p8() -> RunConfig:
    """p7 under the predictor-corrector cycle, periodic, with a delta-f species without refresh."""
    cfg = parity_p7()
    kin = [dataclasses.replace(k) for k in cfg.kinetic]
    kin[0].psd_refresh_frequency = 0.0
    kin[0].shape_order = 3
    return cfg.replace(name="p8_pc_psd_periodic", kinetic=kin, algorithm=ALGO_PC, particle_bc=BC_PERIODIC,
                       xi=0.03)


def parity_p9() -> RunConfig:
    """Delta-f loss-cone H+ (losscone beta 0.3, refreshed at nu = 2) beside a full-f loss-cone He+
    loaded with hot markers and refreshed, in a mirror field (CAM-CL, reflecting)."""
    cfg = parity_p7()
    kin = [dataclasses.replace(k, vdf=VDF_LOSSCONE) for k in cfg.kinetic]
    kin[0].losscone_beta, kin[0].T2_T1 = 0.3, 1.3 * 3.0
    kin[1].losscone_beta, kin[1].T2_T1 = 0.6, 1.6 * 1.5
    return cfg.replace(name="p9_losscone_psd_mirror", kinetic=kin)


def parity_p10() -> RunConfig:
    """Partial-shell species (sin^2 and isotropic shells, vs = 0.5 and 1 thermal speeds) with
    evolving weights under the predictor-corrector cycle in a mirror field, periodic."""
    cfg = parity_p7()
    kin = [dataclasses.replace(k, vdf=VDF_PARTIAL_SHELL) for k in cfg.kinetic]
    kin[0].zeta, kin[0].vs = 2, 0.5 * kin[0].vth1(cfg.c)
    kin[1].zeta, kin[1].vs = 0, 1.0 * kin[1].vth1(cfg.c)
    return cfg.replace(name="p10_pc_shell_psd_mirror", kinetic=kin, algorithm=ALGO_PC, particle_bc=BC_PERIODIC,
                       xi=0.03)


def parity_p11() -> RunConfig:
    """Counter-beam species (pitch-angle widths 0.5 and 1, vs = 0.3 thermal speeds) with evolving
    weights in a mirror field (CAM-CL, reflecting)."""
    cfg = parity_p7()
    kin = [dataclasses.replace(k, vdf=VDF_COUNTER_BEAM) for k in cfg.kinetic]
    kin[0].nu, kin[0].vs = 0.5, 0.3 * kin[0].vth1(cfg.c)
    kin[1].nu, kin[1].vs = 1.0, 0.3 * kin[1].vth1(cfg.c)
    return cfg.replace(name="p11_counterbeam_psd_mirror", kinetic=kin)


PARITY = {f().name: f for f in (parity_p1, parity_p2, parity_p3, parity_p4, parity_p5, parity_p6, parity_p7,
                                parity_p8, parity_p9, parity_p10, parity_p11)}
# parity cases whose equilibrium needs Dawson's integral, which the reference evaluates with its
# own implementation: their oracle agrees with the reference to rounding, not bit for bit
PARITY_ROUNDING = {"p11_counterbeam_psd_mirror"}
PRESETS = {f().name: f for f in (config1, config2, config3)}


# ---------------------------------------------------------------------------------------------
# ensemble members: seeded draws of the ensemble distribution
# ---------------------------------------------------------------------------------------------

ENSEMBLE_NX = (256, 512, 1024, 2048, 4096)


def ensemble_member(seed: int, precision=PREC_MIXED, steps: int = 500, ppc_scale: float = 1.0) -> RunConfig:
    """One member of the ensemble workload, drawn from a generator seeded with ``seed``: Nx uniform
    over ENSEMBLE_NX, particles per cell log-uniform in [100, 2000], T_perp/T_par uniform in
    [1.5, 5], beta_par log-uniform in [0.01, 0.5], xi uniform in [0, 0.004] (redrawn until
    |xi*Dx*q1| < pi/2 holds on the grid), TSC.  The plasma is that of config1 (one hot H+ species
    at 10 % density, cold H+ background, isothermal electrons with beta_e 0.1, c/vA = 100) with
    Dx = 0.3, dt = 0.01, reflecting particles and masking over Nx/16 cells at each end.
    ``ppc_scale`` shrinks the particle count for tests."""
    import numpy as np

    rng = np.random.default_rng(seed)
    Nx = int(rng.choice(ENSEMBLE_NX))
    Nc = max(1, int(round(math.exp(rng.uniform(math.log(100), math.log(2000))) * ppc_scale)))
    T2_T1 = float(rng.uniform(1.5, 5.0))
    beta1 = float(math.exp(rng.uniform(math.log(0.01), math.log(0.5))))
    Dx = 0.3
    while True:
        xi = float(rng.uniform(0.0, 0.004))
        if abs(xi * Dx * (0.5 * Nx + 0.5)) < math.pi / 2 * 0.999:
            break
    ef, kin, cold = plasma(100.0, [dict(f=0.1, Nc=Nc, shape_order=2, beta1=beta1, T2_T1=T2_T1)], 0.9, 0.1)
    inset = Nx // 16
    return RunConfig(f"ensemble_{seed}", Nx=Nx, Dx=Dx, xi=xi, c=100.0, dt=0.01, efluid=ef, kinetic=kin, cold=cold,
                     particle_bc=BC_REFLECTING, phase_retardation=(inset, 1.0), amplitude_damping=(inset, 0.2),
                     precision=precision, steps=steps)
