"""Write an ``Inputs.h`` for the reference build of one run configuration.

TEST INFRASTRUCTURE: the reference (kyungguk1/hybrid_code-hfemic_wave) takes its parameters
as compile-time constants of ``struct Input`` (src/hybrid_1d/Include/Inputs.h), so the
reference build under oracle/_ref/ is compiled once per configuration.  The header written
here holds the same numbers the CUDA library and the C oracle receive at runtime, printed
with ``repr`` so that the C++ literal parses back to the identical double.

Single process, single subdomain, no worker threads; gyro-phase
randomisation of reflected particles is off (the reference seeds it from
std::random_device, Boundary/Delegate.cc:148).

usage: python oracle/ref/gen_inputs.py <config-name> <out-dir>
"""
import importlib.util
import os
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))


def _configs():
    path = os.path.join(ROOT, "hybrid_code-hfemic_wave_b200", "configs.py")
    spec = importlib.util.spec_from_file_location("_h1d_configs", path)
    mod = importlib.util.module_from_spec(spec)
    sys.modules["_h1d_configs"] = mod
    spec.loader.exec_module(mod)
    return mod


SHAPE = {1: "CIC", 2: "TSC", 3: "_3rd"}


def render(cfg) -> str:
    C = _configs()
    r = repr
    algo = "CAMCL" if cfg.algorithm == C.ALGO_CAMCL else "PC"
    if cfg.particle_bc == C.BC_PERIODIC:
        bc = "BC::periodic"
    elif cfg.particle_bc == C.BC_REFLECTING:
        bc = "BC::reflecting"
    else:
        raise SystemExit("the reference has no absorbing particle boundary")
    closure = "isothermal" if cfg.efluid.closure == C.ISOTHERMAL else "adiabatic"
    def kdesc(k):
        scheme = "delta_f" if k.scheme == C.DELTA_F else "full_f"
        base = (f"{{ {{ {r(k.Oc)}, {r(k.op)}, {k.n_smooth} }}, {k.Nc}, {SHAPE[k.shape_order]}, "
                f"{r(float(k.psd_refresh_frequency))}, {scheme}, {r(float(k.initial_weight))}, "
                f"{r(float(k.marker_temp_ratio))} }}")
        bimax = f"BiMaxPlasmaDesc({base}, {r(k.beta1)}, {r(k.T2_T1)})"
        if k.vdf == C.VDF_LOSSCONE:  # PlasmaDesc.h:244-250
            return f"LossconePlasmaDesc({{ {r(k.losscone_beta)} }}, {bimax})"
        if k.vdf == C.VDF_PARTIAL_SHELL:  # PlasmaDesc.h:290-305
            return f"PartialShellPlasmaDesc(KineticPlasmaDesc{base}, {r(k.beta1)}, {int(k.zeta)}U, {r(k.vs)})"
        if k.vdf == C.VDF_COUNTER_BEAM:  # PlasmaDesc.h:326-340
            return f"CounterBeamPlasmaDesc(KineticPlasmaDesc{base}, {r(k.beta1)}, {r(k.nu)}, {r(k.vs)})"
        return bimax

    kin = ",\n        ".join(kdesc(k) for k in cfg.kinetic)
    cold = ",\n        ".join(f"ColdPlasmaDesc({{ {r(c.Oc)}, {r(c.op)}, {c.n_smooth} }})" for c in cfg.cold)
    def cplx(z):
        z = complex(z)
        return f"std::complex<double>{{ {r(z.real)}, {r(z.imag)} }}"

    srcs = []
    for src in cfg.sources:
        n = len(src.points)
        J0 = ", ".join(f"ComplexVector{{ {cplx(J[0])}, {cplx(J[1])}, {cplx(J[2])} }}" for _, J in src.points)
        pos = ", ".join(f"CurviCoord{{ {r(q1)} }}" for q1, _ in src.points)
        srcs.append(f"ExternalSourceDesc<{n}>{{ ExternalSourceBase{{ {r(src.omega)}, Range{{ {r(src.start)}, {r(src.duration)} }}, "
                    f"ExternalSourceBase::EasePhase{{ {r(src.ease_in)}, {r(src.ease_out)} }}, {src.n_smooth} }}, "
                    f"{{ {J0} }}, {{ {pos} }} }}")
    sources = ",\n        ".join(srcs)
    pr, ad = cfg.phase_retardation, cfg.amplitude_damping
    nk = len(cfg.kinetic)
    ndumps = ", ".join(["0"] * nk)
    vh = ", ".join(["std::make_pair(Range{ -1, 2 }, 0U)"] * nk)
    return f"""// generated by oracle/ref/gen_inputs.py for configuration "{cfg.name}"
struct Input {{
    static constexpr unsigned number_of_ghost_cells = 3;
    static constexpr unsigned number_of_subdomains = 1;
    static constexpr unsigned number_of_distributed_particle_subdomain_clones = 1;
    static constexpr unsigned number_of_worker_threads = 0;
    static constexpr Algorithm algorithm = {algo};
    static constexpr unsigned n_subcycles = {cfg.n_subcycles};
    static constexpr BC particle_boundary_condition = {bc};
    static constexpr bool should_randomize_gyrophase_of_reflecting_particles = false;
    static constexpr MaskingFunction phase_retardation{{ {pr[0]}, {r(float(pr[1]))} }};
    static constexpr MaskingFunction amplitude_damping{{ {ad[0]}, {r(float(ad[1]))} }};
    static constexpr Real c = {r(cfg.c)};
    static constexpr Real O0 = {r(cfg.O0)};
    static constexpr Real xi = {r(cfg.xi)};
    static constexpr Real Dx = {r(cfg.Dx)};
    static constexpr unsigned Nx = {cfg.Nx};
    static constexpr Real dt = {r(cfg.dt)};
    static constexpr unsigned inner_Nt = {cfg.inner_Nt};
    static constexpr unsigned outer_Nt = 1;
    static constexpr auto efluid_desc = eFluidDesc({{ {r(cfg.efluid.Oc)}, {r(cfg.efluid.op)} }}, {r(cfg.efluid.beta)}, {closure});
    static constexpr auto part_descs = std::make_tuple(
        {kin});
    static constexpr auto cold_descs = std::make_tuple(
        {cold});
    static constexpr auto source_descs = std::make_tuple(
        {sources});
    static constexpr std::string_view working_directory = "./data";
    static constexpr std::pair<unsigned, Range> energy_recording_frequency = {{ 0, {{}} }};
    static constexpr std::pair<unsigned, Range> field_recording_frequency = {{ 0, {{}} }};
    static constexpr std::pair<unsigned, Range> moment_recording_frequency = {{ 0, {{}} }};
    static constexpr std::pair<unsigned, Range> particle_recording_frequency = {{ 0, {{}} }};
    static constexpr Range particle_recording_domain_extent = Range{{ -0.5 * Real{{ Nx }}, Nx }};
    static constexpr std::array<unsigned, std::tuple_size_v<decltype(part_descs)>> Ndumps = {{ {ndumps} }};
    static constexpr std::pair<unsigned, Range> vhistogram_recording_frequency = {{ 0, {{}} }};
    static constexpr Range vhistogram_recording_domain_extent = Range{{ -0.5 * Real{{ Nx }}, Nx }};
    static constexpr std::array<std::pair<Range, unsigned>, std::tuple_size_v<decltype(part_descs)>> v1hist_specs = {{ {vh} }};
    static constexpr std::array<std::pair<Range, unsigned>, std::tuple_size_v<decltype(part_descs)>> v2hist_specs = {{ {vh} }};
}};

namespace Debug {{
constexpr bool zero_out_electromagnetic_field = false;
constexpr Real initial_bfield_noise_amplitude = 0e0;
constexpr bool should_use_unified_snapshot    = false;
}} // namespace Debug
"""


def main(argv):
    if len(argv) != 3:
        raise SystemExit(__doc__)
    C = _configs()
    table = {**C.PARITY, **C.PRESETS}
    cfg = table[argv[1]]()
    os.makedirs(argv[2], exist_ok=True)
    with open(os.path.join(argv[2], "Inputs.h"), "w") as f:
        f.write(render(cfg))


if __name__ == "__main__":
    main(sys.argv)
