/*
 * Domain_GPU.cc -- the drop-in GPU Domain (Domain_GPU.h) over the C ABI of libh1d_gpu.so.
 */
#include "Domain_GPU.h"

#include <cmath>
#include <complex>
#include <random>
#include <stdexcept>
#include <string>
#include <tuple>
#include <type_traits>
#include <utility>

HYBRID1D_BEGIN_NAMESPACE
namespace {
template <class T, long N>
double *raw(GridArray<T, N, Pad> &g) noexcept
{
    return reinterpret_cast<double *>(g.dead_begin());
}
template <class T, long N>
double const *raw(GridArray<T, N, Pad> const &g) noexcept
{
    return reinterpret_cast<double const *>(g.dead_begin());
}

// the equilibrium distribution of a kinetic species' descriptor type (the VDFVariant alternative
// VDFVariant::make picks for it, LibPIC/PIC/VDFVariant.h:55-88) and its parameters
template <class Desc>
void set_vdf(h1d_kinetic_desc &k, Desc const &desc, Real c)
{
    auto const vth = [&](Real beta) { return std::sqrt(beta) * c * std::abs(desc.Oc) / desc.op; };
    if constexpr (std::is_base_of_v<LossconePlasmaDesc, Desc>) { // LossconeVDF.cc:22-44
        k.vdf          = H1D_VDF_LOSSCONE;
        k.vth1         = vth(desc.beta1);
        k.T2_T1        = desc.T2_T1;
        k.vdf_param[0] = desc.losscone.beta;
    } else if constexpr (std::is_base_of_v<BiMaxPlasmaDesc, Desc>) { // MaxwellianVDF.cc:21-31
        k.vdf   = H1D_VDF_BIMAXWELLIAN;
        k.vth1  = vth(desc.beta1);
        k.T2_T1 = desc.T2_T1;
    } else if constexpr (std::is_base_of_v<PartialShellPlasmaDesc, Desc>) { // PartialShellVDF.cc:24-77
        k.vdf          = H1D_VDF_PARTIAL_SHELL;
        k.vth1         = vth(desc.beta);
        k.vdf_param[0] = desc.zeta;
        k.vdf_param[1] = desc.vs;
    } else if constexpr (std::is_base_of_v<CounterBeamPlasmaDesc, Desc>) { // CounterBeamVDF.cc:36-74
        k.vdf          = H1D_VDF_COUNTER_BEAM;
        k.vth1         = vth(desc.beta);
        k.vdf_param[0] = desc.nu;
        k.vdf_param[1] = desc.vs;
    } else { // test particles: zero weights that never change (TestParticleVDF.cc)
        k.vdf  = H1D_VDF_BIMAXWELLIAN;
        k.vth1 = 1;
    }
}

template <class Desc>
h1d_kinetic_desc kinetic_of(ParamSet const &params, Desc const &desc)
{
    h1d_kinetic_desc k{};
    k.Oc          = desc.Oc;
    k.op          = desc.op;
    k.n_smooth    = desc.number_of_source_smoothings;
    k.Nc          = desc.Nc;
    k.shape_order = static_cast<long>(desc.shape_order);
    // PartSpecies::Nc, the reference cell's particle count (Core/PartSpecies.cc:45-49)
    auto const vdf = VDFVariant::make(desc, params.geomtr, params.full_grid_whole_domain_extent, params.c);
    if (long const Np = params.Nx * desc.Nc)
        k.moment_norm = Np * vdf->Nrefcell_div_Ntotal();
    else
        k.moment_norm = 1;
    k.scheme                = desc.scheme == delta_f ? H1D_DELTA_F : H1D_FULL_F;
    k.psd_refresh_frequency = desc.should_refresh_psd ? desc.psd_refresh_frequency : 0.0;
    set_vdf(k, desc, params.c);
    return k;
}

template <unsigned N>
h1d_source_desc source_of(ExternalSourceDesc<N> const &desc)
{
    static_assert(N <= H1D_MAX_SOURCE_POINTS, "too many source points for the GPU library");
    h1d_source_desc s{};
    s.omega    = desc.omega;
    s.start    = desc.extent.loc;
    s.duration = desc.extent.len;
    s.ease_in  = desc.ease.in;
    s.ease_out = desc.ease.out;
    s.n_smooth = desc.number_of_source_smoothings;
    s.n_points = N;
    for (unsigned j = 0; j < N; ++j) {
        s.pos[j] = desc.pos[j].q1;
        std::complex<double> const J[3] = { desc.J0[j].x, desc.J0[j].y, desc.J0[j].z };
        for (int c = 0; c < 3; ++c) {
            s.J0re[j][c] = J[c].real();
            s.J0im[j][c] = J[c].imag();
        }
    }
    return s;
}

bool evolves_weights(PartSpecies const &sp) { return sp->scheme == delta_f || sp->should_refresh_psd; }
} // namespace

h1d_params h1d_params_of(ParamSet const &params, int algorithm, int precision)
{
    static_assert(ParamSet::number_of_subdomains == 1 && ParamSet::number_of_distributed_particle_subdomain_clones == 1,
                  "one GPU holds the whole field line: one subdomain, one particle clone");
    static_assert(std::tuple_size_v<decltype(params.part_descs)> <= H1D_MAX_KINETIC, "too many kinetic species");
    static_assert(std::tuple_size_v<decltype(params.cold_descs)> <= H1D_MAX_COLD, "too many cold species");
    static_assert(std::tuple_size_v<decltype(params.source_descs)> <= H1D_MAX_SOURCES, "too many external sources");
    h1d_params h{};
    h.Nx                       = params.Nx;
    h.Dx                       = params.Dx;
    h.xi                       = params.xi;
    h.O0                       = params.O0;
    h.c                        = params.c;
    h.dt                       = params.dt;
    h.n_subcycles              = params.n_subcycles;
    h.algorithm                = algorithm;
    h.particle_bc              = static_cast<int>(params.particle_boundary_condition); // same enum values
    h.randomize_gyrophase      = params.should_randomize_gyrophase_of_reflecting_particles;
    h.gyrophase_seed           = std::random_device{}(); // as Delegate.cc:148 seeds its generator
    h.precision                = precision;
    h.phase_retardation_inset  = params.phase_retardation.masking_inset;
    h.phase_retardation_factor = params.phase_retardation.masking_factor;
    h.amplitude_damping_inset  = params.amplitude_damping.masking_inset;
    h.amplitude_damping_factor = params.amplitude_damping.masking_factor;
    h.moment_weighting         = 1.0 / params.number_of_distributed_particle_subdomain_clones; // Species.cc:16
    h.efluid                   = { params.efluid_desc.Oc, params.efluid_desc.op, params.efluid_desc.beta,
                                   params.efluid_desc.gamma };
    std::apply([&](auto const &...d) { h.n_kinetic = 0, ((h.kinetic[h.n_kinetic++] = kinetic_of(params, d)), ...); },
               params.part_descs);
    std::apply([&](auto const &...d) { h.n_cold = 0, ((h.cold[h.n_cold++] = { d.Oc, d.op, d.number_of_source_smoothings }), ...); },
               params.cold_descs);
    std::apply([&](auto const &...d) { h.n_sources = 0, ((h.sources[h.n_sources++] = source_of(d)), ...); },
               params.source_descs);
    return h;
}

Domain_GPU::Domain_GPU(ParamSet const &params, Delegate *delegate, int algorithm, int precision)
: Domain{ params, delegate }, m_precision{ precision }, m_uploaded(part_species.size())
{
    h1d_params const hp = h1d_params_of(params, algorithm, precision);
    if (int const st = h1d_create(&hp, &m_run))
        throw std::invalid_argument{ std::string{ __PRETTY_FUNCTION__ } + " - h1d_create: " + h1d_error_name(st) };
}
Domain_GPU::~Domain_GPU()
{
    h1d_destroy(m_run);
}

void Domain_GPU::check(int const status, char const *what) const
{
    if (status == H1D_OK)
        return;
    std::string const msg = std::string{ what } + " - " + h1d_status_string(m_run);
    if (status == H1D_ERR_MOVED_TOO_FAR) // PartSpecies::update_pos (Core/PartSpecies.cc:113)
        throw std::domain_error{ msg };
    if (status == H1D_ERR_INVALID_ARG)
        throw std::invalid_argument{ msg };
    throw std::runtime_error{ msg + " (" + h1d_error_name(status) + ")" };
}

void Domain_GPU::upload()
{
    for (unsigned s = 0; s < part_species.size(); ++s) {
        PartSpecies const  &sp = part_species[s];
        std::size_t const   n  = sp.bucket.size();
        std::vector<double> q1(n), vx(n), vy(n), vz(n), w(n);
        Uploaded           &up = m_uploaded[s];
        up.id.resize(n), up.real_f.resize(n), up.marker.resize(n);
        std::size_t k = 0;
        for (Particle const &ptl : sp.bucket) { // structure of arrays from the deque (PartSpecies.h:33-34)
            q1[k] = ptl.pos.q1, vx[k] = ptl.vel.x, vy[k] = ptl.vel.y, vz[k] = ptl.vel.z, w[k] = ptl.psd.weight;
            up.id[k] = ptl.id, up.real_f[k] = ptl.psd.real_f, up.marker[k] = ptl.psd.marker;
            ++k;
        }
        check(h1d_upload_particles(m_run, static_cast<int>(s), static_cast<int64_t>(n), q1.data(), vx.data(),
                                   vy.data(), vz.data(), w.data()),
              "h1d_upload_particles");
        if (evolves_weights(sp))
            check(h1d_upload_psd(m_run, static_cast<int>(s), static_cast<int64_t>(n), up.real_f.data(), up.marker.data()),
                  "h1d_upload_psd");
    }
    check(h1d_upload_fields(m_run, raw(bfield), raw(efield)), "h1d_upload_fields");
    for (unsigned i = 0; i < cold_species.size(); ++i)
        check(h1d_upload_cold(m_run, static_cast<int>(i), raw(cold_species[i].mom0_full), raw(cold_species[i].mom1_full)),
              "h1d_upload_cold");
    m_on_device = true;
}

void Domain_GPU::download_recorded()
{
    // the post-process of advance_by (Domain_CAMCL.cc:45-55, Domain_PC.cc:67-77): what recorders read
    check(h1d_download_fields(m_run, raw(bfield), raw(efield)), "h1d_download_fields");
    check(h1d_download_sources(m_run, raw(charge), raw(current)), "h1d_download_sources");
    for (unsigned s = 0; s < part_species.size(); ++s) {
        PartSpecies &sp = part_species[s];
        check(h1d_download_moments(m_run, static_cast<int>(s), raw(sp.moment<0>()), raw(sp.moment<1>()), raw(sp.moment<2>())),
              "h1d_download_moments");
    }
    for (unsigned i = 0; i < cold_species.size(); ++i) {
        ColdSpecies &sp = cold_species[i];
        check(h1d_download_cold(m_run, static_cast<int>(i), raw(sp.moment<0>()), raw(sp.moment<1>()), raw(sp.moment<2>()),
                                raw(sp.mom0_full), raw(sp.mom1_full)),
              "h1d_download_cold");
    }
}

void Domain_GPU::advance_by(unsigned const n_steps)
{
    if (!m_on_device)
        upload();
    check(h1d_advance(m_run, n_steps), __PRETTY_FUNCTION__);
    download_recorded();
}

void Domain_GPU::sync_particles()
{
    if (!m_on_device)
        return; // the host copy is current
    for (unsigned s = 0; s < part_species.size(); ++s) {
        PartSpecies &sp = part_species[s];
        int64_t      n  = 0;
        check(h1d_particle_count(m_run, static_cast<int>(s), &n), "h1d_particle_count");
        std::vector<double>  q1(n), vx(n), vy(n), vz(n), w(n), real_f, marker;
        std::vector<int64_t> pid(n);
        check(h1d_download_particles(m_run, static_cast<int>(s), q1.data(), vx.data(), vy.data(), vz.data(), w.data(),
                                     pid.data()),
              "h1d_download_particles");
        bool const evolving = evolves_weights(sp);
        if (evolving) {
            real_f.resize(n), marker.resize(n);
            check(h1d_download_psd(m_run, static_cast<int>(s), real_f.data(), marker.data()), "h1d_download_psd");
        }
        Uploaded const &up = m_uploaded[s];
        sp.bucket.clear();
        for (int64_t k = 0; k < n; ++k) {
            auto const i = static_cast<std::size_t>(pid[k]);
            Particle   ptl;
            ptl.vel = CartVector{ vx[k], vy[k], vz[k] };
            ptl.pos = CurviCoord{ q1[k] };
            ptl.psd = Particle::PSD{ w[k], evolving ? real_f[k] : up.real_f[i], evolving ? marker[k] : up.marker[i] };
            ptl.id  = up.id[i];
            sp.bucket.push_back(ptl);
        }
    }
}

Domain_CAMCL_GPU::Domain_CAMCL_GPU(ParamSet const &params, Delegate *delegate, int precision)
: Domain_GPU{ params, delegate, H1D_ALGO_CAMCL, precision }
{
}
Domain_PC_GPU::Domain_PC_GPU(ParamSet const &params, Delegate *delegate, int precision)
: Domain_GPU{ params, delegate, H1D_ALGO_PC, precision }
{
}
HYBRID1D_END_NAMESPACE
