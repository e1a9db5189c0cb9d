// TEST INFRASTRUCTURE: a driver around the UNMODIFIED reference hot path
// (src/hybrid_1d/Core/*.cc, Boundary/Delegate.cc, ParamSet.cc, src/LibPIC/PIC/*.cc of
// kyungguk1/hybrid_code-hfemic_wave), compiled in place from the reference tree by
// oracle/Makefile.  It replaces what cannot be compiled here (MPI/ParallelKit delegates,
// HDF5 recorders, Driver.cc) with:
//   - SerialDelegate: the Delegate of one subdomain that is its own left and right neighbour,
//     i.e. the semantics of SubdomainDelegate (Boundary/SubdomainDelegate.cc:58-181) with
//     comm.size() == 1: periodic ghost fill, reflecting moment fold at the physical ends,
//     periodic moment fold;
//   - a raw binary state format to load/dump particles, fields and moments.
//
// usage:
//   ref_driver init   <out.bin> [color divisor]                   populate with the reference loader
//                                                                 (PartSpecies::populate(color, divisor))
//   ref_driver run    <in.bin> <steps> <chunks> <out-prefix>      advance_by(steps) x chunks
//   ref_driver at     <in.bin> <out-prefix> <s1> <s2> ...         states after s1 < s2 < ... steps in all
//   ref_driver series <in.bin> <every> <chunks> <out.bin>         advance_by(every) x chunks, the
//                                                                 EnergyRecorder sums after each chunk
//   ref_driver bench  <steps> [color divisor]                     time advance_by(steps)
//
// Built with -DH1D_GPU_DOMAIN (oracle/Makefile target `gpu`, binary ref_driver_gpu) it also runs
// the drop-in GPU Domain of the library (hybrid_code-hfemic_wave_b200/adapter/Domain_GPU.h) in
// place of Domain_CAMCL / Domain_PC, through the same state files:
//   ref_driver_gpu gpu_run <in.bin> <steps> <chunks> <out-prefix> fp64|mixed
#include "Boundary/Delegate.h"
#include "Core/Domain_CAMCL.h"
#include "Core/Domain_PC.h"
#if defined(H1D_GPU_DOMAIN)
#include "Domain_GPU.h"
#endif

#include <chrono>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <memory>
#include <stdexcept>
#include <string>
#include <utility>
#include <vector>

using namespace H1D;

namespace {
struct SerialDelegate final : Delegate {
    template <class T, long N>
    static void pass(GridArray<T, N, Pad> &A)
    {
        for (long p = 0; p < Pad; ++p)
            A.end()[p] = A.begin()[p];
        for (long m = -Pad; m < 0; ++m)
            A.begin()[m] = A.end()[m];
    }
    template <class T, long N>
    static void gather(ParamSet const &params, GridArray<T, N, Pad> &A)
    {
        if (params.particle_boundary_condition == BC::reflecting) {
            for (long i = -Pad; i < 0; ++i)
                A[i + 1] += std::exchange(A[i], T{});
            for (long i = N + Pad - 1; i >= N; --i)
                A[i - 1] += std::exchange(A[i], T{});
        }
        T left[Pad], right[Pad];
        for (long k = 0; k < Pad; ++k) {
            left[k]  = A.begin()[k - Pad];
            right[k] = A.end()[k];
        }
        for (long k = 0; k < Pad; ++k)
            A.end()[k - Pad] = A.end()[k - Pad] + left[k];
        for (long k = 0; k < Pad; ++k)
            A.begin()[k] = A.begin()[k] + right[k];
    }
    void once(Domain &) const override {}
    void prologue(Domain const &, long) const override {}
    void epilogue(Domain const &, long) const override {}
    void boundary_pass(Domain const &, ColdSpecies &sp) const override
    {
        pass(sp.mom0_full);
        pass(sp.mom1_full);
    }
    void boundary_pass(Domain const &, BField &b) const override { pass(b); }
    void boundary_pass(Domain const &, EField &e) const override { pass(e); }
    void boundary_pass(Domain const &, Charge &c) const override { pass(c); }
    void boundary_pass(Domain const &, Current &c) const override { pass(c); }
    void boundary_gather(Domain const &, Charge &c) const override { gather(c.params, c); }
    void boundary_gather(Domain const &, Current &c) const override { gather(c.params, c); }
    void boundary_gather(Domain const &, Species &sp) const override
    {
        gather(sp.params, sp.moment<0>());
        gather(sp.params, sp.moment<1>());
        gather(sp.params, sp.moment<2>());
    }
    using Delegate::boundary_pass;
};

std::unique_ptr<Domain> make_domain(ParamSet const &params, Delegate *delegate)
{
    if (ParamSet::algorithm == CAMCL)
        return std::make_unique<Domain_CAMCL>(params, delegate);
    return std::make_unique<Domain_PC>(params, delegate);
}

// PartSpecies::Nc is private; recompute it the way its constructor does (PartSpecies.cc:45-49)
template <class Desc>
double moment_norm(ParamSet const &params, Desc const &desc)
{
    auto const vdf = VDFVariant::make(desc, params.geomtr, params.full_grid_whole_domain_extent, params.c);
    if (long const Np = params.Nx * desc.Nc)
        return Np * vdf->Nrefcell_div_Ntotal();
    return 1;
}
// the equilibrium moments PartSpecies::populate caches before loading (PartSpecies.cc:82-89), for
// a species whose particles come from a state file instead (as a snapshot load restores them)
template <class Desc>
void cache_equilibrium(ParamSet const &params, Desc const &desc, PartSpecies &sp)
{
    auto const vdf   = VDFVariant::make(desc, params.geomtr, params.full_grid_whole_domain_extent, params.c);
    auto const q1min = params.half_grid_subdomain_extent.min();
    for (long i = 0; i < sp.equilibrium_mom0.size(); ++i) {
        CurviCoord const pos{ i + q1min };
        sp.equilibrium_mom0[i] = vdf->n0(pos);
        sp.equilibrium_mom1[i] = vdf->nV0(pos);
        sp.equilibrium_mom2[i] = vdf->nvv0(pos);
    }
}
template <class... Ts, std::size_t... Is>
void cache_equilibria(ParamSet const &params, std::tuple<Ts...> const &descs, Domain &d, std::index_sequence<Is...>)
{
    (cache_equilibrium(params, std::get<Is>(descs), d.part_species.at(Is)), ...);
}
template <class... Ts, std::size_t... Is>
std::vector<double> moment_norms(ParamSet const &params, std::tuple<Ts...> const &descs, std::index_sequence<Is...>)
{
    return { moment_norm(params, std::get<Is>(descs))... };
}

struct Writer {
    FILE *f;
    explicit Writer(char const *path)
    : f{ std::fopen(path, "wb") }
    {
        if (!f)
            throw std::runtime_error{ std::string{ "cannot open " } + path };
    }
    ~Writer() { std::fclose(f); }
    template <class T>
    void put(T const *p, std::size_t n)
    {
        if (n && std::fwrite(p, sizeof(T), n, f) != n)
            throw std::runtime_error{ "write failed" };
    }
    void i64(int64_t v) { put(&v, 1); }
};
struct Reader {
    FILE *f;
    explicit Reader(char const *path)
    : f{ std::fopen(path, "rb") }
    {
        if (!f)
            throw std::runtime_error{ std::string{ "cannot open " } + path };
    }
    ~Reader() { std::fclose(f); }
    template <class T>
    void get(T *p, std::size_t n)
    {
        if (n && std::fread(p, sizeof(T), n, f) != n)
            throw std::runtime_error{ "read failed" };
    }
    int64_t i64()
    {
        int64_t v;
        get(&v, 1);
        return v;
    }
};

template <class T, long N>
double const *raw(GridArray<T, N, Pad> const &g) { return reinterpret_cast<double const *>(g.dead_begin()); }
template <class T, long N>
double *raw(GridArray<T, N, Pad> &g) { return reinterpret_cast<double *>(g.dead_begin()); }
template <class T, long N>
constexpr std::size_t count(GridArray<T, N, Pad> const &) { return sizeof(T) / sizeof(double) * (N + 2 * Pad); }

// state file: see tests/golden/state_io.py for the reader
void dump(Domain const &d, ParamSet const &params, char const *path, int64_t step)
{
    Writer w{ path };
    w.put("H1DSTAT2", 8);
    w.i64(params.Nx);
    w.i64(Pad);
    w.i64(static_cast<int64_t>(d.part_species.size()));
    w.i64(static_cast<int64_t>(d.cold_species.size()));
    w.i64(step);
    auto const norms = moment_norms(params, params.part_descs, ParamSet::part_indices{});
    w.put(norms.data(), norms.size());
    for (PartSpecies const &sp : d.part_species) {
        int64_t const       n = static_cast<int64_t>(sp.bucket.size());
        std::vector<double> a(n);
        w.i64(n);
        for (int c = 0; c < 5; ++c) {
            int64_t k = 0;
            for (Particle const &p : sp.bucket)
                a[k++] = c == 0 ? p.pos.q1 : c == 1 ? p.vel.x : c == 2 ? p.vel.y : c == 3 ? p.vel.z : p.psd.weight;
            w.put(a.data(), n);
        }
        std::vector<int64_t> ids;
        for (Particle const &p : sp.bucket)
            ids.push_back(p.id);
        w.put(ids.data(), ids.size());
        for (int c = 0; c < 2; ++c) { // phase-space density: real_f, marker
            int64_t k = 0;
            for (Particle const &p : sp.bucket)
                a[k++] = c == 0 ? p.psd.real_f : p.psd.marker;
            w.put(a.data(), n);
        }
    }
    w.put(raw(d.bfield), count(d.bfield));
    w.put(raw(d.efield), count(d.efield));
    w.put(raw(d.charge), count(d.charge));
    w.put(raw(d.current), count(d.current));
    for (PartSpecies const &sp : d.part_species) {
        w.put(raw(sp.moment<0>()), count(sp.moment<0>()));
        w.put(raw(sp.moment<1>()), count(sp.moment<1>()));
        w.put(raw(sp.moment<2>()), count(sp.moment<2>()));
    }
    for (ColdSpecies const &sp : d.cold_species) {
        w.put(raw(sp.mom0_full), count(sp.mom0_full));
        w.put(raw(sp.mom1_full), count(sp.mom1_full));
        w.put(raw(sp.moment<0>()), count(sp.moment<0>()));
        w.put(raw(sp.moment<1>()), count(sp.moment<1>()));
        w.put(raw(sp.moment<2>()), count(sp.moment<2>()));
    }
}

int64_t load(Domain &d, ParamSet const &params, char const *path)
{
    Reader r{ path };
    char   magic[8];
    r.get(magic, 8);
    bool const with_psd = std::memcmp(magic, "H1DSTAT2", 8) == 0;
    if (!with_psd && std::memcmp(magic, "H1DSTATE", 8) != 0)
        throw std::runtime_error{ "bad state file" };
    if (r.i64() != params.Nx || r.i64() != Pad || r.i64() != int64_t(d.part_species.size())
        || r.i64() != int64_t(d.cold_species.size()))
        throw std::runtime_error{ "state file does not match this configuration" };
    int64_t const       step = r.i64();
    std::vector<double> norms(d.part_species.size());
    r.get(norms.data(), norms.size());
    for (PartSpecies &sp : d.part_species) {
        int64_t const                      n = r.i64();
        std::vector<std::vector<double>> a(5, std::vector<double>(n));
        for (auto &v : a)
            r.get(v.data(), n);
        std::vector<int64_t> ids(n);
        r.get(ids.data(), n);
        std::vector<double> real_f(a[4]), marker(n, 1.0); // without a PSD: real_f = weight, marker = 1
        if (with_psd) {
            r.get(real_f.data(), n);
            r.get(marker.data(), n);
        }
        sp.bucket.clear();
        for (int64_t k = 0; k < n; ++k) {
            Particle p;
            p.pos    = CurviCoord{ a[0][k] };
            p.vel    = CartVector{ a[1][k], a[2][k], a[3][k] };
            p.psd    = Particle::PSD{ a[4][k], real_f[k], marker[k] };
            p.id     = ids[k];
            sp.bucket.push_back(p);
        }
    }
    r.get(raw(d.bfield), count(d.bfield));
    r.get(raw(d.efield), count(d.efield));
    r.get(raw(d.charge), count(d.charge));
    r.get(raw(d.current), count(d.current));
    for (PartSpecies &sp : d.part_species) {
        r.get(raw(sp.moment<0>()), count(sp.moment<0>()));
        r.get(raw(sp.moment<1>()), count(sp.moment<1>()));
        r.get(raw(sp.moment<2>()), count(sp.moment<2>()));
    }
    for (ColdSpecies &sp : d.cold_species) {
        r.get(raw(sp.mom0_full), count(sp.mom0_full));
        r.get(raw(sp.mom1_full), count(sp.mom1_full));
        r.get(raw(sp.moment<0>()), count(sp.moment<0>()));
        r.get(raw(sp.moment<1>()), count(sp.moment<1>()));
        r.get(raw(sp.moment<2>()), count(sp.moment<2>()));
    }
    return step;
}

// The sums of EnergyRecorder::dump (src/hybrid_1d/Recorder/EnergyRecorder.cc:98-140), which
// cannot be compiled here (its Recorder base needs MPI): dB^2/2 and dE^2/2 per field-aligned
// component over the interior / (2 Nx), then for every kinetic and every cold species KE_lab and
// KE_pla from its moments.  cart_to_mfa is the identity on the field line (MFABasis.h:98-100).
// Appends 6 + 6 (kinetic + cold) doubles to `out`.
void energies(Domain const &d, ParamSet const &params, std::vector<double> &out)
{
    double dB[3] = {}, dE[3] = {};
    for (long i = 0; i < d.bfield.size(); ++i) {
        CartVector const b = d.bfield[i], e = d.efield[i];
        dB[0] += b.x * b.x, dB[1] += b.y * b.y, dB[2] += b.z * b.z;
        dE[0] += e.x * e.x, dE[1] += e.y * e.y, dE[2] += e.z * e.z;
    }
    for (double v : dB)
        out.push_back(v / (2 * params.Nx));
    for (double v : dE)
        out.push_back(v / (2 * params.Nx));
    auto species = [&](Species const &sp) {
        double lab[3] = {}, pla[3] = {};
        for (long i = 0; i < sp.moment<0>().size(); ++i) {
            double const n = Real{ sp.moment<0>()[i] };
            if (n < 1e-15)
                continue;
            CartTensor const nvv = sp.moment<2>()[i];
            CartVector const nV  = sp.moment<1>()[i];
            double const     diag[3] = { nvv.xx, nvv.yy, nvv.zz };
            double const     v[3]    = { nV.x, nV.y, nV.z };
            for (int k = 0; k < 3; ++k) {
                lab[k] += diag[k];
                pla[k] += diag[k] - v[k] * v[k] / n;
            }
        }
        double const f = sp.energy_density_conversion_factor() / (2 * params.Nx);
        for (double x : lab)
            out.push_back(x * f);
        for (double x : pla)
            out.push_back(x * f);
    };
    for (PartSpecies const &sp : d.part_species)
        species(sp);
    for (ColdSpecies const &sp : d.cold_species)
        species(sp);
}
} // namespace

int main(int argc, char **argv)
try {
    if (argc < 2)
        throw std::invalid_argument{ "usage: ref_driver init|run|bench ..." };
    std::string const mode = argv[1];
    Options           opts;
    ParamSet const    params{ 0, opts };
    SerialDelegate    delegate;
    auto              domain = make_domain(params, &delegate);

    if (mode == "init" && (argc == 3 || argc == 5)) {
        long const color   = argc == 5 ? std::atol(argv[3]) : 0;
        long const divisor = argc == 5 ? std::atol(argv[4]) : 1;
        for (PartSpecies &sp : domain->part_species)
            sp.populate(color, divisor);
        for (ColdSpecies &sp : domain->cold_species)
            sp.populate(color, divisor);
        dump(*domain, params, argv[2], 0);
        return 0;
    }
    if (mode == "at" && argc >= 5) {
        int64_t step = load(*domain, params, argv[2]);
        cache_equilibria(params, params.part_descs, *domain, ParamSet::part_indices{});
        long done = 0;
        for (int k = 4; k < argc; ++k) {
            long const target = std::atol(argv[k]);
            if (target <= done)
                throw std::invalid_argument{ "step counts must increase" };
            domain->advance_by(static_cast<unsigned>(target - done));
            step += target - done;
            done = target;
            dump(*domain, params, (std::string{ argv[3] } + std::to_string(target) + ".bin").c_str(), step);
        }
        return 0;
    }
    if (mode == "series" && argc == 6) {
        load(*domain, params, argv[2]);
        cache_equilibria(params, params.part_descs, *domain, ParamSet::part_indices{});
        long const          every  = std::atol(argv[3]);
        long const          chunks = std::atol(argv[4]);
        std::vector<double> out;
        for (long k = 0; k < chunks; ++k) {
            domain->advance_by(static_cast<unsigned>(every));
            energies(*domain, params, out);
        }
        Writer w{ argv[5] };
        w.put(out.data(), out.size());
        return 0;
    }
    if (mode == "run" && argc == 6) {
        int64_t    step   = load(*domain, params, argv[2]);
        cache_equilibria(params, params.part_descs, *domain, ParamSet::part_indices{});
        long const steps  = std::atol(argv[3]);
        long const chunks = std::atol(argv[4]);
        for (long k = 1; k <= chunks; ++k) {
            domain->advance_by(static_cast<unsigned>(steps));
            step += steps;
            dump(*domain, params, (std::string{ argv[5] } + std::to_string(k) + ".bin").c_str(), step);
        }
        return 0;
    }
#if defined(H1D_GPU_DOMAIN)
    if (mode == "gpu_run" && argc == 7) {
        std::string const prec = argv[6];
        if (prec != "fp64" && prec != "mixed")
            throw std::invalid_argument{ "precision must be fp64 or mixed" };
        int const                   precision = prec == "fp64" ? H1D_PREC_FP64 : H1D_PREC_MIXED;
        std::unique_ptr<Domain_GPU> gpu;
        if (ParamSet::algorithm == CAMCL)
            gpu = std::make_unique<Domain_CAMCL_GPU>(params, &delegate, precision);
        else
            gpu = std::make_unique<Domain_PC_GPU>(params, &delegate, precision);
        int64_t step = load(*gpu, params, argv[2]);
        cache_equilibria(params, params.part_descs, *gpu, ParamSet::part_indices{});
        long const steps  = std::atol(argv[3]);
        long const chunks = std::atol(argv[4]);
        for (long k = 1; k <= chunks; ++k) {
            gpu->advance_by(static_cast<unsigned>(steps));
            step += steps;
            gpu->sync_particles(); // as the Driver does before particle recorders and snapshots
            dump(*gpu, params, (std::string{ argv[5] } + std::to_string(k) + ".bin").c_str(), step);
        }
        return 0;
    }
#endif
    if (mode == "bench" && (argc == 3 || argc == 5)) {
        long const steps   = std::atol(argv[2]);
        long const color   = argc == 5 ? std::atol(argv[3]) : 0;
        long const divisor = argc == 5 ? std::atol(argv[4]) : 1;
        auto const t0      = std::chrono::steady_clock::now();
        long       np      = 0;
        for (PartSpecies &sp : domain->part_species) {
            sp.populate(color, divisor);
            np += static_cast<long>(sp.bucket.size());
        }
        for (ColdSpecies &sp : domain->cold_species)
            sp.populate(color, divisor);
        auto const t1 = std::chrono::steady_clock::now();
        domain->advance_by(static_cast<unsigned>(steps));
        auto const   t2      = std::chrono::steady_clock::now();
        double const init_s  = std::chrono::duration<double>(t1 - t0).count();
        double const advance = std::chrono::duration<double>(t2 - t1).count();
        double       dB2     = 0;
        for (long i = 0; i < domain->bfield.size(); ++i)
            dB2 += domain->bfield[i].y * domain->bfield[i].y + domain->bfield[i].z * domain->bfield[i].z;
        std::printf("{\"particles\": %ld, \"steps\": %ld, \"init_s\": %.6f, \"advance_s\": %.6f, "
                    "\"particle_steps_per_s\": %.6e, \"sum_dBperp2\": %.17e}\n",
                    np, steps, init_s, advance, double(np) * double(steps) / advance, dB2);
        return 0;
    }
    throw std::invalid_argument{ "bad arguments" };
} catch (std::domain_error const &e) { // PartSpecies::update_pos (Core/PartSpecies.cc:113)
    std::fprintf(stderr, "ref_driver: std::domain_error: %s\n", e.what());
    return 1;
} catch (std::exception const &e) {
    std::fprintf(stderr, "ref_driver: %s\n", e.what());
    return 1;
}
