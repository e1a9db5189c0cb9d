// libh1d_gpu.so: host side and C-ABI of the B200 implementation of the hybrid_1d hot path.
// The entry points are declared, with the reference interface each one replaces, in
// include/h1d_gpu.h.
#include "h1d_gpu.h"

#include "device_common.cuh"
#include "fields.cuh"
#include "particle_io.cuh"
#include "push_launch.h"
#include "sort.cuh"
#include "launchers.h"

#include <algorithm>
#include <chrono>
#include <cmath>
#include <deque>
#include <map>
#include <memory>
#include <mutex>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <new>
#include <string>
#include <tuple>
#include <vector>

using namespace h1d;

namespace {

// ------------------------------------------------------------------------------------------------
// Device memory of the library.  Runs, batches and served requests come and go, and each holds
// tens of buffers; with cudaMalloc / cudaFree every one of them maps or unmaps device memory
// through the driver, which on a busy host took from milliseconds up to a second per run.  So
// the library allocates from a memory pool of its own per device that keeps freed blocks
// (release threshold: never), with the semantics of cudaMalloc / cudaFree kept:
//   dmalloc  a block from the pool, allocated on an internal stream that is then synchronised,
//            so the block is usable from any stream on return;
//   dfree    waits for the device to be idle (as cudaFree does) and returns the block to the pool.
// Blocks the pool holds but no run uses count as free device memory for admission
// (pool_idle_bytes).  A pinned slab holds the runs' status words (one cudaMallocHost per slab
// of 4096 words instead of one per run).
// ------------------------------------------------------------------------------------------------
constexpr int MAX_DEVICES = 64;
struct DevicePool {
    cudaMemPool_t pool   = nullptr;
    cudaStream_t  stream = nullptr;
};
std::mutex pool_mu;
DevicePool pools[MAX_DEVICES];

cudaError_t device_pool(int dev, DevicePool *&out)
{
    if (dev < 0 || dev >= MAX_DEVICES)
        return cudaErrorInvalidDevice;
    std::lock_guard<std::mutex> lock(pool_mu);
    DevicePool &P = pools[dev];
    if (!P.pool) {
        cudaMemPoolProps props{};
        props.allocType     = cudaMemAllocationTypePinned;
        props.handleTypes   = cudaMemHandleTypeNone;
        props.location.type = cudaMemLocationTypeDevice;
        props.location.id   = dev;
        cudaMemPool_t pool  = nullptr;
        if (cudaError_t const e = cudaMemPoolCreate(&pool, &props))
            return e;
        uint64_t keep = UINT64_MAX;
        cudaStream_t st = nullptr;
        cudaError_t e   = cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep);
        if (e == cudaSuccess)
            e = cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking);
        if (e != cudaSuccess) {
            cudaMemPoolDestroy(pool);
            return e;
        }
        P.pool = pool, P.stream = st;
    }
    out = &P;
    return cudaSuccess;
}

cudaError_t dmalloc_raw(void **p, size_t bytes)
{
    *p      = nullptr;
    int dev = 0;
    if (cudaError_t const e = cudaGetDevice(&dev))
        return e;
    DevicePool *P = nullptr;
    if (cudaError_t const e = device_pool(dev, P))
        return e;
    if (cudaError_t const e = cudaMallocFromPoolAsync(p, bytes ? bytes : 1, P->pool, P->stream)) {
        *p = nullptr;
        return e;
    }
    cudaError_t const e = cudaStreamSynchronize(P->stream);
    if (e != cudaSuccess) {
        cudaFreeAsync(*p, P->stream);
        *p = nullptr;
    }
    return e;
}
template <class T>
cudaError_t dmalloc(T **p, size_t bytes)
{
    return dmalloc_raw(reinterpret_cast<void **>(p), bytes);
}

// the block goes back to the pool of the device it lives on, once the device is idle
void dfree(void *p)
{
    if (!p)
        return;
    cudaPointerAttributes at{};
    DevicePool           *P = nullptr;
    if (cudaPointerGetAttributes(&at, p) != cudaSuccess || device_pool(at.device, P) != cudaSuccess) {
        cudaGetLastError();
        cudaFree(p);
        return;
    }
    cudaDeviceSynchronize();
    cudaFreeAsync(p, P->stream);
}

// device memory the library's pool on `dev` holds without a run using it
size_t pool_idle_bytes(int dev)
{
    DevicePool *P = nullptr;
    if (device_pool(dev, P) != cudaSuccess)
        return 0;
    uint64_t reserved = 0, used = 0;
    if (cudaMemPoolGetAttribute(P->pool, cudaMemPoolAttrReservedMemCurrent, &reserved) != cudaSuccess
        || cudaMemPoolGetAttribute(P->pool, cudaMemPoolAttrUsedMemCurrent, &used) != cudaSuccess)
        return 0;
    return reserved > used ? static_cast<size_t>(reserved - used) : 0;
}

// pinned status words from slabs of 4096
struct StatusSlabs {
    std::mutex              mu;
    std::vector<unsigned *> slabs, free;
};
StatusSlabs status_slabs;
constexpr int STATUS_SLAB = 4096;

unsigned *status_word()
{
    std::lock_guard<std::mutex> lock(status_slabs.mu);
    if (status_slabs.free.empty()) {
        unsigned *slab = nullptr;
        if (cudaMallocHost(&slab, sizeof(unsigned) * STATUS_SLAB) != cudaSuccess)
            return nullptr;
        status_slabs.slabs.push_back(slab);
        for (int i = STATUS_SLAB - 1; i >= 0; --i)
            status_slabs.free.push_back(slab + i);
    }
    unsigned *w = status_slabs.free.back();
    status_slabs.free.pop_back();
    *w = 0;
    return w;
}
void release_status_word(unsigned *w)
{
    if (!w)
        return;
    std::lock_guard<std::mutex> lock(status_slabs.mu);
    status_slabs.free.push_back(w);
}

constexpr int FIELD_BLOCK_MIN = 256;

// shared memory of a field launch of L threads: the predictor-corrector layout or the CAM-CL
// layout with smoothing groups of fb items, whichever is larger
size_t field_smem_bytes(int L, int fb)
{
    return std::max(sizeof(double) * static_cast<size_t>(L) * (SMEM_SCALARS + 3 * SMEM_VECTORS), camcl_smem_bytes(L, fb));
}
// the largest CAM-CL smoothing group whose layout fits `budget` bytes of shared memory: a single
// run's launch (a few CTAs, one per SM) takes what a block can have; a batched launch (hundreds of
// CTAs) keeps two CTAs per SM beside their FieldArgs copies
constexpr size_t FIELD_SMEM_RUN   = 227 * 1024 - sizeof(FieldArgs) - 1024;
constexpr size_t FIELD_SMEM_BATCH = 113 * 1024 - sizeof(FieldArgs) - 1024;
int field_group(int L, size_t budget)
{
    int fb = FB_MAX;
    while (fb > 1 && field_smem_bytes(L, fb) > budget)
        --fb;
    return fb;
}
constexpr int64_t STAGE_N      = int64_t{ 1 } << 22; // doubles in a mixed run's staging buffer (32 MB)

struct SpeciesState {
    int64_t  n = 0, cap = 0;
    double  *buf[2][5] = {}; // FP64: [parity][q1, vx, vy, vz, w]
    int32_t *pos[2]    = {}; // mixed precision: [parity] fixed-point position (pos_cell, pos_off)
    float   *fbuf[2][4] = {}; // mixed precision: [parity][vx, vy, vz, w]
    int32_t *pid[2]    = {};
    double  *psd[2][2] = {}; // FP64 with evolving weights: [parity][real_f, marker]
    float   *fpsd[2][2] = {}; // the same in FP32 for mixed precision
    int      cur       = 0;
    bool     upload_order = false; // the particles are still in the order of their upload
    // sort scratch
    uint32_t *keys[2] = {}, *idx[2] = {};
    unsigned long long *dead = nullptr;
    int       since_sort = 1 << 30;
    // deposits [set][deposit][q] -> M doubles each, contiguous
    double *dep = nullptr;
    // collect_all raw sums: 10 x M
    double *mom_raw = nullptr;
    // finalized moments (GridArray layout): n (M), nV (3M), nvv (6M)
    double *mom = nullptr;
    // delta-f: equilibrium moments n0 (M) and nvv0 (6M) on the half grid, ghosts zero
    double *eq = nullptr;
};

// histogram and scan partials of the cell sort, grown to the largest launch set sorted so far
struct SortScratch {
    uint32_t *hist = nullptr, *part = nullptr;
    int64_t   hist_cap = 0, part_cap = 0;
    void      release()
    {
        dfree(hist), dfree(part);
        hist = part = nullptr, hist_cap = part_cap = 0;
    }
};

struct ColdState {
    double *n   = nullptr;  // M
    double *nV[2] = {};     // 3M ping-pong
    int     cur   = 0;
    double *mom   = nullptr; // n (M), nV (3M), nvv (6M)
};

} // namespace

struct h1d_run {
    h1d_params   p;
    int          device = 0, num_sms = 148;
    cudaStream_t stream = nullptr;
    long         Nx = 0, M = 0;
    int          H = 0, seg = 0, L = 0, nblocks_field = 0, fb = 1;
    size_t       field_smem = 0;
    double      *geo = nullptr;
    double      *B[2] = {}, *E[2] = {}, *EB = nullptr, *charge = nullptr, *current = nullptr;
    float       *EBf = nullptr; // FP32 push record of the mixed-precision particle pass
    double      *stage = nullptr; // mixed precision: FP64 staging of particle uploads and downloads
    int64_t      stage_n = 0;     // its length in doubles
    double      *src_dep = nullptr; // per external source: moment<0> (zero), moment<1> x, y, z (M each)
    bool         mixed = false;
    int          fbits = 0;     // mixed precision: fraction bits F of the fixed-point positions,
    double       pos_scale = 1; // 2^F, with (Nx + 2) 2^F <= 2^31
    double      *E1[2] = {}; // predictor-corrector: averaged E of phases 1 and 2
    int          fcur = 0; // field parity
    int          dset = 0; // deposit set parity
    SpeciesState sp[H1D_MAX_KINETIC];
    SortScratch  sorter;
    ColdState    cold[H1D_MAX_COLD];
    unsigned    *d_status = nullptr;
    unsigned long long *d_fallbacks = nullptr;
    unsigned    *h_status = nullptr; // pinned
    double      *d_energy = nullptr;
    bool         recurring = false, moments_stale = true, fields_dirty = true;
    int64_t      step = 0;
    int          sort_interval = 16;
    int          ctas_per_sm   = 0; // CTAs per SM of the particle pass; 0: the kernel's default
    uint64_t     gen           = 0; // bumped by every upload and particle-count change
    // collect_all formed by the particle pass of the last step (fused_collect): valid while the
    // step count and the particle generation are unchanged
    int64_t      collected_step = -1;
    uint64_t     collected_gen  = 0;
    int          batch_count   = 0; // batches this run is a member of (at most one)
    std::string  msg;
    // profiling: event pairs per phase (0 push, 1 sort, 2 field)
    bool                                           profiling = false;
    std::vector<std::pair<int, cudaEvent_t>>       ev_open;
    std::vector<std::tuple<int, cudaEvent_t, cudaEvent_t>> ev_done;
    std::vector<cudaEvent_t>                       ev_pool;
    h1d_profile                                    prof{};
};

namespace {

std::string fmt(char const *f, ...)
{
    char    b[512];
    va_list ap;
    va_start(ap, f);
    std::vsnprintf(b, sizeof b, f, ap);
    va_end(ap);
    return b;
}

int set_err(h1d_run *r, int code, std::string const &m)
{
    if (r)
        r->msg = m;
    return code;
}

cudaEvent_t pool_event(h1d_run *r)
{
    if (!r->ev_pool.empty()) {
        cudaEvent_t e = r->ev_pool.back();
        r->ev_pool.pop_back();
        return e;
    }
    cudaEvent_t e = nullptr;
    cudaEventCreate(&e);
    return e;
}
void phase_begin(h1d_run *r, int kind)
{
    if (!r->profiling)
        return;
    cudaEvent_t e = pool_event(r);
    cudaEventRecord(e, r->stream);
    r->ev_open.emplace_back(kind, e);
}
void phase_end(h1d_run *r, int kernels)
{
    if (!r->profiling)
        return;
    cudaEvent_t e = pool_event(r);
    cudaEventRecord(e, r->stream);
    auto const [kind, b] = r->ev_open.back();
    r->ev_open.pop_back();
    r->ev_done.emplace_back(kind, b, e);
    r->prof.kernel_launches += kernels;
    if (kind == 0)
        r->prof.push_launches += 1;
    else if (kind == 1)
        r->prof.sort_calls += 1;
    else
        r->prof.field_launches += 1;
}

#define CU(call)                                                                                             \
    do {                                                                                                     \
        cudaError_t const e_ = (call);                                                                       \
        if (e_ != cudaSuccess)                                                                               \
            return set_err(run, e_ == cudaErrorMemoryAllocation ? H1D_ERR_OOM : H1D_ERR_CUDA,                \
                           fmt("%s: %s (%s:%d)", #call, cudaGetErrorString(e_), __FILE__, __LINE__));        \
    } while (0)

// the weights of a species change every step (delta-f, or full-f with PSD refresh)
bool evolves_psd(h1d_kinetic_desc const &d) { return d.scheme == H1D_DELTA_F || d.psd_refresh_frequency != 0; }

// Dawson's integral F(x) = exp(-x^2) int_0^x exp(t^2) dt for x > 0: its Maclaurin series
// sum_n (-2x^2)^n x / (2n+1)!! below 0.2, Rybicki's sampling-theorem sum
// F(x) = pi^-1/2 sum_{n odd} exp(-(x - n h)^2) / n with h = 0.2 (G. B. Rybicki, Computers in
// Physics 3(2), 85 (1989)) up to 50, and the asymptotic series (1/2x) sum_k (2k-1)!! / (2x^2)^k
// beyond; relative error below 2e-15 against an independent evaluation.  CounterBeamVDF needs it
// through B(nu) = 2 nu F(1/nu) (CounterBeamVDF.cc:14-17).
double dawson(double x)
{
    if (x < 0.2) {
        double t = x, sum = x;
        for (int n = 1; n < 40 && std::fabs(t) > 1e-18 * sum; ++n)
            sum += (t *= -2 * x * x / (2 * n + 1));
        return sum;
    }
    if (x > 50) {
        double const r = 1 / (2 * x * x);
        double       t = 1, sum = 1;
        for (int k = 1; k < 12; ++k)
            sum += (t *= (2 * k - 1) * r);
        return sum / (2 * x);
    }
    constexpr double h    = 0.2, span = 7;
    long const       lo   = static_cast<long>(std::floor((x - span) / h)) | 1;
    long const       hi   = static_cast<long>(std::ceil((x + span) / h));
    double           sum  = 0;
    for (long n = lo; n <= hi; n += 2) {
        double const d = x - static_cast<double>(n) * h;
        sum += std::exp(-d * d) / static_cast<double>(n);
    }
    return sum / std::sqrt(M_PI);
}

// the constants of a species' equilibrium distribution (h1d_kinetic_desc::vdf) that its f0 on the
// device (equilibrium_f0 / update_weight_f) and its equilibrium moments need; layout of vc as
// PushArgs::vc
struct VdfConsts {
    double vc[4]     = { 0, 0, 0, 0 };
    double T1_by_vth2 = 0; // partial shell: T_par / vth^2 (PartialShellVDF.cc:19-21)
    double T_by_vth2  = 0; // counter-beam: T / vth^2 (CounterBeamVDF.cc:30-34)
};
// A(xs) = (xs exp(-xs^2) + sqrt(pi) (1/2 + xs^2) erfc(-xs)) / 2, the speed normalisation of the
// shell distributions, and the second speed moment (1/2A)(xs (5/2 + xs^2) exp(-xs^2) +
// sqrt(pi) (3/4 + xs^2 (3 + xs^2)) erfc(-xs)) = T / vth^2 (PartialShellVDF.cc:14-22)
void shell_speed_moments(double xs, double &Ab, double &T_vth2)
{
    double const sqrt_pi = 2 / M_2_SQRTPI;
    Ab     = .5 * (xs * std::exp(-xs * xs) + sqrt_pi * (.5 + xs * xs) * std::erfc(-xs));
    T_vth2 = .5 / Ab * (xs * (2.5 + xs * xs) * std::exp(-xs * xs) + sqrt_pi * (0.75 + xs * xs * (3 + xs * xs)) * std::erfc(-xs));
}
VdfConsts vdf_consts(h1d_kinetic_desc const &d)
{
    VdfConsts k;
    switch (d.vdf) {
        case H1D_VDF_LOSSCONE: { // LossconeVDF.cc:15-35: beta kept 1e-10 away from 0 and 1
            double b = d.vdf_param[0];
            if (b < 1e-10)
                b = 1e-10;
            else if (std::fabs(b - 1) < 1e-10)
                b += std::copysign(1e-10, b - 1);
            k.vc[0] = b, k.vc[1] = d.T2_T1 / (1 + b), k.vc[2] = b * k.vc[1];
            break;
        }
        case H1D_VDF_PARTIAL_SHELL: { // B(zeta) = sqrt(pi) Gamma(1 + zeta/2) / Gamma(3/2 + zeta/2)
            double const zeta = d.vdf_param[0], xs = d.vdf_param[1] / d.vth1;
            double       Ab, T_vth2;
            shell_speed_moments(xs, Ab, T_vth2);
            k.vc[0] = zeta, k.vc[1] = xs, k.vc[2] = Ab;
            k.vc[3] = 2 / M_2_SQRTPI * std::tgamma(1 + .5 * zeta) / std::tgamma(1.5 + .5 * zeta);
            k.T1_by_vth2 = T_vth2 / (3 + zeta);
            break;
        }
        case H1D_VDF_COUNTER_BEAM: { // B(nu) = 2 nu F(1/nu)
            double const nu0 = d.vdf_param[0], xs = d.vdf_param[1] / d.vth1;
            double       Ab, T_vth2;
            shell_speed_moments(xs, Ab, T_vth2);
            k.vc[0] = nu0, k.vc[1] = xs, k.vc[2] = Ab, k.vc[3] = 2 * nu0 * dawson(1 / nu0);
            k.T_by_vth2 = T_vth2;
            break;
        }
        default:
            break;
    }
    return k;
}

// PartSpecies::populate's cache of the equilibrium moments (PartSpecies.cc:82-89) on the interior
// half-grid points, times m_moment_weighting_factor as collect_part adds them: n0 (M doubles) then
// nvv0 (6M, {xx, yy, zz, xy, yz, zx}; mfa_to_cart is the identity on the field line); nV0 = 0;
// ghost cells zero.  Per distribution (impl_n / impl_nvv):
//   bi-Maxwellian (MaxwellianVDF.h:56-70, .cc:33-43): n0 = eta, nvv0 = n0 vth1^2/2 {1, T2OT1, T2OT1};
//   loss-cone (LossconeVDF.h:69-83): n0 = (eta - beta eta_b) / (1 - beta),
//     nvv0 = n0 vth1^2/2 {1, T, T} with T = (1 + beta(q1)) xth2^2(q1);
//   partial shell (PartialShellVDF.h:62-76): n0 = cos^zeta, nvv0 = n0 T1 {1, T, T}, T = (2 + zeta)/2;
//   counter-beam (CounterBeamVDF.h:62-75, .cc:117-133): n0 = B(nu)/B(nu0),
//     nvv0 = n0 T {T1/T, T2/T, T2/T} with T1/T = nu (1/F(1/nu) - nu)/2, T2/T = (1 - T1/T)/2.
std::vector<double> equilibrium_moments(h1d_params const &p, h1d_kinetic_desc const &d)
{
    long const          M = p.Nx + 2 * PAD;
    std::vector<double> eq(7 * M, 0.0);
    double const        q1min = -0.5 * p.Nx + 0.5;
    VdfConsts const     k     = vdf_consts(d);
    double const        w     = p.moment_weighting;
    for (long i = 0; i < p.Nx; ++i) {
        double const q1 = static_cast<double>(i) + q1min;
        double const cs = std::cos(p.xi * p.Dx * q1);
        double       n0, vv[3]; // n0 and the diagonal of nvv0 / n0 in field-aligned components
        if (d.vdf == H1D_VDF_LOSSCONE) {
            double const X = k.vc[1], beq = k.vc[0];
            double const eta   = 1 / (X + (1 - X) * cs * cs);
            double const eta_b = 1 / (k.vc[2] + (1 - k.vc[2]) * cs * cs);
            double       beta  = beq * eta_b / eta;
            if (std::fabs(beta - 1) < 1e-10)
                beta += std::copysign(1e-10, beta - 1);
            double const T = (1 + beta) * (X * eta), hv2 = .5 * d.vth1 * d.vth1;
            n0 = 1 * (eta - beq * eta_b) / (1 - beq);
            vv[0] = 1 * hv2, vv[1] = T * hv2, vv[2] = T * hv2;
        } else if (d.vdf == H1D_VDF_PARTIAL_SHELL) {
            double const zeta = k.vc[0], T = (2 + zeta) / 2, T1 = k.T1_by_vth2 * (d.vth1 * d.vth1);
            n0 = 1 * (zeta == 0 ? 1 : std::pow(cs, zeta));
            vv[0] = 1 * T1, vv[1] = T * T1, vv[2] = T * T1;
        } else if (d.vdf == H1D_VDF_COUNTER_BEAM) {
            double const nu0 = k.vc[0], nu = nu0 * std::sqrt((1 / cs) * (1 / cs));
            double const F = dawson(1 / nu), T1OT = 0.5 * nu * (1 / F - nu), T2OT = 0.5 * (1 - T1OT);
            n0 = 1 * ((2 * nu * F) / k.vc[3]);
            double const T = k.T_by_vth2 * (d.vth1 * d.vth1);
            vv[0] = T1OT * T, vv[1] = T2OT * T, vv[2] = T2OT * T;
        } else {
            double const eta = 1 / (d.T2_T1 + (1 - d.T2_T1) * cs * cs), hv2 = .5 * (d.vth1 * d.vth1);
            n0 = 1 * eta;
            vv[0] = 1 * hv2, vv[1] = (d.T2_T1 * eta) * hv2, vv[2] = (d.T2_T1 * eta) * hv2;
        }
        eq[i + PAD] = n0 * w;
        double *e   = eq.data() + M + 6 * (i + PAD);
        for (int c = 0; c < 3; ++c)
            e[c] = (vv[c] * n0) * w, e[c + 3] = (0 * n0) * w;
    }
    return eq;
}

int validate(h1d_params const *p, std::string &m)
{
#define BAD(...) return m = fmt(__VA_ARGS__), H1D_ERR_INVALID_ARG
    if (!p)
        BAD("null params");
    if (p->Nx < 2 * PAD || p->Nx > 65535)
        BAD("Nx must be in [%d, 65535]", 2 * PAD);
    if (!(p->Dx > 0) || !(p->c > 0) || !(p->O0 > 0) || !(p->dt > 0) || !(p->xi >= 0))
        BAD("Dx, c, O0 and dt must be positive and xi non-negative");
    if (p->n_subcycles < 2 || p->n_subcycles > 256)
        BAD("n_subcycles should be in [2, 256]");
    if (p->algorithm != H1D_ALGO_PC && p->algorithm != H1D_ALGO_CAMCL)
        BAD("unknown algorithm %d", p->algorithm);
    if (p->particle_bc < 0 || p->particle_bc > 2)
        BAD("unknown particle boundary condition %d", p->particle_bc);
    if (p->precision != H1D_PREC_FP64 && p->precision != H1D_PREC_MIXED)
        BAD("unknown precision %d", p->precision);
    if (p->n_kinetic < 0 || p->n_kinetic > H1D_MAX_KINETIC || p->n_cold < 0 || p->n_cold > H1D_MAX_COLD)
        BAD("too many species");
    if (p->phase_retardation_inset < 0 || p->phase_retardation_inset > p->Nx / 2 || p->amplitude_damping_inset < 0
        || p->amplitude_damping_inset > p->Nx / 2)
        BAD("masking inset is greater than half the domain length");
    if (!(p->phase_retardation_factor >= 0 && p->phase_retardation_factor <= 1)
        || !(p->amplitude_damping_factor >= 0 && p->amplitude_damping_factor <= 1))
        BAD("masking factor outside [0, 1]");
    if (!(p->efluid.Oc < 0) || !(p->efluid.op > 0) || !(p->efluid.beta >= 0))
        BAD("invalid electron fluid descriptor");
    for (int s = 0; s < p->n_kinetic; ++s) {
        h1d_kinetic_desc const &d = p->kinetic[s];
        if (d.Oc == 0 || !(d.op > 0))
            BAD("kinetic species %d: Oc should not be zero and op should be positive", s);
        if (d.shape_order < 1 || d.shape_order > 3)
            BAD("kinetic species %d: shape order must be 1, 2 or 3", s);
        if (!(d.moment_norm > 0))
            BAD("kinetic species %d: moment_norm must be positive", s);
        if (d.n_smooth < 0 || d.n_smooth > 64)
            BAD("kinetic species %d: smoothing count outside [0, 64]", s);
        if ((d.scheme != H1D_FULL_F && d.scheme != H1D_DELTA_F) || !(d.psd_refresh_frequency >= 0))
            BAD("kinetic species %d: unknown particle scheme or negative psd_refresh_frequency", s);
        if (d.vdf < H1D_VDF_BIMAXWELLIAN || d.vdf > H1D_VDF_COUNTER_BEAM)
            BAD("kinetic species %d: unknown equilibrium distribution %d", s, d.vdf);
        if (evolves_psd(d)) {
            bool const bimax = d.vdf == H1D_VDF_BIMAXWELLIAN || d.vdf == H1D_VDF_LOSSCONE;
            double const *v  = d.vdf_param;
            if (!(d.vth1 > 0) || (bimax && !(d.T2_T1 > 0)))
                BAD("kinetic species %d: evolving weights need the equilibrium vth1 > 0 (and T2_T1 > 0)", s);
            if (d.vdf == H1D_VDF_LOSSCONE && !(v[0] >= 0))
                BAD("kinetic species %d: losscone.beta should be non-negative", s);
            if (d.vdf == H1D_VDF_PARTIAL_SHELL && (!(v[0] >= 0 && v[0] <= 64) || v[0] != std::floor(v[0]) || !(v[1] >= 0)))
                BAD("kinetic species %d: partial shell zeta should be an integer in [0, 64] and vs non-negative", s);
            if (d.vdf == H1D_VDF_COUNTER_BEAM && (!(v[0] > 0) || !(v[1] >= 0)))
                BAD("kinetic species %d: counter-beam nu should be positive and vs non-negative", s);
        }
    }
    for (int s = 0; s < p->n_cold; ++s)
        if (p->cold[s].Oc == 0 || !(p->cold[s].op > 0) || p->cold[s].n_smooth < 0 || p->cold[s].n_smooth > 64)
            BAD("cold species %d: invalid descriptor", s);
    if (p->n_sources < 0 || p->n_sources > H1D_MAX_SOURCES)
        BAD("too many external sources");
    for (int e = 0; e < p->n_sources; ++e) { // ExternalSourceBase (PlasmaDesc.h:383-403)
        h1d_source_desc const &d = p->sources[e];
        if (!(d.ease_in >= 0) || !(d.ease_out >= 0))
            BAD("external source %d: ease-in/-out should be non-negative", e);
        if (d.n_points < 0 || d.n_points > H1D_MAX_SOURCE_POINTS || d.n_smooth < 0 || d.n_smooth > 64)
            BAD("external source %d: invalid descriptor", e);
    }
    if (p->xi > 0) { // ParamSet.cc:25-29
        double const xd   = p->xi * p->Dx;
        double const e[4] = { -0.5 * p->Nx, -0.5 * p->Nx + p->Nx, -0.5 * p->Nx + 0.5, -0.5 * p->Nx + 0.5 + p->Nx };
        for (double q : e)
            if (!(std::fabs(xd * q) < M_PI_2))
                BAD("invalid domain extent: |xi*D1*q1| >= pi/2");
    }
    return H1D_OK;
#undef BAD
}

double mask_fn(long inset, double factor, double offset)
{
    double const a = offset < 0 ? -offset : offset;
    if (0 == inset || a > static_cast<double>(inset))
        return 1;
    double const tmp = factor * (1 - a / static_cast<double>(inset));
    return (1 - tmp) * (1 + tmp);
}

// per-cell geometry, computed on the host with libm (CurviBasis.h:42, 52-69; MFABasis.h:47;
// MaskingFunction.h:28-35 applied as in BField.cc:40-48)
std::vector<double> geometry_table(h1d_params const &p)
{
    long const          N = p.Nx;
    std::vector<double> g(static_cast<size_t>(G_COUNT) * N);
    double const        D1 = p.Dx, D2 = 1, D3 = 1, iD1 = 1 / D1, iD2 = 1 / D2, iD3 = 1 / D3;
    double const        full_min = -0.5 * N, half_min = full_min + 0.5;
    for (long i = 0; i < N; ++i) {
        double const cf = std::cos(p.xi * D1 * (static_cast<double>(i) + full_min));
        double const ch = std::cos(p.xi * D1 * (static_cast<double>(i) + half_min));
        g[G_FCOV_X * N + i] = D1 / (cf * cf), g[G_FCOV_Y * N + i] = D2 * cf, g[G_FCOV_Z * N + i] = D3 * cf;
        g[G_FCON_X * N + i] = iD1 * (cf * cf), g[G_FCON_Y * N + i] = iD2 / cf, g[G_FCON_Z * N + i] = iD3 / cf;
        g[G_HCOV_X * N + i] = D1 / (ch * ch), g[G_HCOV_Y * N + i] = D2 * ch, g[G_HCOV_Z * N + i] = D3 * ch;
        g[G_HCON_X * N + i] = iD1 * (ch * ch), g[G_HCON_Y * N + i] = iD2 / ch, g[G_HCON_Z * N + i] = iD3 / ch;
        double const ih     = 1 / ch;
        g[G_HBX * N + i]    = (ih * ih) * p.O0;
        long const   a = i < N - 1 - i ? i : N - 1 - i, b = i < N - 1 - i ? N - 1 - i : i;
        g[G_MP1 * N + i] = mask_fn(p.phase_retardation_inset, p.phase_retardation_factor, 0.0 + a);
        g[G_MP2 * N + i] = mask_fn(p.phase_retardation_inset, p.phase_retardation_factor, 0.0 + b);
        g[G_MA1 * N + i] = mask_fn(p.amplitude_damping_inset, p.amplitude_damping_factor, 0.0 + a);
        g[G_MA2 * N + i] = mask_fn(p.amplitude_damping_inset, p.amplitude_damping_factor, 0.0 + b);
    }
    return g;
}

double cdcf(h1d_params const &p, double Oc, double op) { return ((op * op) * p.O0) / Oc; }
double ccf(h1d_params const &p, double Oc, double op) { return cdcf(p, Oc, op) / p.c; }

template <class T>
int dalloc(h1d_run *run, T **ptr, size_t count)
{
    CU(dmalloc(reinterpret_cast<void **>(ptr), sizeof(T) * (count ? count : 1)));
    CU(cudaMemsetAsync(*ptr, 0, sizeof(T) * (count ? count : 1), run->stream));
    return H1D_OK;
}

#define TRY(x)                                                                                               \
    do {                                                                                                     \
        int const st_ = (x);                                                                                 \
        if (st_ != H1D_OK)                                                                                   \
            return st_;                                                                                      \
    } while (0)

double *dep_ptr(h1d_run *run, int s, int set, int d, int q)
{
    return run->sp[s].dep + ((static_cast<size_t>(set) * 2 + d) * 4 + q) * run->M + PAD;
}

// the end of the fixed-point grid, Nx 2^F (below 2^31 by the choice of F)
int32_t pos_len(h1d_run const *run) { return static_cast<int32_t>(run->Nx << run->fbits); }

int ppt_for(h1d_run const *run, int s)
{
    return mom_ppt(static_cast<double>(run->sp[s].n) / static_cast<double>(run->Nx));
}

PushArgs push_args(h1d_run *run, int s)
{
    h1d_params const       &p = run->p;
    h1d_kinetic_desc const &d = p.kinetic[s];
    SpeciesState           &S = run->sp[s];
    PushArgs                a{};
    a.q1 = S.buf[S.cur][0], a.vx = S.buf[S.cur][1], a.vy = S.buf[S.cur][2], a.vz = S.buf[S.cur][3];
    a.w = S.buf[S.cur][4], a.pid = S.pid[S.cur];
    a.n = S.n, a.Nx = static_cast<int>(run->Nx);
    a.EB = run->EB + 6 * PAD;
    for (int dd = 0; dd < 2; ++dd)
        for (int q = 0; q < 4; ++q)
            a.dep[dd][q] = dep_ptr(run, s, run->dset, dd, q);
    a.full_min = -0.5 * p.Nx, a.full_len = static_cast<double>(p.Nx), a.full_max = a.full_min + a.full_len;
    a.half_min = a.full_min + 0.5;
    a.xi = p.xi, a.xi2 = p.xi * p.xi, a.xiD1 = p.xi * p.Dx, a.D1 = p.Dx, a.inv_D1 = 1 / p.Dx, a.O0 = p.O0;
    a.Oc = d.Oc, a.dt = p.dt, a.travel_scale = 1.0, a.boris = boris_make(p.dt, p.c, p.O0, d.Oc);
    a.xiO0_Oc = p.xi * p.O0 / d.Oc;
    a.status = run->d_status, a.fallbacks = run->d_fallbacks, a.seed = p.gyrophase_seed, a.counter = static_cast<uint64_t>(run->step) * 8;
    a.species = s, a.randomize = p.randomize_gyrophase, a.homogeneous_poly = p.xi < 1e-10;
    a.move_steps = 1, a.deposit_mask = 3, a.write_back = 1;
    if (S.psd[S.cur][0]) {
        a.real_f = S.psd[S.cur][0], a.marker = S.psd[S.cur][1];
        a.nu_dt = d.psd_refresh_frequency * p.dt, a.psd_refresh = d.psd_refresh_frequency != 0;
        a.delta_f = d.scheme == H1D_DELTA_F;
        a.vth1 = d.vth1, a.vth1_cubed = d.vth1 * d.vth1 * d.vth1, a.T2_T1 = d.T2_T1;
        VdfConsts const k = vdf_consts(d);
        a.vdf = d.vdf;
        for (int j = 0; j < 4; ++j)
            a.vc[j] = k.vc[j];
    }
    return a;
}

// the mixed-precision arguments of species s with the pass settings of `a` (constants in FP32)
PushArgsMixed mixed_args(h1d_run *run, int s, PushArgs const &a)
{
    SpeciesState &S = run->sp[s];
    PushArgsMixed m{};
    m.pos = S.pos[S.cur], m.vx = S.fbuf[S.cur][0], m.vy = S.fbuf[S.cur][1], m.vz = S.fbuf[S.cur][2];
    m.w = S.fbuf[S.cur][3], m.pid = S.pid[S.cur], m.n = a.n, m.Nx = a.Nx;
    m.fbits = run->fbits, m.scale = static_cast<float>(run->pos_scale), m.inv_scale = static_cast<float>(1 / run->pos_scale);
    m.EB = run->EBf + EBF_STRIDE * PAD;
    for (int d = 0; d < 2; ++d)
        for (int q = 0; q < 4; ++q)
            m.dep[d][q] = a.dep[d][q];
    for (int q = 0; q < 6; ++q)
        m.nvv[q] = a.nvv[q];
    m.full_min = static_cast<float>(a.full_min), m.xiD1 = static_cast<float>(a.xiD1);
    m.inv_D1 = static_cast<float>(a.inv_D1), m.O0 = static_cast<float>(a.O0), m.dt = static_cast<float>(a.dt);
    m.travel_scale = static_cast<float>(a.travel_scale), m.xiO0_Oc = static_cast<float>(a.xiO0_Oc);
    m.dtOc_2O0 = static_cast<float>(a.boris.dtOc_2O0), m.cDtOc_2O0 = static_cast<float>(a.boris.cDtOc_2O0);
    m.status = a.status, m.fallbacks = a.fallbacks, m.seed = a.seed, m.counter = a.counter;
    m.species = a.species, m.randomize = a.randomize;
    m.move_steps = a.move_steps, m.deposit_mask = a.deposit_mask, m.write_back = a.write_back;
    if (S.fpsd[S.cur][0]) {
        h1d_kinetic_desc const &d = run->p.kinetic[s];
        m.real_f = S.fpsd[S.cur][0], m.marker = S.fpsd[S.cur][1];
        m.nu_dt = static_cast<float>(d.psd_refresh_frequency * run->p.dt), m.psd_refresh = d.psd_refresh_frequency != 0;
        m.delta_f = d.scheme == H1D_DELTA_F, m.vth1 = static_cast<float>(d.vth1);
        m.vth1_cubed = static_cast<float>(d.vth1 * d.vth1 * d.vth1), m.T2_T1 = static_cast<float>(d.T2_T1);
        VdfConsts const k = vdf_consts(d); // push_args fills its copy only for FP64 PSD arrays
        m.vdf = d.vdf;
        for (int j = 0; j < 4; ++j)
            m.vc[j] = static_cast<float>(k.vc[j]);
    }
    return m;
}

int launch_push(h1d_run *run, int s, PushArgs const &a)
{
    if (a.n == 0)
        return H1D_OK;
    int const  order  = run->p.kinetic[s].shape_order;
    bool const mirror = run->p.xi != 0;
    if (run->mixed && run->sp[s].fpsd[0][0]) {
        PushArgsMixed const m = mixed_args(run, s, a);
        CU(launch_push_psd(m, order, mirror, run->p.particle_bc, run->num_sms * PIPE_CTAS_PER_SM_MIXED, run->stream));
    } else if (run->mixed) {
        PushArgsMixed const m = mixed_args(run, s, a);
        CU(launch_push_groups(&m, 1, order, mirror, run->p.particle_bc,
                              run->num_sms * (run->ctas_per_sm ? run->ctas_per_sm : PIPE_CTAS_PER_SM_MIXED), run->stream));
    } else if (a.real_f) {
        CU(launch_push_psd(a, order, mirror, run->p.particle_bc, run->num_sms * PIPE_CTAS_PER_SM, run->stream));
    } else {
        CU(launch_push_groups(&a, 1, order, mirror, run->p.particle_bc,
                              run->num_sms * (run->ctas_per_sm ? std::min(run->ctas_per_sm, PIPE_CTAS_PER_SM) : PIPE_CTAS_PER_SM),
                              run->stream));
    }
    return H1D_OK;
}

// ---- cell sort (sort.cuh): the species of one run, or of every member of an ensemble, sorted
// together, one launch per kernel for up to SORT_SEGS species ----
constexpr int      SORT_SEGS    = 64;
constexpr uint64_t SORT_SET_MAX = 0xffffffffull; // particles of one launch set (32-bit places)

struct SortItem {
    h1d_run *run;
    int      s;
};

bool has_psd(SpeciesState const &S) { return S.psd[0][0] != nullptr || S.fpsd[0][0] != nullptr; }

cudaError_t grow(uint32_t *&buf, int64_t &cap, int64_t need)
{
    if (need <= cap)
        return cudaSuccess;
    dfree(buf);
    buf = nullptr, cap = 0;
    cudaError_t const e = dmalloc(&buf, sizeof(uint32_t) * need);
    if (e == cudaSuccess)
        cap = need;
    return e;
}

template <bool PSD>
void fill_move(MoveFP64T<PSD> &m, SpeciesState const &P)
{
    for (int k = 0; k < 5; ++k)
        m.src[k] = P.buf[P.cur][k], m.dst[k] = P.buf[1 - P.cur][k];
    if constexpr (PSD)
        for (int k = 0; k < 2; ++k)
            m.src[5 + k] = P.psd[P.cur][k], m.dst[5 + k] = P.psd[1 - P.cur][k];
    m.pid_src = P.pid[P.cur], m.pid_dst = P.pid[1 - P.cur];
}
template <bool PSD>
void fill_move(MoveMixedT<PSD> &m, SpeciesState const &P)
{
    for (int k = 0; k < 4; ++k)
        m.src[k] = P.fbuf[P.cur][k], m.dst[k] = P.fbuf[1 - P.cur][k];
    if constexpr (PSD)
        for (int k = 0; k < 2; ++k)
            m.src[4 + k] = P.fpsd[P.cur][k], m.dst[4 + k] = P.fpsd[1 - P.cur][k];
    m.pos_src = P.pos[P.cur], m.pos_dst = P.pos[1 - P.cur];
    m.pid_src = P.pid[P.cur], m.pid_dst = P.pid[1 - P.cur];
}

// the last pass: the particle records of every segment move to their places
template <int KIND, class Move, int MAXS>
cudaError_t scatter_records(SortSegs<MAXS> const &S, SortItem const *it, int shift, unsigned mask,
                            uint32_t const *offsets, unsigned nt, cudaStream_t st)
{
    std::unique_ptr<MoveSegs<Move, MAXS>> M(new (std::nothrow) MoveSegs<Move, MAXS>{});
    if (!M)
        return cudaErrorMemoryAllocation;
    for (int g = 0; g < S.n; ++g)
        fill_move(M->mv[g], it[g].run->sp[it[g].s]);
    scatter_kernel<KIND, Move, MAXS><<<nt, SORT_THREADS, 0, st>>>(S, *M, shift, mask, offsets);
    return cudaGetLastError();
}
template <int KIND, int MAXS>
cudaError_t scatter_records(SortSegs<MAXS> const &S, SortItem const *it, bool mixed, bool psd, int shift,
                            unsigned mask, uint32_t const *offsets, unsigned nt, cudaStream_t st)
{
    if (mixed)
        return psd ? scatter_records<KIND, MoveMixedT<true>>(S, it, shift, mask, offsets, nt, st)
                   : scatter_records<KIND, MoveMixedT<false>>(S, it, shift, mask, offsets, nt, st);
    return psd ? scatter_records<KIND, MoveFP64T<true>>(S, it, shift, mask, offsets, nt, st)
               : scatter_records<KIND, MoveFP64T<false>>(S, it, shift, mask, offsets, nt, st);
}

// one launch set: m non-empty species of one precision and one PSD kind, fewer than 2^32
// particles in all; sorts them into their other parity buffers (the caller flips `cur`)
template <int MAXS>
cudaError_t sort_set(SortItem const *it, int m, SortScratch &sc, cudaStream_t st, int64_t &launches)
{
    std::unique_ptr<SortSegs<MAXS>> S(new (std::nothrow) SortSegs<MAXS>{});
    if (!S)
        return cudaErrorMemoryAllocation;
    bool const mixed = it[0].run->mixed;
    bool const psd   = has_psd(it[0].run->sp[it[0].s]);
    int        Nx    = 1;
    int64_t    tiles = 0, first = 0;
    S->n             = m;
    for (int g = 0; g < m; ++g) {
        h1d_run *const      r = it[g].run;
        SpeciesState const &P = r->sp[it[g].s];
        S->tile0[g]           = static_cast<int>(tiles);
        S->first[g]           = static_cast<uint32_t>(first);
        S->count[g]           = static_cast<uint32_t>(P.n);
        tiles += (P.n + SORT_TILE - 1) / SORT_TILE;
        first += P.n;
        SortKeys &k = S->key[g];
        k.full_min = -0.5 * static_cast<double>(r->Nx), k.Nx = static_cast<int>(r->Nx);
        k.dead = P.dead, k.status = r->d_status, k.absorbing = r->p.particle_bc == H1D_BC_ABSORBING;
        if (mixed)
            k.pos = P.pos[P.cur], k.fbits = r->fbits, k.wf = P.fbuf[P.cur][3];
        else
            k.q1 = P.buf[P.cur][0], k.w = P.buf[P.cur][4];
        if (k.absorbing) { // absorbed particles are counted by the first histogram
            cudaError_t const e = cudaMemsetAsync(P.dead, 0, sizeof(unsigned long long), st);
            if (e != cudaSuccess)
                return e;
        }
        Nx = std::max(Nx, k.Nx);
    }
    S->tile0[m]          = static_cast<int>(tiles);
    SortPlan const plan  = sort_plan(Nx); // the widest grid's digits serve every segment
    int64_t const  hlen  = (int64_t{1} << std::max(plan.bits[0], plan.bits[1])) * tiles;
    cudaError_t    e     = grow(sc.hist, sc.hist_cap, hlen);
    if (e == cudaSuccess)
        e = grow(sc.part, sc.part_cap, (hlen + SCAN_SEG - 1) / SCAN_SEG);
    if (e != cudaSuccess)
        return e;
    unsigned const nt    = static_cast<unsigned>(tiles);
    int            shift = 0, src = 0; // keys/idx buffer the current pass reads (the first pass reads the particles)
    for (int pass = 0; pass < plan.passes; ++pass) {
        unsigned const mask = (1u << plan.bits[pass]) - 1u;
        int64_t const  len  = static_cast<int64_t>(mask + 1) * tiles;
        unsigned const np   = static_cast<unsigned>((len + SCAN_SEG - 1) / SCAN_SEG);
        bool const     last = pass == plan.passes - 1;
        for (int g = 0; g < m; ++g) {
            SpeciesState const &P = it[g].run->sp[it[g].s];
            S->key[g].keys        = P.keys[src];
            S->idx_in[g]          = P.idx[src];
        }
        if (pass > 0)
            hist_kernel<KEYS_ARRAY, MAXS><<<nt, SORT_THREADS, 0, st>>>(*S, shift, mask, sc.hist);
        else if (mixed)
            hist_kernel<KEYS_MIXED, MAXS><<<nt, SORT_THREADS, 0, st>>>(*S, shift, mask, sc.hist);
        else
            hist_kernel<KEYS_FP64, MAXS><<<nt, SORT_THREADS, 0, st>>>(*S, shift, mask, sc.hist);
        scan_reduce_kernel<<<np, SCAN_THREADS, 0, st>>>(sc.hist, len, sc.part);
        scan_partials_kernel<<<1, 1024, 0, st>>>(sc.part, static_cast<int>(np));
        scan_down_kernel<<<np, SCAN_THREADS, 0, st>>>(sc.hist, len, sc.part);
        if (!last) { // (key, index) pairs for the next pass
            std::unique_ptr<MoveSegs<MoveKeys, MAXS>> K(new (std::nothrow) MoveSegs<MoveKeys, MAXS>{});
            if (!K)
                return cudaErrorMemoryAllocation;
            for (int g = 0; g < m; ++g) {
                SpeciesState const &P = it[g].run->sp[it[g].s];
                K->mv[g]              = MoveKeys{ P.keys[1 - src], P.idx[1 - src] };
            }
            if (pass > 0)
                scatter_kernel<KEYS_ARRAY, MoveKeys, MAXS><<<nt, SORT_THREADS, 0, st>>>(*S, *K, shift, mask, sc.hist);
            else if (mixed)
                scatter_kernel<KEYS_MIXED, MoveKeys, MAXS><<<nt, SORT_THREADS, 0, st>>>(*S, *K, shift, mask, sc.hist);
            else
                scatter_kernel<KEYS_FP64, MoveKeys, MAXS><<<nt, SORT_THREADS, 0, st>>>(*S, *K, shift, mask, sc.hist);
            e = cudaGetLastError();
        } else if (pass > 0) {
            e = scatter_records<KEYS_ARRAY>(*S, it, mixed, psd, shift, mask, sc.hist, nt, st);
        } else if (mixed) {
            e = scatter_records<KEYS_MIXED>(*S, it, mixed, psd, shift, mask, sc.hist, nt, st);
        } else {
            e = scatter_records<KEYS_FP64>(*S, it, mixed, psd, shift, mask, sc.hist, nt, st);
        }
        if (e != cudaSuccess)
            return e;
        shift += plan.bits[pass];
        src = 1 - src;
    }
    launches += 5 * plan.passes;
    return cudaGetLastError();
}

// sorts the listed species (any runs, any mix of precisions) in as few launch sets as their
// kinds allow; under the absorbing boundary the absorbed particles are then trimmed (one host
// synchronisation for all of them)
cudaError_t sort_items(std::vector<SortItem> const &items, SortScratch &sc, cudaStream_t st, int64_t &launches)
{
    std::vector<SortItem> todo;
    bool                  absorbing = false;
    for (SortItem const &x : items) {
        SpeciesState &P = x.run->sp[x.s];
        P.since_sort    = 0;
        P.upload_order  = false;
        if (P.n > 0)
            todo.push_back(x), absorbing |= x.run->p.particle_bc == H1D_BC_ABSORBING;
    }
    for (int kind = 0; kind < 4; ++kind) { // (mixed, psd) kinds, in turn
        std::vector<SortItem> set;
        uint64_t              total = 0;
        auto const            flush = [&]() -> cudaError_t {
            if (set.empty())
                return cudaSuccess;
            cudaError_t const e = set.size() == 1 ? sort_set<1>(set.data(), 1, sc, st, launches)
                                                  : sort_set<SORT_SEGS>(set.data(), static_cast<int>(set.size()), sc, st, launches);
            set.clear(), total = 0;
            return e;
        };
        for (SortItem const &x : todo) {
            SpeciesState const &P = x.run->sp[x.s];
            if ((x.run->mixed ? 2 : 0) + (has_psd(P) ? 1 : 0) != kind)
                continue;
            if (set.size() == SORT_SEGS || total + static_cast<uint64_t>(P.n) > SORT_SET_MAX)
                if (cudaError_t const e = flush())
                    return e;
            set.push_back(x), total += static_cast<uint64_t>(P.n);
        }
        if (cudaError_t const e = flush())
            return e;
    }
    for (SortItem const &x : todo)
        x.run->sp[x.s].cur ^= 1;
    if (!absorbing)
        return cudaSuccess;
    std::vector<unsigned long long> dead(todo.size(), 0);
    for (size_t i = 0; i < todo.size(); ++i)
        if (todo[i].run->p.particle_bc == H1D_BC_ABSORBING)
            if (cudaError_t const e = cudaMemcpyAsync(&dead[i], todo[i].run->sp[todo[i].s].dead, sizeof(unsigned long long),
                                                      cudaMemcpyDeviceToHost, st))
                return e;
    if (cudaError_t const e = cudaStreamSynchronize(st))
        return e;
    for (size_t i = 0; i < todo.size(); ++i) // removed particles were sorted to the end
        if (dead[i]) {
            todo[i].run->sp[todo[i].s].n -= static_cast<int64_t>(dead[i]);
            todo[i].run->gen++;
        }
    return cudaSuccess;
}

// stable cell sort of the listed species of one run
int sort_run(h1d_run *run, std::vector<SortItem> const &items)
{
    if (items.empty())
        return H1D_OK;
    int64_t launches = 0;
    phase_begin(run, 1);
    CU(sort_items(items, run->sorter, run->stream, launches));
    phase_end(run, static_cast<int>(launches));
    return H1D_OK;
}
int sort_species(h1d_run *run, int s) { return sort_run(run, { SortItem{ run, s } }); }

// the species of the run whose sort interval is up, sorted together
int sort_due(h1d_run *run)
{
    std::vector<SortItem> due;
    for (int s = 0; s < run->p.n_kinetic; ++s)
        if (run->sp[s].since_sort >= run->sort_interval)
            due.push_back({ run, s });
    return sort_run(run, due);
}

FieldArgs field_args(h1d_run *run)
{
    h1d_params const &p = run->p;
    FieldArgs         a{};
    a.Nx = static_cast<int>(run->Nx), a.H = run->H, a.seg = run->seg, a.bc = p.particle_bc == H1D_BC_PERIODIC ? 0 : 1;
    a.geo = run->geo;
    a.B_in = run->B[run->fcur] + 3 * PAD, a.E_in = run->E[run->fcur] + 3 * PAD;
    a.B_out = run->B[1 - run->fcur] + 3 * PAD, a.E_out = run->E[1 - run->fcur] + 3 * PAD;
    a.EB_out = run->EB + 6 * PAD, a.EBf_out = run->EBf ? run->EBf + EBF_STRIDE * PAD : nullptr, a.charge_out = run->charge + PAD, a.current_out = run->current + 3 * PAD;
    a.nk = p.n_kinetic, a.nc = p.n_cold;
    for (int s = 0; s < p.n_kinetic; ++s) {
        h1d_kinetic_desc const &d = p.kinetic[s];
        KinSrc                 &K = a.k[s];
        for (int dd = 0; dd < 2; ++dd)
            for (int q = 0; q < 4; ++q) {
                K.raw[dd][q]  = dep_ptr(run, s, run->dset, dd, q);
                K.zero[dd][q] = dep_ptr(run, s, 1 - run->dset, dd, q);
            }
        K.s1 = 1.0 / d.moment_norm, K.cdcf = cdcf(p, d.Oc, d.op), K.ccf = ccf(p, d.Oc, d.op);
        K.lamf = K.cdcf * d.Oc / p.O0, K.gamf = K.ccf * d.Oc / p.O0, K.nsm = static_cast<int>(d.n_smooth);
        K.eq = run->sp[s].eq ? run->sp[s].eq + PAD : nullptr;
    }
    for (int c = 0; c < p.n_cold; ++c) {
        h1d_cold_desc const &d = p.cold[c];
        ColdSrc             &K = a.c[c];
        ColdState           &C = run->cold[c];
        K.n = C.n + PAD, K.nV_in = C.nV[C.cur] + 3 * PAD, K.nV_out = C.nV[1 - C.cur] + 3 * PAD;
        K.boris = boris_make(p.dt, p.c, p.O0, d.Oc);
        K.cdcf = cdcf(p, d.Oc, d.op), K.ccf = ccf(p, d.Oc, d.op), K.lamf = K.cdcf * d.Oc / p.O0, K.gamf = K.ccf * d.Oc / p.O0;
        K.w = p.moment_weighting, K.nsm = static_cast<int>(d.n_smooth);
    }
    a.ne = p.n_sources;
    for (int e = 0; e < p.n_sources; ++e) {
        KinSrc &K = a.e[e];
        for (int dd = 0; dd < 2; ++dd)
            for (int q = 0; q < 4; ++q)
                K.raw[dd][q] = run->src_dep + (static_cast<size_t>(e) * 4 + q) * run->M + PAD, K.zero[dd][q] = nullptr;
        K.s1 = 1.0, K.cdcf = 0.0, K.ccf = 1.0;
        K.lamf = 0.0 * p.O0 / p.O0, K.gamf = 1.0 * p.O0 / p.O0; // Oc = O0 (ExternalSource.hh:19)
        K.nsm = static_cast<int>(p.sources[e].n_smooth);
    }
    a.dt = p.dt, a.sub_dt = p.dt / p.n_subcycles, a.c_light = p.c, a.sqrt_g = p.Dx * 1 * 1, a.O0 = p.O0, a.inv_D1 = 1 / p.Dx;
    a.m = static_cast<int>(p.n_subcycles);
    a.fb = run->fb;
    h1d_efluid_desc const &ef = p.efluid;
    a.O02beO2 = (p.O0 * p.O0) * ef.beta * 0.5, a.mOeOO0oe2 = -ef.Oc / (p.O0 * (ef.op * ef.op)), a.gamma = ef.gamma;
    a.cO2 = p.c / 2, a.cOsqrtg = p.c / a.sqrt_g;
    return a;
}

// first advance: fill ghost cells of E and B (Domain_CAMCL.cc:27-35) and B on the half grid
int prepare_fields(h1d_run *run)
{
    CU(launch_prep_fields(run->B[run->fcur] + 3 * PAD, run->E[run->fcur] + 3 * PAD, run->EB + 6 * PAD,
                          run->EBf ? run->EBf + EBF_STRIDE * PAD : nullptr, static_cast<int>(run->Nx), run->stream));
    run->fields_dirty = false;
    return H1D_OK;
}

// ExternalSource::update at time t of every external source (its moment<1> for the field kernel)
int launch_run_sources(h1d_run *run, double t)
{
    h1d_params const &p = run->p;
    if (p.n_sources == 0)
        return H1D_OK;
    SourceArgs a{};
    a.ne = p.n_sources, a.t = t, a.half_min = -0.5 * p.Nx + 0.5, a.half_len = static_cast<double>(p.Nx);
    a.weighting = p.moment_weighting, a.M = static_cast<int>(run->M);
    for (int e = 0; e < p.n_sources; ++e) {
        a.d[e] = p.sources[e];
        for (int c = 0; c < 3; ++c)
            a.J[e][c] = run->src_dep + (static_cast<size_t>(e) * 4 + 1 + c) * run->M + PAD;
    }
    CU(launch_sources(a, run->stream));
    if (run->profiling)
        run->prof.kernel_launches += 1;
    return H1D_OK;
}

// a particle pass of every species of a run with the arguments args_of(s): species of one shape
// order whose weights do not evolve share one launch, as the groups of a batch do
template <class ArgsOf>
int push_run(h1d_run *run, ArgsOf const &args_of)
{
    h1d_params const &p = run->p;
    int const         K = p.n_kinetic;
    bool              done[H1D_MAX_KINETIC] = {};
    for (int s = 0; s < K; ++s) {
        if (done[s])
            continue;
        int grp[H1D_MAX_KINETIC], m = 0;
        grp[m++] = s;
        done[s]  = true;
        if (!evolves_psd(p.kinetic[s]) && run->sp[s].n > 0)
            for (int t = s + 1; t < K; ++t)
                if (!done[t] && run->sp[t].n > 0 && !evolves_psd(p.kinetic[t]) && p.kinetic[t].shape_order == p.kinetic[s].shape_order)
                    grp[m++] = t, done[t] = true;
        phase_begin(run, 0);
        if (m == 1) {
            TRY(launch_push(run, s, args_of(s)));
        } else {
            int const  order  = static_cast<int>(p.kinetic[s].shape_order);
            bool const mirror = p.xi != 0;
            if (run->mixed) {
                PushArgsMixed g[H1D_MAX_KINETIC];
                for (int i = 0; i < m; ++i)
                    g[i] = mixed_args(run, grp[i], args_of(grp[i]));
                CU(launch_push_groups(g, m, order, mirror, p.particle_bc,
                                      run->num_sms * (run->ctas_per_sm ? run->ctas_per_sm : PIPE_CTAS_PER_SM_MIXED), run->stream));
            } else {
                PushArgs g[H1D_MAX_KINETIC];
                for (int i = 0; i < m; ++i)
                    g[i] = args_of(grp[i]);
                CU(launch_push_groups(g, m, order, mirror, p.particle_bc,
                                      run->num_sms * (run->ctas_per_sm ? std::min(run->ctas_per_sm, PIPE_CTAS_PER_SM) : PIPE_CTAS_PER_SM),
                                      run->stream));
            }
        }
        phase_end(run, run->sp[s].n > 0 ? 1 : 0);
    }
    return H1D_OK;
}

// collect_all (PartSpecies.cc:225-244) deposits with CIC whatever the species' shape, and the
// particle pass deposits n and nV at the end position with the same weights and velocities.  So
// when every species is CIC with fixed weights, the pass of an advance_by's last step also
// deposits the second moments w v_i v_j, and finalize_moments takes n and nV from that step's
// end-position deposit: no sort and no separate pass over the particles.
bool fused_collect(h1d_run const *run)
{
    h1d_params const &p = run->p;
    if (p.algorithm != H1D_ALGO_CAMCL || p.n_kinetic < 1)
        return false;
    for (int s = 0; s < p.n_kinetic; ++s)
        if (p.kinetic[s].shape_order != 1 || evolves_psd(p.kinetic[s]))
            return false;
    return true;
}

// the particle pass of one CAM-CL step that also forms collect_all's second moments into mom_raw
int push_collect(h1d_run *run)
{
    h1d_params const &p      = run->p;
    bool const        mirror = p.xi != 0;
    for (int s = 0; s < p.n_kinetic; ++s) {
        SpeciesState &S = run->sp[s];
        CU(cudaMemsetAsync(S.mom_raw + 4 * run->M, 0, sizeof(double) * 6 * run->M, run->stream));
        PushArgs a = push_args(run, s);
        for (int q = 0; q < 6; ++q)
            a.nvv[q] = S.mom_raw + static_cast<size_t>(4 + q) * run->M + PAD;
        if (a.n == 0)
            continue;
        phase_begin(run, 0);
        if (run->mixed)
            CU(launch_push_nvv(mixed_args(run, s, a), mirror, p.particle_bc, run->num_sms * PIPE_CTAS_PER_SM_NVV_MIXED,
                               run->stream));
        else
            CU(launch_push_nvv(a, mirror, p.particle_bc, run->num_sms * PIPE_CTAS_PER_SM_NVV_FP64, run->stream));
        phase_end(run, 1);
    }
    return H1D_OK;
}

int camcl_step(h1d_run *run, bool collect = false)
{
    h1d_params const &p = run->p;
    TRY(sort_due(run));
    if (collect)
        TRY(push_collect(run));
    else
        TRY(push_run(run, [run](int s) { return push_args(run, s); }));
    for (int s = 0; s < p.n_kinetic; ++s) {
        if (run->profiling)
            run->prof.particles_pushed += run->sp[s].n;
        run->sp[s].since_sort++;
    }
    TRY(launch_run_sources(run, static_cast<double>(run->step) * p.dt + 0.5 * p.dt)); // update(0.5 dt)
    FieldArgs const a = field_args(run);
    phase_begin(run, 2);
    CU(launch_camcl_fields(a, run->nblocks_field, run->L, run->field_smem, run->stream));
    phase_end(run, 1);
    run->fcur = 1 - run->fcur;
    run->dset = 1 - run->dset;
    for (int c = 0; c < p.n_cold; ++c)
        run->cold[c].cur = 1 - run->cold[c].cur;
    run->step++;
    if (collect)
        run->collected_step = run->step, run->collected_gen = run->gen;
    return H1D_OK;
}


// Domain_PC::cycle (Domain_PC.cc:79-205): predicted fields, predictor pass (particles not kept),
// re-predicted fields, corrector pass, corrected fields.  Deposit set X = dset takes the
// predictor's deposit, Y = 1 - dset the corrector's; each field phase clears the set the next
// particle pass uses.
// the field arguments of predictor-corrector phase `phase` (0: initial sources, 1: B1 and E1
// predicted, 2: re-predicted, 3: corrected) reading deposit set raw_set and clearing zero_set
FieldArgs pc_field_args(h1d_run *run, int phase, int raw_set, int zero_set, double const *E1_in, double *E1_out)
{
    FieldArgs a = field_args(run);
    for (int s = 0; s < run->p.n_kinetic; ++s)
        for (int d = 0; d < 2; ++d)
            for (int q = 0; q < 4; ++q) {
                a.k[s].raw[d][q]  = dep_ptr(run, s, raw_set, d, q);
                a.k[s].zero[d][q] = dep_ptr(run, s, zero_set, d, q);
            }
    a.phase = phase;
    if (phase != 3) {
        a.charge_in  = run->charge + PAD;
        a.current_in = run->current + 3 * PAD;
    }
    a.E1_in  = E1_in ? E1_in + 3 * PAD : nullptr;
    a.E1_out = E1_out ? E1_out + 3 * PAD : nullptr;
    return a;
}

int pc_launch_fields(h1d_run *run, int phase, int raw_set, int zero_set, double const *E1_in, double *E1_out)
{
    FieldArgs const a = pc_field_args(run, phase, raw_set, zero_set, E1_in, E1_out);
    phase_begin(run, 2);
    CU(launch_pc_fields(a, run->nblocks_field, run->L, run->field_smem, run->stream));
    phase_end(run, 1);
    return H1D_OK;
}

// the particle-pass arguments of species s in predictor-corrector pass `pass` (0 predictor:
// particles not kept; 1 corrector; 2 initial deposit only), depositing into set dep_set
PushArgs pc_pass_args(h1d_run *run, int s, int pass, int dep_set)
{
    PushArgs a = push_args(run, s);
    for (int q = 0; q < 4; ++q)
        a.dep[0][q] = dep_ptr(run, s, dep_set, 0, q), a.dep[1][q] = dep_ptr(run, s, dep_set, 1, q);
    a.move_steps   = pass == 2 ? 0 : 2;
    a.deposit_mask = 2;
    a.write_back   = pass == 1;
    a.travel_scale = 1.0 / 0.5;
    a.counter      = static_cast<uint64_t>(run->step) * 8 + (pass == 1 ? 2 : 0);
    return a;
}

int pc_particles(h1d_run *run, int pass, int dep_set) // pass 0 predictor, 1 corrector, 2 initial deposit
{
    if (pass != 2)
        TRY(sort_due(run));
    TRY(push_run(run, [&](int s) { return pc_pass_args(run, s, pass, dep_set); }));
    for (int s = 0; s < run->p.n_kinetic; ++s) {
        if (run->profiling)
            run->prof.particles_pushed += run->sp[s].n;
        if (pass == 1)
            run->sp[s].since_sort++;
    }
    return H1D_OK;
}

int pc_initial_sources(h1d_run *run) // Domain_PC.cc:36-56
{
    int const X = run->dset, Y = 1 - X;
    // the cold fluid's boundary_pass (Domain_PC.cc:46).  The reference updates mom1_full in place
    // and never writes its ghosts again; here the steps alternate between two nV buffers and write
    // their interiors, so both buffers get the ghosts
    int const Nx = static_cast<int>(run->Nx);
    for (int c = 0; c < run->p.n_cold; ++c) {
        ColdState &C = run->cold[c];
        double    *v = C.nV[C.cur] + 3 * PAD;
        CU(launch_ghost_fill(C.n + PAD, C.n + PAD, 1, Nx, run->stream));
        CU(launch_ghost_fill(v, v, 3, Nx, run->stream));
        CU(launch_ghost_fill(C.nV[1 - C.cur] + 3 * PAD, v, 3, Nx, run->stream));
    }
    TRY(pc_particles(run, 2, Y));
    TRY(launch_run_sources(run, static_cast<double>(run->step) * run->p.dt + 0)); // a predictor copy's update(0)
    TRY(pc_launch_fields(run, 0, Y, X, nullptr, nullptr));
    return H1D_OK;
}

int pc_step(h1d_run *run)
{
    int const X = run->dset, Y = 1 - X;
    TRY(pc_launch_fields(run, 1, X, X, nullptr, run->E1[0])); // B1, E1 predicted and averaged (clears nothing new)
    TRY(pc_particles(run, 0, X));
    TRY(launch_run_sources(run, static_cast<double>(run->step) * run->p.dt + run->p.dt)); // update(dt), both passes
    TRY(pc_launch_fields(run, 2, X, Y, run->E1[0], run->E1[1]));
    TRY(pc_particles(run, 1, Y));
    TRY(pc_launch_fields(run, 3, Y, X, run->E1[1], nullptr));
    run->fcur = 1 - run->fcur;
    for (int c = 0; c < run->p.n_cold; ++c)
        run->cold[c].cur = 1 - run->cold[c].cur;
    run->step++;
    return H1D_OK;
}

// The C-ABI status of a device status word and its message: the first of its bits in the order
// moved too far, timeout, outside the grid / non-finite; a bit the kernels do not define is a CUDA
// error.
int status_of_bits(unsigned s, std::string &msg)
{
    if (s & ST_MOVED_TOO_FAR)
        return msg = "PartSpecies::update_pos - particle(s) moved too far", H1D_ERR_MOVED_TOO_FAR;
    if (s & ST_TIMEOUT)
        return msg = "a particle-pipeline barrier wait timed out", H1D_ERR_TIMEOUT;
    if (s & (ST_OUT_OF_RANGE | ST_NAN))
        return msg = "particle(s) outside the padded grid (non-finite or lost particle state)", H1D_ERR_NAN;
    if (s)
        return msg = fmt("device status 0x%x", s), H1D_ERR_CUDA;
    return H1D_OK;
}

int check_status(h1d_run *run)
{
    CU(cudaStreamSynchronize(run->stream));
    CU(cudaMemcpy(run->h_status, run->d_status, sizeof(unsigned), cudaMemcpyDeviceToHost));
    std::string m;
    if (int const st = status_of_bits(*run->h_status, m))
        return set_err(run, st, m);
    return H1D_OK;
}

// post-process of advance_by: collect_all + boundary_gather (Domain_CAMCL.cc:45-55), on demand
int finalize_moments(h1d_run *run)
{
    if (!run->moments_stale)
        return H1D_OK;
    h1d_params const &p = run->p;
    if (fused_collect(run) && run->collected_step == run->step && run->collected_gen == run->gen) {
        // the last step's pass formed the sums: n and nV are its end-position deposit, which
        // the field kernel of that step read and left in place (it clears the other set)
        int const set = 1 - run->dset;
        for (int s = 0; s < p.n_kinetic; ++s) {
            SpeciesState &S = run->sp[s];
            for (int q = 0; q < 4; ++q)
                CU(cudaMemcpyAsync(S.mom_raw + static_cast<size_t>(q) * run->M, dep_ptr(run, s, set, 1, q) - PAD,
                                   sizeof(double) * run->M, cudaMemcpyDeviceToDevice, run->stream));
            CU(launch_finalize_kinetic(S.mom_raw, S.eq, S.mom, static_cast<int>(run->Nx), 1.0 / p.kinetic[s].moment_norm,
                                       p.particle_bc == H1D_BC_PERIODIC ? 0 : 1, run->stream));
        }
        for (int c = 0; c < p.n_cold; ++c) {
            ColdState &C = run->cold[c];
            CU(launch_finalize_cold(C.n, C.nV[C.cur], C.mom, static_cast<int>(run->Nx), p.moment_weighting,
                                    run->stream));
        }
        CU(cudaGetLastError());
        run->moments_stale = false;
        return H1D_OK;
    }
    // particles that drifted since their last sort are sorted first: a warp's particles then
    // share a few cells and collect_all accumulates in registers (the next steps gain too)
    std::vector<SortItem> drifted;
    for (int s = 0; s < p.n_kinetic; ++s)
        if (run->sp[s].n > 0 && run->sp[s].since_sort > 0)
            drifted.push_back({ run, s });
    TRY(sort_run(run, drifted));
    for (int s = 0; s < p.n_kinetic; ++s) {
        SpeciesState &S = run->sp[s];
        CU(cudaMemsetAsync(S.mom_raw, 0, sizeof(double) * 10 * run->M, run->stream));
        if (S.n > 0 && run->mixed) {
            MomentArgsMixed a{};
            a.pos = S.pos[S.cur], a.vx = S.fbuf[S.cur][0], a.vy = S.fbuf[S.cur][1], a.vz = S.fbuf[S.cur][2];
            a.w = S.fbuf[S.cur][3], a.n = S.n, a.ppt = ppt_for(run, s), a.vec = 1;
            a.fbits = run->fbits, a.inv_scale = static_cast<float>(1 / run->pos_scale);
            a.Nx = static_cast<int>(run->Nx), a.status = run->d_status;
            for (int q = 0; q < 10; ++q)
                a.out[q] = S.mom_raw + static_cast<size_t>(q) * run->M + PAD;
            int64_t const chunks = (S.n + 32LL * a.ppt - 1) / (32LL * a.ppt);
            moments_kernel<<<static_cast<unsigned>((chunks + 3) / 4), MOM_THREADS, 0, run->stream>>>(a);
        } else if (S.n > 0) {
            MomentArgs a{};
            a.q1 = S.buf[S.cur][0], a.vx = S.buf[S.cur][1], a.vy = S.buf[S.cur][2], a.vz = S.buf[S.cur][3];
            a.w = S.buf[S.cur][4], a.n = S.n, a.ppt = ppt_for(run, s), a.Nx = static_cast<int>(run->Nx), a.vec = 1;
            a.half_min = -0.5 * p.Nx + 0.5, a.status = run->d_status;
            for (int q = 0; q < 10; ++q)
                a.out[q] = S.mom_raw + static_cast<size_t>(q) * run->M + PAD;
            int64_t const chunks = (S.n + 32LL * a.ppt - 1) / (32LL * a.ppt);
            moments_kernel<<<static_cast<unsigned>((chunks + 3) / 4), MOM_THREADS, 0, run->stream>>>(a);
        }
        CU(launch_finalize_kinetic(S.mom_raw, S.eq, S.mom, static_cast<int>(run->Nx), 1.0 / p.kinetic[s].moment_norm,
                                   p.particle_bc == H1D_BC_PERIODIC ? 0 : 1, run->stream));
    }
    for (int c = 0; c < p.n_cold; ++c) {
        ColdState &C = run->cold[c];
        CU(launch_finalize_cold(C.n, C.nV[C.cur], C.mom, static_cast<int>(run->Nx), p.moment_weighting,
                                run->stream));
    }
    CU(cudaGetLastError());
    run->moments_stale = false;
    return H1D_OK;
}

__global__ void math_check_kernel(double const *x, int64_t n, double *out)
{
    int64_t const k = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (k >= n)
        return;
    double const v = x[k];
    out[5 * k + 0] = floor_ir(v).d + 0.0 * floor_ir(v).i;
    out[5 * k + 1] = static_cast<double>(round_ir(v).i);
    out[5 * k + 2] = static_cast<double>(ceil_ir(v).i);
    double s, c;
    sincos_taylor(v, s, c);
    out[5 * k + 3] = s;
    out[5 * k + 4] = c;
    if (floor_ir(v).d != static_cast<double>(floor_ir(v).i)) // integer and real parts must agree
        out[5 * k + 0] = __longlong_as_double(0x7ff8000000000000LL);
}

// Fixed scratch of h1d_collect_moments_noalloc: raw sums (10 x M), finalized moments (10 x M) and a
// status word.  Host code must not use the symbol as a pointer; it looks up the device address
// with cudaGetSymbolAddress, once per device.
constexpr int64_t NOALLOC_M = H1D_NOALLOC_MAX_NX + 2 * PAD;
static __device__ __align__(256) double noalloc_scratch[20 * NOALLOC_M + 2];

constexpr int NOALLOC_MAX_DEVICES = 64;
std::mutex    noalloc_mutex;
double       *noalloc_addr[NOALLOC_MAX_DEVICES] = {};

int noalloc_scratch_address(double **out)
{
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess)
        return H1D_ERR_NO_DEVICE;
    if (dev < 0 || dev >= NOALLOC_MAX_DEVICES)
        return H1D_ERR_INVALID_ARG;
    std::lock_guard<std::mutex> lock(noalloc_mutex);
    if (!noalloc_addr[dev]) {
        void *p = nullptr;
        if (cudaGetSymbolAddress(&p, noalloc_scratch) != cudaSuccess || !p)
            return H1D_ERR_CUDA;
        noalloc_addr[dev] = static_cast<double *>(p);
    }
    *out = noalloc_addr[dev];
    return H1D_OK;
}


// device storage for n particles of species s (both buffer sets and the sort scratch)
int ensure_capacity(h1d_run *run, int s, int64_t n)
{
    SpeciesState &S = run->sp[s];
    if (n <= S.cap)
        return H1D_OK;
    int64_t const cap = n + 64; // slack for the 16-byte rounding of the last bulk copy of a pass
    for (int k = 0; k < 2; ++k) {
        if (run->mixed) {
            for (auto *&b : S.fbuf[k]) {
                dfree(b);
                b = nullptr;
                CU(dmalloc(&b, sizeof(float) * cap));
            }
            dfree(S.pos[k]);
            S.pos[k] = nullptr;
            CU(dmalloc(&S.pos[k], sizeof(int32_t) * cap));
            if (evolves_psd(run->p.kinetic[s]))
                for (auto *&b : S.fpsd[k]) {
                    dfree(b);
                    b = nullptr;
                    CU(dmalloc(&b, sizeof(float) * cap));
                }
        } else {
            for (auto *&b : S.buf[k]) {
                dfree(b);
                b = nullptr;
                CU(dmalloc(&b, sizeof(double) * cap));
            }
            if (evolves_psd(run->p.kinetic[s]))
                for (auto *&b : S.psd[k]) {
                    dfree(b);
                    b = nullptr;
                    CU(dmalloc(&b, sizeof(double) * cap));
                }
        }
        dfree(S.pid[k]), dfree(S.keys[k]), dfree(S.idx[k]);
        S.pid[k] = nullptr, S.keys[k] = nullptr, S.idx[k] = nullptr;
        CU(dmalloc(&S.pid[k], sizeof(int32_t) * cap));
        CU(dmalloc(&S.keys[k], sizeof(uint32_t) * cap));
        CU(dmalloc(&S.idx[k], sizeof(uint32_t) * cap));
    }
    S.cap = cap;
    return H1D_OK;
}

// MaxwellianVDF::N_of_q1 (VDF/MaxwellianVDF.cc:44-54)
double n_of_q1(h1d_params const &p, double T2OT1, double q1)
{
    if (p.xi < 1e-10) {
        double const xiD1q1 = p.xi * p.Dx * q1;
        return q1 * (1 - (xiD1q1 * xiD1q1) * (T2OT1 - 1) / 3);
    }
    double const s = std::sqrt(T2OT1);
    return std::atan(s * std::tan(p.xi * p.Dx * q1)) / (s * p.Dx * p.xi);
}


// ------------------------------------------------------------------------------------------------
// Ensembles (h1d_batch_*): many CAM-CL runs advanced together on one stream.  A step is one
// launch of the particle pass per kind of group (shape order, geometry, boundary, precision) over
// every species of every member, then one launch of the field cycle over every member's grid.
// Steps come in blocks of sort_interval steps; every group is cell-sorted at the start of a block.
// Two blocks restore every ping-pong parity, so a pair of blocks is captured once as a CUDA graph
// and replayed while the members' state signature is unchanged.
// ------------------------------------------------------------------------------------------------
} // namespace

struct h1d_batch {
    std::vector<h1d_run *>     runs;
    std::vector<cudaStream_t>  saved;
    cudaStream_t               stream = nullptr;
    int                        device = 0, num_sms = 148;
    int                        k = 16;          // sort interval = steps per block
    int                        ctas = 0;        // CTAs per SM of the particle pass (0: defaults)
    bool                       use_graphs = true;
    int                        since_block = 1 << 30;
    int                        L = 0, nblocks = 0;
    size_t                     smem = 0;
    bool                       pc = false;        // predictor-corrector members (else CAM-CL)
    SortScratch                sorter;            // the members' cell sort
    FieldArgs                 *d_table = nullptr; // CAM-CL: [parity][runs]; PC: [phase 1-3][parity][runs]
    FieldBlock                *d_map = nullptr;
    std::vector<FieldBlock>    map_all, map_live;  // every member's field blocks / those launched now
    std::vector<char>          active;             // members the next steps advance (all when empty)
    int                        parity = 0;
    cudaGraph_t                graph = nullptr;
    cudaGraphExec_t            exec = nullptr;
    std::vector<int64_t>       graph_sig;
    int64_t                    graph_kernels = 0;
    bool                       capturing = false, graphs_warm = false;
    h1d_batch_stats            stats{};
    std::string                msg;
};

namespace {

int bset_err(h1d_batch *b, int code, std::string const &m)
{
    if (b)
        b->msg = m;
    return code;
}
#define BCU(call)                                                                                            \
    do {                                                                                                     \
        cudaError_t const e_ = (call);                                                                       \
        if (e_ != cudaSuccess)                                                                               \
            return bset_err(b, e_ == cudaErrorMemoryAllocation ? H1D_ERR_OOM : H1D_ERR_CUDA,                 \
                            fmt("%s: %s (%s:%d)", #call, cudaGetErrorString(e_), __FILE__, __LINE__));       \
    } while (0)
#define BTRY(r, x)                                                                                           \
    do {                                                                                                     \
        int const st_ = (x);                                                                                 \
        if (st_ != H1D_OK)                                                                                   \
            return bset_err(b, st_, (r)->msg);                                                               \
    } while (0)

// whether member i takes the next step (every member, unless an advance by member counts runs)
bool member_on(h1d_batch const *b, size_t i) { return b->active.empty() || b->active[i]; }

bool graph_eligible(h1d_batch const *b)
{
    if (!b->use_graphs)
        return false;
    for (h1d_run const *r : b->runs) // host-side trims and per-step draws and times are not capturable
        if (r->p.particle_bc == H1D_BC_ABSORBING || r->p.randomize_gyrophase || r->p.n_sources > 0)
            return false;
    return true;
}

// everything a captured pair of blocks depends on
std::vector<int64_t> batch_signature(h1d_batch const *b)
{
    std::vector<int64_t> sig{ b->k, b->ctas, b->parity, static_cast<int64_t>(b->runs.size()) };
    for (h1d_run const *r : b->runs) {
        sig.push_back(static_cast<int64_t>(r->gen));
        sig.push_back(r->fcur), sig.push_back(r->dset);
        for (int c = 0; c < r->p.n_cold; ++c)
            sig.push_back(r->cold[c].cur);
        for (int s = 0; s < r->p.n_kinetic; ++s)
            sig.push_back(r->sp[s].cur), sig.push_back(r->sp[s].n);
    }
    return sig;
}

void drop_graph(h1d_batch *b)
{
    if (b->exec)
        cudaGraphExecDestroy(b->exec);
    if (b->graph)
        cudaGraphDestroy(b->graph);
    b->exec = nullptr, b->graph = nullptr;
    b->graph_sig.clear();
}

// field launch geometry shared by the members (one block size) and the per-parity argument tables
int build_field_tables(h1d_batch *b)
{
    int L = FIELD_BLOCK_MIN;
    for (h1d_run const *r : b->runs)
        L = std::max(L, r->L);
    std::vector<FieldArgs>  tab((b->pc ? 6 : 2) * b->runs.size());
    std::vector<FieldBlock> map;
    for (size_t i = 0; i < b->runs.size(); ++i) {
        h1d_run *r   = b->runs[i];
        int const seg = static_cast<int>(std::min<long>(L - 2 * r->H, r->Nx));
        int const nb  = static_cast<int>((r->Nx + seg - 1) / seg);
        for (int blk = 0; blk < nb; ++blk)
            map.push_back({ static_cast<int>(i), blk });
        for (int par = 0; par < 2; ++par) {
            auto const flip = [&] { // the state after one step (a PC step keeps its deposit sets)
                r->fcur ^= 1;
                if (!b->pc)
                    r->dset ^= 1;
                for (int c = 0; c < r->p.n_cold; ++c)
                    r->cold[c].cur ^= 1;
            };
            if (par)
                flip();
            if (b->pc) { // the three field phases of pc_step
                int const X = r->dset, Y = 1 - X;
                FieldArgs ph[3] = { pc_field_args(r, 1, X, X, nullptr, r->E1[0]),
                                    pc_field_args(r, 2, X, Y, r->E1[0], r->E1[1]),
                                    pc_field_args(r, 3, Y, X, r->E1[1], nullptr) };
                for (int f = 0; f < 3; ++f) {
                    ph[f].seg = seg;
                    tab[(f * 2 + par) * b->runs.size() + i] = ph[f];
                }
            } else {
                FieldArgs a = field_args(r);
                a.seg       = seg;
                tab[par * b->runs.size() + i] = a;
            }
            if (par)
                flip();
        }
    }
    int const    fb   = field_group(L, FIELD_SMEM_BATCH);
    for (FieldArgs &a : tab)
        a.fb = fb;
    size_t const smem = field_smem_bytes(L, fb);
    if (L != b->L || static_cast<int>(map.size()) != b->nblocks || !b->d_table) {
        dfree(b->d_table), dfree(b->d_map);
        b->d_table = nullptr, b->d_map = nullptr;
        BCU(dmalloc(&b->d_table, sizeof(FieldArgs) * tab.size()));
        BCU(dmalloc(&b->d_map, sizeof(FieldBlock) * map.size()));
        BCU(set_field_batch_smem(smem));
        drop_graph(b);
    }
    b->L = L, b->nblocks = static_cast<int>(map.size()), b->smem = smem, b->parity = 0;
    b->map_all = map, b->active.clear();
    BCU(cudaMemcpyAsync(b->d_table, tab.data(), sizeof(FieldArgs) * tab.size(), cudaMemcpyHostToDevice, b->stream));
    BCU(cudaMemcpyAsync(b->d_map, map.data(), sizeof(FieldBlock) * map.size(), cudaMemcpyHostToDevice, b->stream));
    BCU(cudaStreamSynchronize(b->stream));
    return H1D_OK;
}

// sort every species of every member at the start of a block of b->k steps, all of them in one
// launch set per kind (precision, evolving weights) of up to SORT_SEGS species
int batch_sort_block(h1d_batch *b)
{
    if (b->since_block >= b->k) {
        std::vector<SortItem> items;
        for (size_t i = 0; i < b->runs.size(); ++i)
            if (member_on(b, i))
                for (int s = 0; s < b->runs[i]->p.n_kinetic; ++s)
                    items.push_back({ b->runs[i], s });
        if (!items.empty())
            BCU(sort_items(items, b->sorter, b->stream, b->stats.kernel_launches));
        b->since_block = 0;
    }
    return H1D_OK;
}

// one particle pass of every member: one launch per kind of group, and one per species whose
// weights evolve; `pass` < 0 is the CAM-CL pass, else the predictor-corrector pass of pc_pass_args
int batch_push(h1d_batch *b, int pass)
{
    struct Kind {
        int  order, bc;
        bool mirror, mixed;
        bool operator==(Kind const &o) const
        {
            return order == o.order && bc == o.bc && mirror == o.mirror && mixed == o.mixed;
        }
    };
    std::vector<Kind>                       kinds;
    std::vector<std::vector<PushArgs>>      fp;
    std::vector<std::vector<PushArgsMixed>> mx;
    for (size_t i = 0; i < b->runs.size(); ++i) {
        if (!member_on(b, i))
            continue;
        h1d_run *r = b->runs[i];
        for (int s = 0; s < r->p.n_kinetic; ++s) {
            if (r->sp[s].n == 0)
                continue;
            int const      X = r->dset;
            PushArgs const a = pass < 0 ? push_args(r, s) : pc_pass_args(r, s, pass, pass == 1 ? 1 - X : X);
            if (evolves_psd(r->p.kinetic[s])) { // the weight-evolving pass, one species per launch
                BTRY(r, launch_push(r, s, a));
                b->stats.kernel_launches += 1;
                continue;
            }
            Kind const kd{ static_cast<int>(r->p.kinetic[s].shape_order), r->p.particle_bc, r->p.xi != 0, r->mixed };
            size_t     ki = 0;
            while (ki < kinds.size() && !(kinds[ki] == kd))
                ++ki;
            if (ki == kinds.size())
                kinds.push_back(kd), fp.emplace_back(), mx.emplace_back();
            if (kd.mixed)
                mx[ki].push_back(mixed_args(r, s, a));
            else
                fp[ki].push_back(a);
        }
    }
    for (size_t ki = 0; ki < kinds.size(); ++ki) {
        Kind const &kd = kinds[ki];
        if (kd.mixed)
            BCU(launch_push_groups(mx[ki].data(), static_cast<int>(mx[ki].size()), kd.order, kd.mirror, kd.bc,
                                   b->num_sms * (b->ctas ? b->ctas : PIPE_CTAS_PER_SM_MIXED), b->stream));
        else
            BCU(launch_push_groups(fp[ki].data(), static_cast<int>(fp[ki].size()), kd.order, kd.mirror, kd.bc,
                                   b->num_sms * (b->ctas ? std::min(b->ctas, PIPE_CTAS_PER_SM) : PIPE_CTAS_PER_SM),
                                   b->stream));
        size_t const groups = kd.mixed ? mx[ki].size() : fp[ki].size();
        b->stats.kernel_launches += static_cast<int64_t>((groups + BATCH_GROUPS - 1) / BATCH_GROUPS);
    }
    return H1D_OK;
}

// the host side of one step of every member
void batch_step_done(h1d_batch *b)
{
    for (size_t i = 0; i < b->runs.size(); ++i) {
        if (!member_on(b, i))
            continue;
        h1d_run *r = b->runs[i];
        r->fcur ^= 1;
        if (!b->pc)
            r->dset ^= 1;
        for (int c = 0; c < r->p.n_cold; ++c)
            r->cold[c].cur ^= 1;
        for (int s = 0; s < r->p.n_kinetic; ++s)
            r->sp[s].since_sort++;
        r->step++;
        r->moments_stale = true;
    }
    b->parity ^= 1;
    b->since_block++;
    b->stats.steps++;
}

// one Domain_PC::cycle of every member (pc_step): three batched field phases around the predictor
// and corrector particle passes
int batch_step_pc(h1d_batch *b)
{
    TRY(batch_sort_block(b));
    size_t const R     = b->runs.size();
    auto const   table = [&](int phase) { return b->d_table + ((phase - 1) * 2 + b->parity) * R; };
    BCU(launch_pc_fields_batch(table(1), b->d_map, b->nblocks, b->L, b->smem, b->stream));
    TRY(batch_push(b, 0));
    for (size_t i = 0; i < b->runs.size(); ++i)
        if (h1d_run *r = b->runs[i]; member_on(b, i) && r->p.n_sources > 0) {
            BTRY(r, launch_run_sources(r, static_cast<double>(r->step) * r->p.dt + r->p.dt));
            b->stats.kernel_launches += 1;
        }
    BCU(launch_pc_fields_batch(table(2), b->d_map, b->nblocks, b->L, b->smem, b->stream));
    TRY(batch_push(b, 1));
    BCU(launch_pc_fields_batch(table(3), b->d_map, b->nblocks, b->L, b->smem, b->stream));
    b->stats.kernel_launches += 3;
    batch_step_done(b);
    return H1D_OK;
}

// one CAM-CL step of every member (sorting all groups first at a block start)
int batch_step(h1d_batch *b)
{
    if (b->pc)
        return batch_step_pc(b);
    TRY(batch_sort_block(b));
    TRY(batch_push(b, -1));
    // external sources of the members that have them, then the field cycle of every member
    for (size_t i = 0; i < b->runs.size(); ++i)
        if (h1d_run *r = b->runs[i]; member_on(b, i) && r->p.n_sources > 0) {
            BTRY(r, launch_run_sources(r, static_cast<double>(r->step) * r->p.dt + 0.5 * r->p.dt));
            b->stats.kernel_launches += 1;
        }
    BCU(launch_camcl_fields_batch(b->d_table + b->parity * b->runs.size(), b->d_map, b->nblocks, b->L, b->smem,
                                  b->stream));
    b->stats.kernel_launches += 1;
    batch_step_done(b);
    return H1D_OK;
}

// the members' first advance: ghost cells of E and B and the push record
int batch_prepare(h1d_batch *b)
{
    for (h1d_run *r : b->runs) {
        bool const first = !r->recurring;
        if (first || r->fields_dirty) {
            BTRY(r, prepare_fields(r));
            b->stats.kernel_launches += 1;
        }
        if (first && r->p.algorithm == H1D_ALGO_PC) // Domain_PC::advance_by's initial sources
            BTRY(r, pc_initial_sources(r));
        r->recurring = true;
    }
    return H1D_OK;
}

int batch_advance(h1d_batch *b, uint32_t n_steps)
{
    if (n_steps == 0)
        return H1D_OK;
    for (h1d_run *r : b->runs)
        r->profiling = false; // phase events are not recorded inside a batch
    if (int const st = batch_prepare(b))
        return st;
    if (int const st = build_field_tables(b))
        return st;
    uint32_t left = n_steps;
    // finish the current block eagerly
    for (; left > 0 && b->since_block < b->k; --left)
        if (int const st = batch_step(b))
            return st;
    uint32_t const pair = 2u * static_cast<uint32_t>(b->k);
    if (graph_eligible(b)) {
        while (left >= pair) {
            std::vector<int64_t> const sig = batch_signature(b);
            if (b->exec && sig == b->graph_sig) {
                BCU(cudaGraphLaunch(b->exec, b->stream));
                for (h1d_run *r : b->runs) { // the host side of the replayed steps
                    r->step += pair;
                    for (int s = 0; s < r->p.n_kinetic; ++s)
                        r->sp[s].since_sort = b->k;
                    r->moments_stale = true;
                }
                b->stats.graph_launches++;
                b->stats.kernel_launches += b->graph_kernels;
                b->stats.steps += pair;
                left -= pair;
                continue;
            }
            if (b->exec) { // the members changed: the next capture follows an eager pair again
                drop_graph(b);
                b->graphs_warm = false;
            }
            if (!b->graphs_warm) { // a first eager pair sizes every scratch buffer
                for (uint32_t i = 0; i < pair; ++i)
                    if (int const st = batch_step(b))
                        return st;
                b->graphs_warm = true;
                left -= pair;
                continue;
            }
            int64_t const k0 = b->stats.kernel_launches, s0 = b->stats.steps;
            BCU(cudaStreamBeginCapture(b->stream, cudaStreamCaptureModeThreadLocal));
            b->capturing = true;
            int st       = H1D_OK;
            for (uint32_t i = 0; i < pair && st == H1D_OK; ++i)
                st = batch_step(b);
            cudaGraph_t       g  = nullptr;
            cudaError_t const ec = cudaStreamEndCapture(b->stream, &g);
            b->capturing         = false;
            if (st != H1D_OK) {
                if (g)
                    cudaGraphDestroy(g);
                return st;
            }
            BCU(ec);
            b->graph = g;
            BCU(cudaGraphInstantiate(&b->exec, g, 0));
            b->graph_kernels = b->stats.kernel_launches - k0;
            b->stats.kernel_launches = k0, b->stats.steps = s0;
            // the capture advanced the host state by a pair; the signature is that of its start
            b->graph_sig = sig;
            b->stats.graphs_built++;
            BCU(cudaGraphLaunch(b->exec, b->stream));
            b->stats.graph_launches++;
            b->stats.kernel_launches += b->graph_kernels;
            b->stats.steps += pair;
            left -= pair;
        }
    }
    for (; left > 0; --left)
        if (int const st = batch_step(b))
            return st;
    return H1D_OK;
}

// the members the next steps advance (on[i] != 0), and the field launch's blocks to match: the
// block map keeps only their blocks (each block still names its member's table entry)
int batch_set_active(h1d_batch *b, std::vector<char> const &on)
{
    b->active = on;
    b->map_live.clear();
    for (FieldBlock const &f : b->map_all)
        if (on[static_cast<size_t>(f.run)])
            b->map_live.push_back(f);
    b->nblocks = static_cast<int>(b->map_live.size());
    if (b->nblocks > 0)
        BCU(cudaMemcpyAsync(b->d_map, b->map_live.data(), sizeof(FieldBlock) * b->map_live.size(),
                            cudaMemcpyHostToDevice, b->stream));
    return H1D_OK;
}
int batch_set_all(h1d_batch *b)
{
    b->active.clear();
    b->nblocks = static_cast<int>(b->map_all.size());
    if (b->nblocks > 0)
        BCU(cudaMemcpyAsync(b->d_map, b->map_all.data(), sizeof(FieldBlock) * b->map_all.size(),
                            cudaMemcpyHostToDevice, b->stream));
    return H1D_OK;
}

// advance member i by steps[i] (eager steps): every member steps until the smallest count is
// reached, that member drops out of the particle passes, the sorts and the field launch, and the
// others go on; each member's state is then that of its own advance_by(steps[i])
int batch_advance_members(h1d_batch *b, uint32_t const *steps)
{
    size_t const R = b->runs.size();
    uint32_t     n = 0;
    for (size_t i = 0; i < R; ++i)
        n = std::max(n, steps[i]);
    bool uniform = true;
    for (size_t i = 0; i < R; ++i)
        uniform = uniform && steps[i] == n;
    if (uniform)
        return batch_advance(b, n);
    for (h1d_run *r : b->runs)
        r->profiling = false;
    std::vector<h1d_run *> moving;
    for (size_t i = 0; i < R; ++i)
        if (steps[i] > 0)
            moving.push_back(b->runs[i]);
    std::vector<h1d_run *> const all = b->runs;
    b->runs                          = moving; // members that do not step are not prepared either
    int st                           = batch_prepare(b);
    b->runs                          = all;
    if (st != H1D_OK)
        return st;
    TRY(build_field_tables(b));
    std::vector<char> on(R, 0);
    uint32_t          done = 0;
    while (st == H1D_OK && done < n) {
        uint32_t next = n; // the next count at which a member stops
        for (size_t i = 0; i < R; ++i) {
            on[i] = steps[i] > done;
            if (on[i])
                next = std::min(next, steps[i]);
        }
        st = batch_set_active(b, on);
        for (; st == H1D_OK && done < next; ++done)
            st = batch_step(b);
    }
    int const back = batch_set_all(b);
    return st != H1D_OK ? st : back;
}

int batch_check(h1d_batch *b)
{
    BCU(cudaStreamSynchronize(b->stream));
    for (h1d_run *r : b->runs)
        if (int const st = check_status(r))
            return bset_err(b, st, fmt("member run %p: %s", static_cast<void *>(r), r->msg.c_str()));
    return H1D_OK;
}

// time `steps` batch steps (eager, whole blocks) in milliseconds
int batch_time(h1d_batch *b, uint32_t steps, float *ms)
{
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    BCU(cudaEventCreate(&e0));
    BCU(cudaEventCreate(&e1));
    int st = H1D_OK;
    if (cudaEventRecord(e0, b->stream) != cudaSuccess)
        st = bset_err(b, H1D_ERR_CUDA, "event record failed");
    for (uint32_t i = 0; i < steps && st == H1D_OK; ++i)
        st = batch_step(b);
    if (st == H1D_OK && (cudaEventRecord(e1, b->stream) != cudaSuccess || cudaEventSynchronize(e1) != cudaSuccess
                         || cudaEventElapsedTime(ms, e0, e1) != cudaSuccess))
        st = bset_err(b, H1D_ERR_CUDA, "event timing failed");
    cudaEventDestroy(e0), cudaEventDestroy(e1);
    if (st == H1D_OK)
        st = batch_check(b);
    return st;
}

} // namespace

// ------------------------------------------------------------------------------------------------
// C-ABI
// ------------------------------------------------------------------------------------------------
extern "C" {

int    h1d_abi_version(void) { return H1D_ABI_VERSION; }
size_t h1d_params_size(void) { return sizeof(h1d_params); }

char const *h1d_error_name(int status)
{
    switch (status) {
    case H1D_OK: return "ok";
    case H1D_ERR_INVALID_ARG: return "invalid argument";
    case H1D_ERR_MOVED_TOO_FAR: return "particle(s) moved too far";
    case H1D_ERR_OOM: return "out of device memory";
    case H1D_ERR_CUDA: return "CUDA error";
    case H1D_ERR_TIMEOUT: return "timeout";
    case H1D_ERR_NAN: return "non-finite state";
    case H1D_ERR_STATE: return "call out of order";
    case H1D_ERR_NO_DEVICE: return "no CUDA device";
    default: return "unknown";
    }
}

char const *h1d_status_string(h1d_run *run) { return run ? run->msg.c_str() : "null run"; }

int h1d_math_check(double const *x, int64_t n, double *out)
{
    if (n < 0 || (n > 0 && (!x || !out)))
        return H1D_ERR_INVALID_ARG;
    if (n == 0)
        return H1D_OK;
    double *dx = nullptr, *dout = nullptr;
    if (dmalloc(&dx, sizeof(double) * n) != cudaSuccess || dmalloc(&dout, sizeof(double) * 5 * n) != cudaSuccess) {
        dfree(dx);
        return H1D_ERR_OOM;
    }
    int st = H1D_OK;
    if (cudaMemcpy(dx, x, sizeof(double) * n, cudaMemcpyHostToDevice) != cudaSuccess)
        st = H1D_ERR_CUDA;
    if (st == H1D_OK) {
        math_check_kernel<<<static_cast<unsigned>((n + 255) / 256), 256>>>(dx, n, dout);
        if (cudaGetLastError() != cudaSuccess
            || cudaMemcpy(out, dout, sizeof(double) * 5 * n, cudaMemcpyDeviceToHost) != cudaSuccess)
            st = H1D_ERR_CUDA;
    }
    dfree(dx);
    dfree(dout);
    return st;
}

int h1d_collect_moments_noalloc(int64_t Nx, double moment_norm, int particle_bc, double const *q1, double const *vx,
                                double const *vy, double const *vz, double const *w, int64_t n, double *n_out,
                                double *nV_out, double *nvv_out, void *stream)
{
    if (Nx < 2 * PAD || Nx > H1D_NOALLOC_MAX_NX) {
        std::fprintf(stderr, "h1d_collect_moments_noalloc: Nx = %lld is outside [%d, %d], the size of its fixed scratch\n",
                     static_cast<long long>(Nx), 2 * PAD, H1D_NOALLOC_MAX_NX);
        return H1D_ERR_INVALID_ARG;
    }
    if (!(moment_norm > 0) || n < 0 || n > (int64_t{ 1 } << 31) - 1 || particle_bc < 0 || particle_bc > 2
        || (n > 0 && (!q1 || !vx || !vy || !vz || !w)) || !n_out || !nV_out || !nvv_out)
        return H1D_ERR_INVALID_ARG;
    double *scratch = nullptr;
    if (int const st = noalloc_scratch_address(&scratch))
        return st;
    cudaStream_t const st     = static_cast<cudaStream_t>(stream);
    int64_t const      M      = Nx + 2 * PAD;
    double            *raw    = scratch;
    double            *fin    = scratch + 10 * M;
    unsigned          *status = reinterpret_cast<unsigned *>(scratch + 20 * NOALLOC_M);
    // a failure after work was queued waits for that work first, so that a failed call leaves
    // nothing running on the shared scratch
    auto const fail = [st] {
        cudaStreamSynchronize(st);
        return H1D_ERR_CUDA;
    };
    // the raw sums are accumulated with atomics and must start at zero, as must the status word
    if (cudaMemsetAsync(raw, 0, sizeof(double) * 10 * M, st) != cudaSuccess
        || cudaMemsetAsync(status, 0, sizeof(unsigned), st) != cudaSuccess)
        return fail();
    if (n > 0) {
        MomentArgs a{};
        a.q1 = q1, a.vx = vx, a.vy = vy, a.vz = vz, a.w = w, a.n = n, a.Nx = static_cast<int>(Nx);
        double const ppc = static_cast<double>(n) / static_cast<double>(Nx);
        a.ppt            = mom_ppt(ppc);
        auto const al16  = [](void const *p) { return (reinterpret_cast<uintptr_t>(p) & 15) == 0; };
        a.vec            = al16(q1) && al16(vx) && al16(vy) && al16(vz) && al16(w); // caller buffers
        a.half_min       = -0.5 * static_cast<double>(Nx) + 0.5;
        a.status         = status;
        for (int q = 0; q < 10; ++q)
            a.out[q] = raw + static_cast<int64_t>(q) * M + PAD;
        int64_t const chunks = (n + 32LL * a.ppt - 1) / (32LL * a.ppt);
        moments_kernel<<<static_cast<unsigned>((chunks + 3) / 4), MOM_THREADS, 0, st>>>(a);
        if (cudaGetLastError() != cudaSuccess)
            return fail();
    }
    if (launch_finalize_kinetic(raw, nullptr, fin, static_cast<int>(Nx), 1.0 / moment_norm, particle_bc == H1D_BC_PERIODIC ? 0 : 1, st)
            != cudaSuccess
        || cudaMemcpyAsync(n_out, fin, sizeof(double) * M, cudaMemcpyDeviceToDevice, st) != cudaSuccess
        || cudaMemcpyAsync(nV_out, fin + M, sizeof(double) * 3 * M, cudaMemcpyDeviceToDevice, st) != cudaSuccess
        || cudaMemcpyAsync(nvv_out, fin + 4 * M, sizeof(double) * 6 * M, cudaMemcpyDeviceToDevice, st) != cudaSuccess)
        return fail();
    unsigned hstatus = 0;
    if (cudaMemcpyAsync(&hstatus, status, sizeof hstatus, cudaMemcpyDeviceToHost, st) != cudaSuccess
        || cudaStreamSynchronize(st) != cudaSuccess)
        return fail();
    std::string msg;
    int const   code = status_of_bits(hstatus, msg);
    if (code)
        std::fprintf(stderr, "h1d_collect_moments_noalloc: %s\n", msg.c_str());
    return code;
}

int h1d_create(h1d_params const *params, h1d_run **out)
{
    if (!out)
        return H1D_ERR_INVALID_ARG;
    *out = nullptr;
    std::string m;
    if (int const st = validate(params, m)) {
        std::fprintf(stderr, "h1d_create: %s\n", m.c_str());
        return st;
    }
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0)
        return H1D_ERR_NO_DEVICE;
    h1d_run *run = new (std::nothrow) h1d_run{};
    if (!run)
        return H1D_ERR_OOM;
    run->p = *params;
    if (!(run->p.moment_weighting > 0))
        run->p.moment_weighting = 1;
    h1d_params const &p = run->p;
    auto const        fail = [&](int st) {
        h1d_destroy(run);
        return st;
    };
    if (cudaGetDevice(&run->device) != cudaSuccess || cudaStreamCreateWithFlags(&run->stream, cudaStreamNonBlocking) != cudaSuccess)
        return fail(H1D_ERR_CUDA);
    run->Nx            = p.Nx;
    run->M             = p.Nx + 2 * PAD;
    run->sort_interval = p.sort_interval > 0 ? p.sort_interval : 16;
    // halo of the field kernel: reach of one cycle (2 x smoothing + subcycle + E*, advance, E, Bh)
    int rs = 0;
    for (int s = 0; s < p.n_kinetic; ++s)
        rs = std::max(rs, static_cast<int>(p.kinetic[s].n_smooth));
    for (int c = 0; c < p.n_cold; ++c)
        rs = std::max(rs, static_cast<int>(p.cold[c].n_smooth));
    run->H   = 2 * rs + static_cast<int>(p.n_subcycles) + 6;
    int L    = FIELD_BLOCK_MIN;
    while (L - 2 * run->H < 64 && L < 512)
        L += 64;
    if (L - 2 * run->H < 32)
        return fail(set_err(run, H1D_ERR_INVALID_ARG, "n_subcycles / smoothing counts too large for one field block"));
    run->L             = L;
    run->seg           = static_cast<int>(std::min<long>(L - 2 * run->H, run->Nx));
    run->nblocks_field = static_cast<int>((run->Nx + run->seg - 1) / run->seg);
    run->fb            = field_group(L, FIELD_SMEM_RUN);
    run->field_smem    = field_smem_bytes(L, run->fb);
    run->mixed = p.precision == H1D_PREC_MIXED;
    // the most fraction bits (at most FP32's 24) with positions in (-2, Nx + 2) cells inside an int32
    run->fbits = 24;
    while (run->fbits > 0 && ((static_cast<int64_t>(p.Nx) + 2) << run->fbits) > (int64_t{ 1 } << 31))
        --run->fbits;
    run->pos_scale = std::ldexp(1.0, run->fbits);
    run->stage_n = 1 << 16;
    for (int s = 0; s < p.n_kinetic; ++s)
        run->stage_n = std::max<int64_t>(run->stage_n, std::min<int64_t>(STAGE_N, p.Nx * std::max<int64_t>(p.kinetic[s].Nc, 0)));
    if (set_field_smem(run->field_smem) != cudaSuccess || set_push_smem_fp64() != cudaSuccess
        || set_push_smem_mixed() != cudaSuccess)
        return fail(H1D_ERR_CUDA);
    cudaDeviceGetAttribute(&run->num_sms, cudaDevAttrMultiProcessorCount, run->device);

    long const M = run->M;
    if (dalloc(run, &run->geo, G_COUNT * run->Nx) || dalloc(run, &run->B[0], 3 * M) || dalloc(run, &run->B[1], 3 * M)
        || dalloc(run, &run->E[0], 3 * M) || dalloc(run, &run->E[1], 3 * M) || dalloc(run, &run->EB, 6 * M)
        || dalloc(run, &run->charge, M) || dalloc(run, &run->current, 3 * M) || dalloc(run, &run->d_status, 1)
        || dalloc(run, &run->E1[0], 3 * M) || dalloc(run, &run->E1[1], 3 * M) || dalloc(run, &run->d_fallbacks, 1)
        || dalloc(run, &run->d_energy, 6 + 6 * (H1D_MAX_KINETIC + H1D_MAX_COLD))
        || (run->mixed && dalloc(run, &run->EBf, EBF_STRIDE * M))
        || (run->mixed && dalloc(run, &run->stage, run->stage_n))
        || (p.n_sources > 0 && dalloc(run, &run->src_dep, 4 * M * p.n_sources)))
        return fail(H1D_ERR_OOM);
    if (!(run->h_status = status_word()))
        return fail(H1D_ERR_OOM);
    for (int s = 0; s < p.n_kinetic; ++s) {
        SpeciesState &S = run->sp[s];
        if (dalloc(run, &S.dep, 16 * M) || dalloc(run, &S.mom_raw, 10 * M) || dalloc(run, &S.mom, 10 * M)
            || dalloc(run, &S.dead, 1))
            return fail(H1D_ERR_OOM);
        if (p.kinetic[s].scheme == H1D_DELTA_F) {
            std::vector<double> const eq = equilibrium_moments(p, p.kinetic[s]);
            if (dalloc(run, &S.eq, 7 * M)
                || cudaMemcpy(S.eq, eq.data(), sizeof(double) * eq.size(), cudaMemcpyHostToDevice) != cudaSuccess)
                return fail(H1D_ERR_OOM);
        }
    }
    for (int c = 0; c < p.n_cold; ++c) {
        ColdState &C = run->cold[c];
        if (dalloc(run, &C.n, M) || dalloc(run, &C.nV[0], 3 * M) || dalloc(run, &C.nV[1], 3 * M) || dalloc(run, &C.mom, 10 * M))
            return fail(H1D_ERR_OOM);
    }
    // the particle buffers of the declared load (Nx x Nc per species), so that the first upload
    // or populate allocates nothing
    for (int s = 0; s < p.n_kinetic; ++s)
        if (p.kinetic[s].Nc > 0 && p.kinetic[s].Nc <= (int64_t{ 1 } << 31) / p.Nx && ensure_capacity(run, s, p.Nx * p.kinetic[s].Nc) != H1D_OK)
            return fail(H1D_ERR_OOM);
    std::vector<double> const g = geometry_table(p);
    if (cudaMemcpyAsync(run->geo, g.data(), sizeof(double) * g.size(), cudaMemcpyHostToDevice, run->stream) != cudaSuccess
        || cudaStreamSynchronize(run->stream) != cudaSuccess)
        return fail(H1D_ERR_CUDA);
    *out = run;
    return H1D_OK;
}

int h1d_trim_device_memory(size_t keep_bytes, size_t *pool_bytes)
{
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) {
        cudaGetLastError();
        return H1D_ERR_NO_DEVICE;
    }
    DevicePool *P = nullptr;
    if (device_pool(dev, P) != cudaSuccess || cudaDeviceSynchronize() != cudaSuccess
        || cudaMemPoolTrimTo(P->pool, keep_bytes) != cudaSuccess) {
        cudaGetLastError();
        return H1D_ERR_CUDA;
    }
    if (pool_bytes) {
        uint64_t reserved = 0;
        if (cudaMemPoolGetAttribute(P->pool, cudaMemPoolAttrReservedMemCurrent, &reserved) != cudaSuccess)
            return H1D_ERR_CUDA;
        *pool_bytes = static_cast<size_t>(reserved);
    }
    return H1D_OK;
}

int h1d_destroy(h1d_run *run)
{
    if (!run)
        return H1D_OK;
    if (run->stream)
        cudaStreamSynchronize(run->stream);
    dfree(run->geo);
    for (int k = 0; k < 2; ++k)
        dfree(run->B[k]), dfree(run->E[k]), dfree(run->E1[k]);
    dfree(run->d_fallbacks);
    dfree(run->EB), dfree(run->EBf), dfree(run->src_dep), dfree(run->charge), dfree(run->current), dfree(run->d_status), dfree(run->d_energy);
    dfree(run->stage);
    run->sorter.release();
    release_status_word(run->h_status);
    for (auto &S : run->sp) {
        for (int k = 0; k < 2; ++k) {
            for (auto *b : S.buf[k])
                dfree(b);
            for (auto *b : S.fbuf[k])
                dfree(b);
            dfree(S.pos[k]);
            dfree(S.pid[k]), dfree(S.keys[k]), dfree(S.idx[k]);
            dfree(S.psd[k][0]), dfree(S.psd[k][1]);
            dfree(S.fpsd[k][0]), dfree(S.fpsd[k][1]);
        }
        dfree(S.dead), dfree(S.dep), dfree(S.mom_raw), dfree(S.mom);
        dfree(S.eq);
    }
    for (auto &C : run->cold)
        dfree(C.n), dfree(C.nV[0]), dfree(C.nV[1]), dfree(C.mom);
    for (auto &[k, b, e] : run->ev_done)
        cudaEventDestroy(b), cudaEventDestroy(e);
    for (auto e : run->ev_pool)
        cudaEventDestroy(e);
    if (run->stream)
        cudaStreamDestroy(run->stream);
    delete run;
    return H1D_OK;
}

int h1d_upload_particles(h1d_run *run, int s, int64_t n, double const *q1, double const *vx, double const *vy,
                         double const *vz, double const *w)
{
    if (!run || s < 0 || s >= run->p.n_kinetic || n < 0 || n > (int64_t{ 1 } << 31) - 1
        || (n > 0 && (!q1 || !vx || !vy || !vz || !w)))
        return set_err(run, H1D_ERR_INVALID_ARG, "h1d_upload_particles: bad arguments");
    SpeciesState &S = run->sp[s];
    CU(cudaStreamSynchronize(run->stream));
    TRY(ensure_capacity(run, s, n));
    S.cur              = 0;
    S.n                = n;
    double const *src[5] = { q1, vx, vy, vz, w };
    if (run->mixed && n) { // each FP64 component through the staging buffer, converted chunk by chunk
        for (int k = 0; k < 5; ++k)
            for (int64_t o = 0; o < n; o += run->stage_n) {
                int64_t const  c  = std::min<int64_t>(run->stage_n, n - o);
                unsigned const nb = static_cast<unsigned>((c + 255) / 256);
                CU(cudaMemcpyAsync(run->stage, src[k] + o, sizeof(double) * c, cudaMemcpyHostToDevice, run->stream));
                if (k == 0)
                    q1_to_pos_kernel<<<nb, 256, 0, run->stream>>>(run->stage, c, -0.5 * run->Nx, run->pos_scale,
                                                                  pos_len(run), S.pos[0] + o);
                else
                    to_f32_kernel<<<nb, 256, 0, run->stream>>>(run->stage, c, S.fbuf[0][k - 1] + o);
                CU(cudaGetLastError());
            }
    }
    for (int k = 0; k < 5 && !run->mixed; ++k)
        if (n)
            CU(cudaMemcpyAsync(S.buf[0][k], src[k], sizeof(double) * n, cudaMemcpyHostToDevice, run->stream));
    if (n && S.psd[0][0]) { // until h1d_upload_psd: real_f = w, marker = 1 (weight = real_f / marker)
        CU(cudaMemcpyAsync(S.psd[0][0], S.buf[0][4], sizeof(double) * n, cudaMemcpyDeviceToDevice, run->stream));
        CU(launch_fill(S.psd[0][1], n, 1.0, run->stream));
    }
    if (n && S.fpsd[0][0]) {
        CU(cudaMemcpyAsync(S.fpsd[0][0], S.fbuf[0][3], sizeof(float) * n, cudaMemcpyDeviceToDevice, run->stream));
        CU(launch_fill_f(S.fpsd[0][1], n, 1.0f, run->stream));
    }
    if (n)
        CU(launch_iota(S.pid[0], n, run->stream));
    S.since_sort       = 1 << 30;
    S.upload_order     = true;
    run->moments_stale = true;
    run->gen++;
    CU(cudaStreamSynchronize(run->stream));
    return H1D_OK;
}


int h1d_upload_psd(h1d_run *run, int s, int64_t n, double const *real_f, double const *marker)
{
    if (!run || s < 0 || s >= run->p.n_kinetic || (n > 0 && (!real_f || !marker)))
        return set_err(run, H1D_ERR_INVALID_ARG, "h1d_upload_psd: bad arguments");
    SpeciesState &S = run->sp[s];
    if (!evolves_psd(run->p.kinetic[s]))
        return set_err(run, H1D_ERR_INVALID_ARG, "h1d_upload_psd: the weights of this species do not evolve");
    if (n != S.n)
        return set_err(run, H1D_ERR_INVALID_ARG, "h1d_upload_psd: count differs from the uploaded particles");
    if (n && !S.upload_order)
        return set_err(run, H1D_ERR_INVALID_ARG, "h1d_upload_psd: the particles were reordered since their upload");
    CU(cudaStreamSynchronize(run->stream));
    if (n && !run->mixed) {
        CU(cudaMemcpyAsync(S.psd[S.cur][0], real_f, sizeof(double) * n, cudaMemcpyHostToDevice, run->stream));
        CU(cudaMemcpyAsync(S.psd[S.cur][1], marker, sizeof(double) * n, cudaMemcpyHostToDevice, run->stream));
    }
    double const *src[2] = { real_f, marker };
    for (int k = 0; k < 2 && n && run->mixed; ++k) // FP32 on the device, through the staging buffer
        for (int64_t o = 0; o < n; o += run->stage_n) {
            int64_t const c = std::min<int64_t>(run->stage_n, n - o);
            CU(cudaMemcpyAsync(run->stage, src[k] + o, sizeof(double) * c, cudaMemcpyHostToDevice, run->stream));
            to_f32_kernel<<<static_cast<unsigned>((c + 255) / 256), 256, 0, run->stream>>>(run->stage, c, S.fpsd[S.cur][k] + o);
            CU(cudaGetLastError());
        }
    CU(cudaStreamSynchronize(run->stream));
    return H1D_OK;
}

int h1d_download_psd(h1d_run *run, int s, double *real_f, double *marker)
{
    if (!run || s < 0 || s >= run->p.n_kinetic)
        return H1D_ERR_INVALID_ARG;
    SpeciesState &S = run->sp[s];
    if (!evolves_psd(run->p.kinetic[s]))
        return set_err(run, H1D_ERR_INVALID_ARG, "h1d_download_psd: the weights of this species do not evolve");
    if (run->p.particle_bc == H1D_BC_ABSORBING && S.n > 0 && S.since_sort > 0)
        TRY(sort_species(run, s)); // drop absorbed particles, as h1d_download_particles does
    if (real_f && S.n && !run->mixed)
        CU(cudaMemcpyAsync(real_f, S.psd[S.cur][0], sizeof(double) * S.n, cudaMemcpyDeviceToHost, run->stream));
    if (marker && S.n && !run->mixed)
        CU(cudaMemcpyAsync(marker, S.psd[S.cur][1], sizeof(double) * S.n, cudaMemcpyDeviceToHost, run->stream));
    double *dst[2] = { real_f, marker };
    for (int k = 0; k < 2 && S.n && run->mixed; ++k) // FP32 on the device, through the staging buffer
        for (int64_t o = 0; dst[k] && o < S.n; o += run->stage_n) {
            int64_t const c = std::min<int64_t>(run->stage_n, S.n - o);
            from_mixed_kernel<<<static_cast<unsigned>((c + 255) / 256), 256, 0, run->stream>>>(nullptr, S.fpsd[S.cur][k] + o, c,
                                                                                             0.0, 1.0, run->stage);
            CU(cudaGetLastError());
            CU(cudaMemcpyAsync(dst[k] + o, run->stage, sizeof(double) * c, cudaMemcpyDeviceToHost, run->stream));
        }
    CU(cudaStreamSynchronize(run->stream));
    return H1D_OK;
}


int h1d_populate(h1d_run *run, int s, int64_t n, uint64_t seed, double beta1, double T2_T1)
{
    if (!run || s < 0 || s >= run->p.n_kinetic || n < 0 || n > (int64_t{ 1 } << 31) - 1 || !(beta1 > 0) || !(T2_T1 > 0))
        return set_err(run, H1D_ERR_INVALID_ARG, "h1d_populate: bad arguments");
    if (evolves_psd(run->p.kinetic[s]))
        return set_err(run, H1D_ERR_INVALID_ARG,
                       "h1d_populate: species with evolving weights are loaded with h1d_upload_particles and h1d_upload_psd");
    if (run->p.kinetic[s].vdf != H1D_VDF_BIMAXWELLIAN)
        return set_err(run, H1D_ERR_INVALID_ARG,
                       "h1d_populate: draws bi-Maxwellian particles; other distributions are uploaded");
    h1d_params const       &p = run->p;
    h1d_kinetic_desc const &d = p.kinetic[s];
    SpeciesState           &S = run->sp[s];
    CU(cudaStreamSynchronize(run->stream));
    TRY(ensure_capacity(run, s, n));
    S.cur = 0, S.n = n;
    PopulateArgs a{};
    a.n = n;
    a.key = populate_key(seed, static_cast<uint64_t>(s));
    a.offset = populate_offset(a.key);
    double const q1min = -0.5 * p.Nx, q1max = q1min + p.Nx;
    a.N_loc = n_of_q1(p, T2_T1, q1min);
    a.N_len = n_of_q1(p, T2_T1, q1max) - a.N_loc;
    a.homogeneous = p.xi < 1e-10;
    a.xiD1 = p.xi * p.Dx, a.T2m1 = T2_T1 - 1, a.sqrtT2 = std::sqrt(T2_T1), a.sDxXi = a.sqrtT2 * p.Dx * p.xi;
    a.T2 = T2_T1, a.oneMinusT2 = 1 - T2_T1, a.vth1 = std::sqrt(beta1) * p.c * std::fabs(d.Oc) / d.op;
    a.q1min = q1min, a.q1max_in = std::nextafter(q1max, q1min), a.full_min = q1min;
    if (run->mixed)
        a.pos = S.pos[0], a.fvx = S.fbuf[0][0], a.fvy = S.fbuf[0][1], a.fvz = S.fbuf[0][2], a.fw = S.fbuf[0][3],
        a.scale = run->pos_scale, a.len = pos_len(run);
    else
        a.q1 = S.buf[0][0], a.vx = S.buf[0][1], a.vy = S.buf[0][2], a.vz = S.buf[0][3], a.w = S.buf[0][4];
    if (n) {
        populate_kernel<<<static_cast<unsigned>((n + 255) / 256), 256, 0, run->stream>>>(a);
        CU(cudaGetLastError());
        CU(launch_iota(S.pid[0], n, run->stream));
    }
    S.since_sort       = 1 << 30;
    S.upload_order     = true;
    run->moments_stale = true;
    run->gen++;
    CU(cudaStreamSynchronize(run->stream));
    return H1D_OK;
}

int h1d_upload_fields(h1d_run *run, double const *B, double const *E)
{
    if (!run)
        return H1D_ERR_INVALID_ARG;
    size_t const bytes = sizeof(double) * 3 * run->M;
    if (B)
        CU(cudaMemcpyAsync(run->B[run->fcur], B, bytes, cudaMemcpyHostToDevice, run->stream));
    if (E)
        CU(cudaMemcpyAsync(run->E[run->fcur], E, bytes, cudaMemcpyHostToDevice, run->stream));
    CU(cudaStreamSynchronize(run->stream));
    run->fields_dirty = true;
    run->gen++;
    return H1D_OK;
}

int h1d_upload_cold(h1d_run *run, int i, double const *n_full, double const *nV_full)
{
    if (!run || i < 0 || i >= run->p.n_cold || !n_full || !nV_full)
        return set_err(run, H1D_ERR_INVALID_ARG, "h1d_upload_cold: bad arguments");
    ColdState &C = run->cold[i];
    CU(cudaMemcpyAsync(C.n, n_full, sizeof(double) * run->M, cudaMemcpyHostToDevice, run->stream));
    CU(cudaMemcpyAsync(C.nV[C.cur], nV_full, sizeof(double) * 3 * run->M, cudaMemcpyHostToDevice, run->stream));
    CU(cudaMemcpyAsync(C.nV[1 - C.cur], nV_full, sizeof(double) * 3 * run->M, cudaMemcpyHostToDevice, run->stream));
    CU(cudaStreamSynchronize(run->stream));
    run->moments_stale = true;
    run->gen++;
    return H1D_OK;
}

int h1d_advance_async(h1d_run *run, uint32_t n_steps)
{
    if (!run)
        return H1D_ERR_INVALID_ARG;
    bool const first = !run->recurring;
    if (first || run->fields_dirty)
        TRY(prepare_fields(run));
    if (first && run->p.algorithm == H1D_ALGO_PC)
        TRY(pc_initial_sources(run));
    run->recurring = true;
    bool const fuse = fused_collect(run);
    for (uint32_t i = 0; i < n_steps; ++i)
        TRY(run->p.algorithm == H1D_ALGO_CAMCL ? camcl_step(run, fuse && i + 1 == n_steps) : pc_step(run));
    run->moments_stale = true;
    return H1D_OK;
}

int h1d_synchronize(h1d_run *run)
{
    if (!run)
        return H1D_ERR_INVALID_ARG;
    return check_status(run);
}

int h1d_advance(h1d_run *run, uint32_t n_steps)
{
    TRY(h1d_advance_async(run, n_steps));
    return h1d_synchronize(run);
}

int h1d_get_stream(h1d_run *run, void **stream)
{
    if (!run || !stream)
        return H1D_ERR_INVALID_ARG;
    *stream = run->stream;
    return H1D_OK;
}

int h1d_profile_enable(h1d_run *run, int on)
{
    if (!run)
        return H1D_ERR_INVALID_ARG;
    CU(cudaStreamSynchronize(run->stream));
    for (auto &[k, b, e] : run->ev_done)
        run->ev_pool.push_back(b), run->ev_pool.push_back(e);
    run->ev_done.clear();
    if (on) {
        run->prof = h1d_profile{};
        CU(cudaMemsetAsync(run->d_fallbacks, 0, sizeof(unsigned long long), run->stream));
    }
    run->profiling = on != 0;
    return H1D_OK;
}

int h1d_profile_read(h1d_run *run, h1d_profile *out)
{
    if (!run || !out)
        return H1D_ERR_INVALID_ARG;
    CU(cudaStreamSynchronize(run->stream));
    for (auto &[k, b, e] : run->ev_done) {
        float ms = 0;
        CU(cudaEventElapsedTime(&ms, b, e));
        (k == 0 ? run->prof.push_ms : k == 1 ? run->prof.sort_ms : run->prof.field_ms) += ms;
        run->ev_pool.push_back(b), run->ev_pool.push_back(e);
    }
    run->ev_done.clear();
    unsigned long long miss = 0;
    CU(cudaMemcpy(&miss, run->d_fallbacks, sizeof miss, cudaMemcpyDeviceToHost));
    run->prof.window_misses = static_cast<int64_t>(miss);
    *out = run->prof;
    return H1D_OK;
}

int h1d_particle_count(h1d_run *run, int s, int64_t *n)
{
    if (!run || s < 0 || s >= run->p.n_kinetic || !n)
        return H1D_ERR_INVALID_ARG;
    if (run->p.particle_bc == H1D_BC_ABSORBING && run->sp[s].n > 0 && run->sp[s].since_sort > 0)
        TRY(sort_species(run, s)); // drop absorbed particles, so that the count is exact
    *n = run->sp[s].n;
    return H1D_OK;
}

int h1d_download_particles(h1d_run *run, int s, double *q1, double *vx, double *vy, double *vz, double *w, int64_t *pid)
{
    if (!run || s < 0 || s >= run->p.n_kinetic)
        return H1D_ERR_INVALID_ARG;
    SpeciesState &S = run->sp[s];
    if (run->p.particle_bc == H1D_BC_ABSORBING && S.n > 0 && S.since_sort > 0)
        TRY(sort_species(run, s)); // drop absorbed particles
    double *dst[5] = { q1, vx, vy, vz, w };
    if (run->mixed && S.n) { // each component converted to FP64 chunk by chunk in the staging buffer
        for (int k = 0; k < 5; ++k) {
            if (!dst[k])
                continue;
            for (int64_t o = 0; o < S.n; o += run->stage_n) {
                int64_t const  c  = std::min<int64_t>(run->stage_n, S.n - o);
                unsigned const nb = static_cast<unsigned>((c + 255) / 256);
                from_mixed_kernel<<<nb, 256, 0, run->stream>>>(k == 0 ? S.pos[S.cur] + o : nullptr,
                                                               k == 0 ? nullptr : S.fbuf[S.cur][k - 1] + o, c, -0.5 * run->Nx,
                                                               1 / run->pos_scale, run->stage);
                CU(cudaGetLastError());
                CU(cudaMemcpyAsync(dst[k] + o, run->stage, sizeof(double) * c, cudaMemcpyDeviceToHost, run->stream));
            }
        }
    }
    for (int k = 0; k < 5 && !run->mixed; ++k)
        if (dst[k] && S.n)
            CU(cudaMemcpyAsync(dst[k], S.buf[S.cur][k], sizeof(double) * S.n, cudaMemcpyDeviceToHost, run->stream));
    if (pid && S.n) {
        std::vector<int32_t> tmp(S.n);
        CU(cudaMemcpyAsync(tmp.data(), S.pid[S.cur], sizeof(int32_t) * S.n, cudaMemcpyDeviceToHost, run->stream));
        CU(cudaStreamSynchronize(run->stream));
        for (int64_t k = 0; k < S.n; ++k)
            pid[k] = tmp[k];
    }
    CU(cudaStreamSynchronize(run->stream));
    return H1D_OK;
}

int h1d_download_fields(h1d_run *run, double *B, double *E)
{
    if (!run)
        return H1D_ERR_INVALID_ARG;
    if (run->fields_dirty)
        TRY(prepare_fields(run));
    size_t const bytes = sizeof(double) * 3 * run->M;
    if (B)
        CU(cudaMemcpyAsync(B, run->B[run->fcur], bytes, cudaMemcpyDeviceToHost, run->stream));
    if (E)
        CU(cudaMemcpyAsync(E, run->E[run->fcur], bytes, cudaMemcpyDeviceToHost, run->stream));
    CU(cudaStreamSynchronize(run->stream));
    return H1D_OK;
}

int h1d_download_sources(h1d_run *run, double *charge, double *current)
{
    if (!run)
        return H1D_ERR_INVALID_ARG;
    if (charge)
        CU(cudaMemcpyAsync(charge, run->charge, sizeof(double) * run->M, cudaMemcpyDeviceToHost, run->stream));
    if (current)
        CU(cudaMemcpyAsync(current, run->current, sizeof(double) * 3 * run->M, cudaMemcpyDeviceToHost, run->stream));
    CU(cudaStreamSynchronize(run->stream));
    return H1D_OK;
}

int h1d_download_moments(h1d_run *run, int s, double *n, double *nV, double *nvv)
{
    if (!run || s < 0 || s >= run->p.n_kinetic)
        return H1D_ERR_INVALID_ARG;
    TRY(finalize_moments(run));
    double const *m = run->sp[s].mom;
    if (n)
        CU(cudaMemcpyAsync(n, m, sizeof(double) * run->M, cudaMemcpyDeviceToHost, run->stream));
    if (nV)
        CU(cudaMemcpyAsync(nV, m + run->M, sizeof(double) * 3 * run->M, cudaMemcpyDeviceToHost, run->stream));
    if (nvv)
        CU(cudaMemcpyAsync(nvv, m + 4 * run->M, sizeof(double) * 6 * run->M, cudaMemcpyDeviceToHost, run->stream));
    CU(cudaStreamSynchronize(run->stream));
    return H1D_OK;
}

int h1d_download_cold(h1d_run *run, int i, double *n, double *nV, double *nvv, double *n_full, double *nV_full)
{
    if (!run || i < 0 || i >= run->p.n_cold)
        return H1D_ERR_INVALID_ARG;
    TRY(finalize_moments(run));
    ColdState const &C = run->cold[i];
    long const       M = run->M;
    if (n)
        CU(cudaMemcpyAsync(n, C.mom, sizeof(double) * M, cudaMemcpyDeviceToHost, run->stream));
    if (nV)
        CU(cudaMemcpyAsync(nV, C.mom + M, sizeof(double) * 3 * M, cudaMemcpyDeviceToHost, run->stream));
    if (nvv)
        CU(cudaMemcpyAsync(nvv, C.mom + 4 * M, sizeof(double) * 6 * M, cudaMemcpyDeviceToHost, run->stream));
    if (n_full)
        CU(cudaMemcpyAsync(n_full, C.n, sizeof(double) * M, cudaMemcpyDeviceToHost, run->stream));
    if (nV_full)
        CU(cudaMemcpyAsync(nV_full, C.nV[C.cur], sizeof(double) * 3 * M, cudaMemcpyDeviceToHost, run->stream));
    CU(cudaStreamSynchronize(run->stream));
    return H1D_OK;
}


// ---- ensembles -----------------------------------------------------------------------------------

int h1d_batch_create(h1d_run *const *runs, int n_runs, h1d_batch **out)
{
    if (!out)
        return H1D_ERR_INVALID_ARG;
    *out = nullptr;
    if (!runs || n_runs <= 0) {
        std::fprintf(stderr, "h1d_batch_create: no runs\n");
        return H1D_ERR_INVALID_ARG;
    }
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess)
        return H1D_ERR_NO_DEVICE;
    for (int i = 0; i < n_runs; ++i) {
        h1d_run *r = runs[i];
        char const *why = !r ? "null run"
                          : r->p.algorithm != runs[0]->p.algorithm ? "members advance by one algorithm (all CAM-CL or all PC)"
                          : r->device != dev                ? "run lives on another device"
                          : r->batch_count                  ? "run is already a member of a batch"
                                                            : nullptr;
        for (int j = 0; j < i && !why; ++j)
            if (runs[j] == r)
                why = "run listed twice";
        if (why) {
            std::fprintf(stderr, "h1d_batch_create: member %d: %s\n", i, why);
            return H1D_ERR_INVALID_ARG;
        }
    }
    h1d_batch *b = new (std::nothrow) h1d_batch{};
    if (!b)
        return H1D_ERR_OOM;
    b->device = dev;
    b->pc     = runs[0]->p.algorithm == H1D_ALGO_PC;
    if (cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking) != cudaSuccess) {
        delete b;
        return H1D_ERR_CUDA;
    }
    cudaDeviceGetAttribute(&b->num_sms, cudaDevAttrMultiProcessorCount, dev);
    b->k = runs[0]->sort_interval;
    for (int i = 0; i < n_runs; ++i) {
        h1d_run *r = runs[i];
        cudaStreamSynchronize(r->stream);
        b->runs.push_back(r);
        b->saved.push_back(r->stream);
        r->stream      = b->stream;
        r->batch_count = 1;
    }
    *out = b;
    return H1D_OK;
}

int h1d_batch_destroy(h1d_batch *b)
{
    if (!b)
        return H1D_OK;
    cudaStreamSynchronize(b->stream);
    for (size_t i = 0; i < b->runs.size(); ++i) {
        b->runs[i]->stream      = b->saved[i];
        b->runs[i]->batch_count = 0;
        for (int s = 0; s < b->runs[i]->p.n_kinetic; ++s) // the run resumes its own sort schedule
            b->runs[i]->sp[s].since_sort = std::min(b->runs[i]->sp[s].since_sort, b->since_block);
    }
    drop_graph(b);
    dfree(b->d_table), dfree(b->d_map);
    b->sorter.release();
    cudaStreamDestroy(b->stream);
    delete b;
    return H1D_OK;
}

int h1d_batch_advance_async(h1d_batch *b, uint32_t n_steps)
{
    if (!b)
        return H1D_ERR_INVALID_ARG;
    return batch_advance(b, n_steps);
}

int h1d_batch_advance_members_async(h1d_batch *b, uint32_t const *n_steps)
{
    if (!b || !n_steps)
        return H1D_ERR_INVALID_ARG;
    return batch_advance_members(b, n_steps);
}

int h1d_batch_synchronize(h1d_batch *b)
{
    if (!b)
        return H1D_ERR_INVALID_ARG;
    return batch_check(b);
}

int h1d_batch_advance(h1d_batch *b, uint32_t n_steps)
{
    TRY(h1d_batch_advance_async(b, n_steps));
    return h1d_batch_synchronize(b);
}

int h1d_batch_get_stream(h1d_batch *b, void **stream)
{
    if (!b || !stream)
        return H1D_ERR_INVALID_ARG;
    *stream = b->stream;
    return H1D_OK;
}

int h1d_batch_configure(h1d_batch *b, int sort_interval, int push_ctas_per_sm, int use_graphs)
{
    if (!b || sort_interval < 0 || sort_interval > 4096 || push_ctas_per_sm < 0 || push_ctas_per_sm > PIPE_CTAS_PER_SM_MIXED)
        return bset_err(b, H1D_ERR_INVALID_ARG, "h1d_batch_configure: sort_interval in [0, 4096], CTAs per SM in [0, 4]");
    if (sort_interval > 0 && sort_interval != b->k)
        b->k = sort_interval, b->since_block = 1 << 30;
    b->ctas       = push_ctas_per_sm;
    b->use_graphs = use_graphs != 0;
    drop_graph(b);
    b->graphs_warm = false;
    return H1D_OK;
}

int h1d_batch_autotune(h1d_batch *b, uint32_t *steps_taken, int *sort_interval, int *push_ctas_per_sm)
{
    if (!b)
        return H1D_ERR_INVALID_ARG;
    TRY(batch_prepare(b));
    TRY(build_field_tables(b));
    drop_graph(b);
    b->graphs_warm = false;
    uint32_t taken = 0;
    // 1. sort interval, at the default CTA count: two whole blocks per candidate
    int   best_k  = b->k;
    float best_ms = 0;
    for (int k : { 8, 12, 16, 24, 32 }) {
        b->k           = k;
        b->since_block = 1 << 30;
        float ms       = 0;
        TRY(batch_time(b, 2u * k, &ms));
        taken += 2u * k;
        float const per = ms / (2.0f * k);
        if (best_ms == 0 || per < best_ms)
            best_ms = per, best_k = k;
    }
    b->k = best_k;
    // 2. CTAs per SM of the particle pass, at the chosen interval
    bool any_mixed = false;
    for (h1d_run const *r : b->runs)
        any_mixed = any_mixed || r->mixed;
    int const max_c  = any_mixed ? PIPE_CTAS_PER_SM_MIXED : PIPE_CTAS_PER_SM;
    int       best_c = 0;
    best_ms          = 0;
    for (int c = 1; c <= max_c; ++c) {
        b->ctas        = c;
        b->since_block = 1 << 30;
        float ms       = 0;
        TRY(batch_time(b, 2u * b->k, &ms));
        taken += 2u * b->k;
        float const per = ms / (2.0f * b->k);
        if (best_ms == 0 || per < best_ms)
            best_ms = per, best_c = c;
    }
    b->ctas = best_c;
    for (h1d_run *r : b->runs)
        r->sort_interval = b->k, r->ctas_per_sm = b->ctas;
    if (steps_taken)
        *steps_taken = taken;
    if (sort_interval)
        *sort_interval = b->k;
    if (push_ctas_per_sm)
        *push_ctas_per_sm = b->ctas;
    return H1D_OK;
}

int h1d_batch_stats_read(h1d_batch *b, h1d_batch_stats *out)
{
    if (!b || !out)
        return H1D_ERR_INVALID_ARG;
    *out = b->stats;
    return H1D_OK;
}

char const *h1d_batch_status_string(h1d_batch *b) { return b ? b->msg.c_str() : "null batch"; }

// ---- tuning of a single run ----------------------------------------------------------------------

int h1d_configure(h1d_run *run, int sort_interval, int push_ctas_per_sm)
{
    if (!run || sort_interval < 0 || sort_interval > 4096 || push_ctas_per_sm < 0 || push_ctas_per_sm > PIPE_CTAS_PER_SM_MIXED)
        return set_err(run, H1D_ERR_INVALID_ARG, "h1d_configure: sort_interval in [0, 4096], CTAs per SM in [0, 4]");
    if (sort_interval > 0)
        run->sort_interval = sort_interval;
    run->ctas_per_sm = push_ctas_per_sm;
    return H1D_OK;
}

int h1d_autotune(h1d_run *run, uint32_t *steps_taken, int *sort_interval, int *push_ctas_per_sm)
{
    if (!run)
        return H1D_ERR_INVALID_ARG;
    if (run->p.algorithm != H1D_ALGO_CAMCL || run->batch_count)
        return set_err(run, H1D_ERR_INVALID_ARG, "h1d_autotune: a CAM-CL run outside any batch");
    h1d_batch *b  = nullptr;
    int        st = h1d_batch_create(&run, 1, &b);
    if (st == H1D_OK)
        st = h1d_batch_autotune(b, steps_taken, sort_interval, push_ctas_per_sm);
    if (st != H1D_OK && b)
        set_err(run, st, b->msg);
    h1d_batch_destroy(b);
    return st;
}


int h1d_vhistogram(h1d_run *run, int s, double ext_loc, double ext_len, double v1min, double v1len, int64_t v1dim,
                   double v2min, double v2len, int64_t v2dim, double *out, int64_t *total)
{
    if (!run || s < 0 || s >= run->p.n_kinetic || v1dim <= 0 || v2dim <= 0 || v1dim * v2dim > (int64_t{ 1 } << 24)
        || !(v1len > 0) || !(v2len > 0) || !out)
        return set_err(run, H1D_ERR_INVALID_ARG, "h1d_vhistogram: bad arguments");
    TRY(finalize_moments(run));
    SpeciesState const &S    = run->sp[s];
    size_t const        bins = static_cast<size_t>(v1dim * v2dim);
    double             *d    = nullptr;
    CU(dmalloc(&d, sizeof(double) * (3 * bins + 1)));
    auto *count = reinterpret_cast<unsigned long long *>(d + 3 * bins);
    int   st    = H1D_OK;
    if (cudaMemsetAsync(d, 0, sizeof(double) * (3 * bins + 1), run->stream) != cudaSuccess)
        st = set_err(run, H1D_ERR_CUDA, "h1d_vhistogram: memset failed");
    if (st == H1D_OK && S.n > 0) {
        VHistArgs a{};
        if (run->mixed)
            a.pos = S.pos[S.cur], a.fvx = S.fbuf[S.cur][0], a.fvy = S.fbuf[S.cur][1], a.fvz = S.fbuf[S.cur][2],
            a.fw = S.fbuf[S.cur][3], a.freal_f = S.fpsd[S.cur][0], a.fmarker = S.fpsd[S.cur][1],
            a.inv_scale = 1 / run->pos_scale;
        else
            a.q1 = S.buf[S.cur][0], a.vx = S.buf[S.cur][1], a.vy = S.buf[S.cur][2], a.vz = S.buf[S.cur][3],
            a.w = S.buf[S.cur][4], a.real_f = S.psd[S.cur][0], a.marker = S.psd[S.cur][1];
        a.n = S.n, a.full_min = -0.5 * run->Nx, a.half_min = a.full_min + 0.5;
        a.ext_lo = ext_loc, a.ext_hi = ext_loc + ext_len, a.v1min = v1min, a.v1len = v1len, a.v2min = v2min, a.v2len = v2len;
        a.v1dim = static_cast<int>(v1dim), a.v2dim = static_cast<int>(v2dim);
        a.mom = S.mom, a.M = run->M, a.out = d, a.count = count;
        vhist_kernel<<<static_cast<unsigned>((S.n + 255) / 256), 256, 0, run->stream>>>(a);
        if (cudaGetLastError() != cudaSuccess)
            st = set_err(run, H1D_ERR_CUDA, "h1d_vhistogram: launch failed");
    }
    std::vector<double> h(3 * bins + 1);
    if (st == H1D_OK && (cudaMemcpyAsync(h.data(), d, sizeof(double) * h.size(), cudaMemcpyDeviceToHost, run->stream) != cudaSuccess
                         || cudaStreamSynchronize(run->stream) != cudaSuccess))
        st = set_err(run, H1D_ERR_CUDA, "h1d_vhistogram: copy failed");
    dfree(d);
    TRY(st);
    unsigned long long c = 0;
    std::memcpy(&c, &h[3 * bins], sizeof c);
    for (size_t i = 0; i < 3 * bins; ++i)
        out[i] = c ? h[i] / static_cast<double>(c) : 0.0;
    if (total)
        *total = static_cast<int64_t>(c);
    return H1D_OK;
}

int h1d_energy(h1d_run *run, double *dB2O2, double *dE2O2, double *KE_lab, double *KE_pla)
{
    if (!run || !dB2O2 || !dE2O2 || !KE_lab || !KE_pla)
        return H1D_ERR_INVALID_ARG;
    TRY(finalize_moments(run));
    h1d_params const &p  = run->p;
    int const         ns = p.n_kinetic + p.n_cold;
    EnergyArgs        a{};
    a.B = run->B[run->fcur] + 3 * PAD, a.E = run->E[run->fcur] + 3 * PAD, a.Nx = static_cast<int>(run->Nx);
    a.ns = ns, a.out = run->d_energy;
    for (int s = 0; s < ns; ++s) {
        double Oc, op;
        double const *m;
        if (s < p.n_kinetic)
            Oc = p.kinetic[s].Oc, op = p.kinetic[s].op, m = run->sp[s].mom;
        else
            Oc = p.cold[s - p.n_kinetic].Oc, op = p.cold[s - p.n_kinetic].op, m = run->cold[s - p.n_kinetic].mom;
        double const tmp = p.O0 / Oc * op / p.c; // Species.h:50-54
        a.n[s]          = m + PAD;
        a.nV[s]         = m + run->M + 3 * PAD;
        a.nvv[s]        = m + 4 * run->M + 6 * PAD;
        a.factor[s]     = tmp * tmp / (2 * static_cast<double>(p.Nx));
    }
    CU(launch_energy(a, run->stream));
    std::vector<double> h(6 + 6 * ns);
    CU(cudaMemcpyAsync(h.data(), run->d_energy, sizeof(double) * h.size(), cudaMemcpyDeviceToHost, run->stream));
    CU(cudaStreamSynchronize(run->stream));
    for (int c = 0; c < 3; ++c)
        dB2O2[c] = h[c], dE2O2[c] = h[3 + c];
    for (int s = 0; s < ns; ++s)
        for (int c = 0; c < 3; ++c)
            KE_lab[3 * s + c] = h[6 + 6 * s + c], KE_pla[3 * s + c] = h[6 + 6 * s + 3 + c];
    return H1D_OK;
}

} // extern "C"

// ---- serving loop --------------------------------------------------------------------------------
// Requests (a run description, a loader seed and a step count) wait in a queue until the HBM they
// need fits the budget; admitted runs are built on the device (h1d_populate) and advance together
// as one batch per algorithm, a quantum of steps per tick; finished runs are read back and freed,
// which lets the next requests in.
//
// Threads.  One thread drives the loop with h1d_server_tick; it alone owns the active runs and
// their batches.  The mutex guards what other threads see -- the queue, every request's state,
// times and results, the memory accounting and the statistics -- and is held only for those short
// updates, never while the GPU works, so submit, poll, result and release return at once while a
// tick runs.  Within a tick the batches' quantum is enqueued first and the requests admitted in
// that tick are built on their own streams while it runs; they join the batches at the next tick.
// A member whose run fails (moved too far, non-finite state) fails alone; the others keep their
// progress.  Served batches run eagerly: their membership changes too often for graph capture to
// pay for itself.

namespace {

struct ServerReq {
    uint64_t            id = 0;
    h1d_request         rq{};
    size_t              bytes = 0;
    int                 state = H1D_REQ_QUEUED, status = H1D_OK;
    uint32_t            done_steps = 0, tick_steps = 0; // steps taken / steps of the current tick
    h1d_run            *run = nullptr;
    double              t_submit = 0, t_admit = 0, t_done = 0;
    std::vector<double> B, E, energy, n, nV, nvv;
    std::string         msg;
};

// device bytes a request needs: particles in both buffer sets with ids and sort keys, the grids
size_t request_bytes(h1d_request const &rq)
{
    h1d_params const &p   = rq.params;
    size_t const      per = p.precision == H1D_PREC_MIXED ? 5 * 4 : 5 * 8;
    size_t            b   = 0;
    for (int s = 0; s < p.n_kinetic; ++s) {
        size_t const n = static_cast<size_t>(std::max<int64_t>(rq.n_particles[s], 0)) + 64;
        b += 2 * n * (per + 4 + 4 + 4) + (n / SORT_TILE + 1) * 256 * 4 * 2;
    }
    size_t const M = static_cast<size_t>(p.Nx + 2 * PAD);
    b += sizeof(double) * M * (G_COUNT + 6 * 3 + 6 + 1 + 3 + 6 + H1D_MAX_KINETIC * 36 + H1D_MAX_COLD * 17);
    if (p.precision == H1D_PREC_MIXED) { // the FP64 staging buffer of uploads and downloads
        int64_t stage = 1 << 16;
        for (int s = 0; s < p.n_kinetic; ++s)
            stage = std::max<int64_t>(stage, std::min<int64_t>(STAGE_N, p.Nx * std::max<int64_t>(p.kinetic[s].Nc, 0)));
        b += sizeof(double) * static_cast<size_t>(stage);
    }
    return b + (size_t{ 1 } << 20);
}

} // namespace

struct h1d_server {
    size_t                                budget = 0, used = 0, peak = 0;
    int                                   quantum = 64, sort_interval = 16;
    std::deque<ServerReq *>               queue;
    std::map<uint64_t, ServerReq *>       all;
    uint64_t                              next_id = 1;
    std::chrono::steady_clock::time_point t0 = std::chrono::steady_clock::now();
    h1d_server_stats                      stats{}; // retired batches' counts included
    h1d_batch_stats                       live{};  // the current batches' counts, as of the last tick
    std::mutex                            mu;      // the state other threads see (see above)
    // owned by the thread that ticks
    std::mutex                            tick_mu; // one tick at a time
    std::vector<ServerReq *>              active;
    h1d_batch                            *batch[2] = { nullptr, nullptr }; // the active runs by algorithm (H1D_ALGO_*)
    bool                                  dirty = false;

    double now() const { return std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count(); }
};

namespace {

// destroy the batches (their runs stay), their counts folded into the statistics; tick thread
void drop_batches(h1d_server *sv)
{
    for (h1d_batch *&b : sv->batch) {
        if (!b)
            continue;
        {
            h1d_batch_stats st{};
            h1d_batch_stats_read(b, &st);
            std::lock_guard<std::mutex> lock(sv->mu);
            sv->stats.kernel_launches += st.kernel_launches;
            sv->stats.graph_launches += st.graph_launches;
            sv->stats.steps += st.steps;
        }
        h1d_batch_destroy(b);
        b = nullptr;
    }
}

// publish the end of a request (caller holds mu); its run is destroyed by the caller
void finish_locked(h1d_server *sv, ServerReq *r, int status, std::string const &msg)
{
    r->status = status;
    r->msg    = msg;
    r->state  = status == H1D_OK ? H1D_REQ_DONE : H1D_REQ_FAILED;
    r->t_done = sv->now();
    sv->used -= r->bytes;
    if (status == H1D_OK)
        sv->stats.completed++;
    else
        sv->stats.failed++;
}

// build a request's run on the device: particles by the device loader, cold fluid at rest; the
// work is enqueued on the run's own stream (tick thread, without the lock)
int admit(int sort_interval, ServerReq *r)
{
    h1d_params p = r->rq.params;
    if (p.sort_interval <= 0)
        p.sort_interval = sort_interval;
    int st = h1d_create(&p, &r->run);
    if (st != H1D_OK)
        return st;
    for (int s = 0; s < p.n_kinetic && st == H1D_OK; ++s)
        st = h1d_populate(r->run, s, r->rq.n_particles[s], r->rq.seed, r->rq.beta1[s], r->rq.T2_T1[s]);
    long const          M = p.Nx + 2 * PAD;
    std::vector<double> n_full(M, 0.0), nV(3 * M, 0.0);
    for (long i = PAD; i < PAD + p.Nx; ++i)
        n_full[i] = 1.0;
    for (int c = 0; c < p.n_cold && st == H1D_OK; ++c)
        st = h1d_upload_cold(r->run, c, n_full.data(), nV.data());
    if (st != H1D_OK)
        r->msg = r->run ? r->run->msg : "";
    return st;
}

// read a finished run back into its request
int collect(ServerReq *r)
{
    h1d_params const &p = r->rq.params;
    long const        M = p.Nx + 2 * PAD;
    int const         ns = p.n_kinetic + p.n_cold;
    r->B.resize(3 * M), r->E.resize(3 * M), r->energy.resize(6 + 6 * ns);
    r->n.resize(static_cast<size_t>(p.n_kinetic) * M), r->nV.resize(3 * r->n.size()), r->nvv.resize(6 * r->n.size());
    TRY(h1d_download_fields(r->run, r->B.data(), r->E.data()));
    std::vector<double> lab(3 * ns), pla(3 * ns);
    TRY(h1d_energy(r->run, r->energy.data(), r->energy.data() + 3, lab.data(), pla.data()));
    for (int s = 0; s < ns; ++s)
        for (int c = 0; c < 3; ++c)
            r->energy[6 + 6 * s + c] = lab[3 * s + c], r->energy[6 + 6 * s + 3 + c] = pla[3 * s + c];
    for (int s = 0; s < p.n_kinetic; ++s)
        TRY(h1d_download_moments(r->run, s, r->n.data() + s * M, r->nV.data() + 3 * s * M, r->nvv.data() + 6 * s * M));
    return H1D_OK;
}

} // namespace

extern "C" {

int h1d_server_create(size_t hbm_budget_bytes, int steps_per_tick, h1d_server **out)
{
    if (!out || steps_per_tick <= 0)
        return H1D_ERR_INVALID_ARG;
    *out          = nullptr;
    h1d_server *sv = new (std::nothrow) h1d_server{};
    if (!sv)
        return H1D_ERR_OOM;
    sv->budget  = hbm_budget_bytes;
    sv->quantum = steps_per_tick;
    *out        = sv;
    return H1D_OK;
}

int h1d_server_configure(h1d_server *sv, int sort_interval)
{
    if (!sv || sort_interval <= 0 || sort_interval > 4096)
        return H1D_ERR_INVALID_ARG;
    std::lock_guard<std::mutex> tick(sv->tick_mu);
    sv->sort_interval = sort_interval;
    sv->dirty         = true;
    return H1D_OK;
}

int h1d_server_submit(h1d_server *sv, h1d_request const *rq, uint64_t *id)
{
    if (!sv || !rq || !id)
        return H1D_ERR_INVALID_ARG;
    std::string m;
    if (int const st = validate(&rq->params, m)) {
        std::fprintf(stderr, "h1d_server_submit: %s\n", m.c_str());
        return st;
    }
    if (rq->n_steps == 0)
        return H1D_ERR_INVALID_ARG;
    for (int s = 0; s < rq->params.n_kinetic; ++s) // built by h1d_populate: bi-Maxwellian, full-f
        if (rq->n_particles[s] < 0 || rq->n_particles[s] > (int64_t{ 1 } << 31) - 1 || !(rq->beta1[s] > 0)
            || !(rq->T2_T1[s] > 0) || rq->params.kinetic[s].vdf != H1D_VDF_BIMAXWELLIAN || evolves_psd(rq->params.kinetic[s]))
            return H1D_ERR_INVALID_ARG;
    auto *r  = new (std::nothrow) ServerReq{};
    if (!r)
        return H1D_ERR_OOM;
    r->rq    = *rq;
    r->bytes = request_bytes(*rq);
    std::lock_guard<std::mutex> lock(sv->mu);
    if (r->bytes > sv->budget) {
        delete r;
        std::fprintf(stderr, "h1d_server_submit: the request needs more device memory than the whole budget\n");
        return H1D_ERR_OOM;
    }
    r->id       = sv->next_id++;
    r->t_submit = sv->now();
    sv->queue.push_back(r);
    sv->all[r->id] = r;
    sv->stats.submitted++;
    *id = r->id;
    return H1D_OK;
}

int h1d_server_tick(h1d_server *sv, int *n_active, int *n_queued)
{
    if (!sv)
        return H1D_ERR_INVALID_ARG;
    std::lock_guard<std::mutex> tick(sv->tick_mu);

    // 1. the batches of the active runs, one per algorithm, after a change of membership
    if (sv->dirty) {
        drop_batches(sv);
        for (int alg = 0; alg < 2; ++alg) {
            std::vector<h1d_run *> runs;
            for (ServerReq *r : sv->active)
                if (r->rq.params.algorithm == alg)
                    runs.push_back(r->run);
            if (runs.empty())
                continue;
            int st = h1d_batch_create(runs.data(), static_cast<int>(runs.size()), &sv->batch[alg]);
            if (st == H1D_OK)
                st = h1d_batch_configure(sv->batch[alg], sv->sort_interval, 0, 0);
            if (st != H1D_OK) { // the algorithm's runs fail (the batch goes before its runs)
                h1d_batch_destroy(sv->batch[alg]);
                sv->batch[alg] = nullptr;
                std::vector<ServerReq *> gone;
                for (auto it = sv->active.begin(); it != sv->active.end();)
                    if ((*it)->rq.params.algorithm == alg)
                        gone.push_back(*it), it = sv->active.erase(it);
                    else
                        ++it;
                {
                    std::lock_guard<std::mutex> lock(sv->mu);
                    for (ServerReq *r : gone)
                        finish_locked(sv, r, st, "batch creation failed");
                }
                for (ServerReq *r : gone)
                    h1d_destroy(r->run), r->run = nullptr;
            }
        }
        sv->dirty = false;
        std::lock_guard<std::mutex> lock(sv->mu);
        sv->stats.batches_built++;
    }

    // 2. the quantum of every batch, enqueued without waiting: each member advances by the quantum
    // or by the steps it has left, whichever is fewer (members in the order their batch was built)
    int launched[2] = { H1D_OK, H1D_OK };
    for (int alg = 0; alg < 2; ++alg) {
        if (!sv->batch[alg])
            continue;
        std::vector<uint32_t> steps;
        for (ServerReq *r : sv->active)
            if (r->rq.params.algorithm == alg) {
                r->tick_steps = std::min(static_cast<uint32_t>(sv->quantum), r->rq.n_steps - r->done_steps);
                steps.push_back(r->tick_steps);
            }
        launched[alg] = h1d_batch_advance_members_async(sv->batch[alg], steps.data());
    }

    // 3. admission while the batches run: every queued request that fits the budget (in arrival
    // order) and the device, its memory reserved under the lock, its run built outside it
    std::vector<ServerReq *> admitted;
    {
        size_t                      free_b = 0, total_b = 0;
        bool                        asked  = false;
        std::lock_guard<std::mutex> lock(sv->mu);
        for (auto it = sv->queue.begin(); it != sv->queue.end();) {
            ServerReq *r = *it;
            if (sv->used + r->bytes > sv->budget) {
                ++it;
                continue;
            }
            if (!asked) { // free device memory, and the blocks the library's pool keeps for reuse
                int dev = 0;
                cudaGetDevice(&dev);
                cudaMemGetInfo(&free_b, &total_b), asked = true;
                free_b += pool_idle_bytes(dev);
            }
            if (r->bytes + (size_t{ 256 } << 20) > free_b) {
                ++it;
                continue;
            }
            it         = sv->queue.erase(it);
            free_b     = free_b > r->bytes ? free_b - r->bytes : 0;
            sv->used  += r->bytes;
            sv->peak   = std::max(sv->peak, sv->used);
            r->state   = H1D_REQ_ACTIVE;
            r->t_admit = sv->now();
            sv->stats.admitted++;
            admitted.push_back(r);
        }
    }
    std::vector<std::pair<ServerReq *, int>> ended;  // (request, status) to publish
    std::vector<ServerReq *>                 joined; // built: they join the batches at the next tick
    for (ServerReq *r : admitted) {
        int const st = admit(sv->sort_interval, r);
        if (st != H1D_OK)
            ended.push_back({ r, st });
        else
            joined.push_back(r);
    }

    // 4. the end of the quantum: members whose run failed fail alone
    for (int alg = 0; alg < 2; ++alg) {
        if (!sv->batch[alg])
            continue;
        int const st = launched[alg] != H1D_OK ? launched[alg] : h1d_batch_synchronize(sv->batch[alg]);
        for (ServerReq *r : sv->active) {
            if (r->rq.params.algorithm != alg)
                continue;
            if (st == H1D_OK) {
                r->done_steps += r->tick_steps;
                continue;
            }
            // a failed launch fails every member; otherwise only the members whose run reports an error
            int const own = launched[alg] != H1D_OK ? st : h1d_synchronize(r->run);
            if (own != H1D_OK)
                ended.push_back({ r, own }), r->msg = h1d_status_string(r->run);
            else
                r->done_steps += r->tick_steps;
        }
    }

    // 5. finished and failed runs leave the batches, are read back and freed; new runs join
    std::vector<ServerReq *> leaving;
    for (auto it = sv->active.begin(); it != sv->active.end();) {
        ServerReq *r      = *it;
        bool const failed = std::any_of(ended.begin(), ended.end(), [r](auto const &e) { return e.first == r; });
        if (failed || r->done_steps >= r->rq.n_steps) {
            leaving.push_back(r);
            it = sv->active.erase(it);
        } else {
            ++it;
        }
    }
    if (!leaving.empty()) {
        drop_batches(sv);
        sv->dirty = true;
    }
    if (!joined.empty()) {
        sv->active.insert(sv->active.end(), joined.begin(), joined.end());
        sv->dirty = true;
    }
    std::vector<std::pair<ServerReq *, int>> results;
    for (ServerReq *r : leaving) {
        auto const f  = std::find_if(ended.begin(), ended.end(), [r](auto const &e) { return e.first == r; });
        int const  st = f != ended.end() ? f->second : collect(r);
        results.push_back({ r, st });
    }
    for (auto const &e : ended) // failed admissions are not in `leaving`
        if (std::find(leaving.begin(), leaving.end(), e.first) == leaving.end())
            results.push_back(e);
    {
        std::lock_guard<std::mutex> lock(sv->mu);
        for (auto const &[r, st] : results)
            finish_locked(sv, r, st, st == H1D_OK ? "" : (r->msg.empty() ? "run failed" : r->msg));
        sv->live = {};
        for (h1d_batch *b : sv->batch)
            if (b) {
                h1d_batch_stats st{};
                h1d_batch_stats_read(b, &st);
                sv->live.kernel_launches += st.kernel_launches, sv->live.graph_launches += st.graph_launches;
                sv->live.steps += st.steps;
            }
        if (n_active)
            *n_active = static_cast<int>(sv->active.size());
        if (n_queued)
            *n_queued = static_cast<int>(sv->queue.size());
    }
    for (auto const &[r, st] : results)
        if (r->run)
            h1d_destroy(r->run), r->run = nullptr;
    return H1D_OK;
}

int h1d_server_poll(h1d_server *sv, uint64_t id, int *state, double *t_submit, double *t_admit, double *t_done)
{
    if (!sv)
        return H1D_ERR_INVALID_ARG;
    std::lock_guard<std::mutex> lock(sv->mu);
    auto const it = sv->all.find(id);
    if (it == sv->all.end())
        return H1D_ERR_INVALID_ARG;
    ServerReq const *r = it->second;
    if (state)
        *state = r->state;
    if (t_submit)
        *t_submit = r->t_submit;
    if (t_admit)
        *t_admit = r->t_admit;
    if (t_done)
        *t_done = r->t_done;
    return r->state == H1D_REQ_FAILED ? r->status : H1D_OK;
}

int h1d_server_result(h1d_server *sv, uint64_t id, double *B, double *E, double *energy, double *n, double *nV,
                      double *nvv)
{
    if (!sv)
        return H1D_ERR_INVALID_ARG;
    std::lock_guard<std::mutex> lock(sv->mu);
    auto const it = sv->all.find(id);
    if (it == sv->all.end())
        return H1D_ERR_INVALID_ARG;
    ServerReq *r = it->second;
    if (r->state == H1D_REQ_FAILED)
        return r->status;
    if (r->state != H1D_REQ_DONE)
        return H1D_ERR_STATE;
    auto cp = [](double *dst, std::vector<double> const &v) {
        if (dst && !v.empty())
            std::memcpy(dst, v.data(), sizeof(double) * v.size());
    };
    cp(B, r->B), cp(E, r->E), cp(energy, r->energy), cp(n, r->n), cp(nV, r->nV), cp(nvv, r->nvv);
    return H1D_OK;
}

int h1d_server_release(h1d_server *sv, uint64_t id)
{
    if (!sv)
        return H1D_ERR_INVALID_ARG;
    std::lock_guard<std::mutex> lock(sv->mu);
    auto const it = sv->all.find(id);
    if (it == sv->all.end() || (it->second->state != H1D_REQ_DONE && it->second->state != H1D_REQ_FAILED))
        return H1D_ERR_STATE;
    delete it->second;
    sv->all.erase(it);
    return H1D_OK;
}

int h1d_server_stats_read(h1d_server *sv, h1d_server_stats *out)
{
    if (!sv || !out)
        return H1D_ERR_INVALID_ARG;
    std::lock_guard<std::mutex> lock(sv->mu);
    *out = sv->stats;
    out->kernel_launches += sv->live.kernel_launches, out->graph_launches += sv->live.graph_launches;
    out->steps += sv->live.steps;
    out->bytes_in_use = static_cast<int64_t>(sv->used);
    out->peak_bytes   = static_cast<int64_t>(sv->peak);
    return H1D_OK;
}

int h1d_server_destroy(h1d_server *sv)
{
    if (!sv)
        return H1D_OK;
    std::lock_guard<std::mutex> tick(sv->tick_mu);
    for (h1d_batch *&b : sv->batch)
        if (b)
            h1d_batch_destroy(b), b = nullptr;
    for (auto &[id, r] : sv->all) {
        if (r->run)
            h1d_destroy(r->run);
        delete r;
    }
    delete sv;
    return H1D_OK;
}

} // extern "C"

// ---- checkpoint / resume ------------------------------------------------------------------------
// The content of the reference's snapshot (Recorder/Snapshot.cc:148-185, 330-375): step count, a
// signature of the parameters (Hash{serialize(params)}, Snapshot.cc:19, 340-342), B and E, the
// particles of every kinetic species (here with their ids and, when their weights evolve, their
// real_f and marker, in the run's own precision so that a resume is exact) and mom0_full /
// mom1_full of every cold species.  Sources and the push record are recomputed on the first step
// after a resume, as after the reference's snapshot load; the delta-f equilibrium moments that the
// snapshot stores are a function of the parameters and are rebuilt by h1d_create.

namespace {

struct CkptHeader {
    char     magic[8];
    uint32_t version, precision;
    uint64_t signature;
    int64_t  step, Nx;
    int32_t  n_kinetic, n_cold;
    int64_t  n[H1D_MAX_KINETIC];
};
constexpr char     CKPT_MAGIC[8] = { 'H', '1', 'D', 'C', 'K', 'P', 'T', 0 };
constexpr uint32_t CKPT_VERSION  = 3;

// FNV-1a over the run's parameters with the tuning knob (sort interval) cleared
uint64_t params_signature(h1d_params p)
{
    p.sort_interval = 0;
    unsigned char const *b = reinterpret_cast<unsigned char const *>(&p);
    uint64_t             h = 1469598103934665603ULL;
    for (size_t i = 0; i < sizeof p; ++i)
        h = (h ^ b[i]) * 1099511628211ULL;
    return h;
}

// bytes of species s with n particles: the record, the id, and real_f / marker when its weights evolve
size_t particle_bytes(h1d_run const *run, int s, int64_t n)
{
    size_t const psd = evolves_psd(run->p.kinetic[s]) ? 2 * (run->mixed ? 4 : 8) : 0;
    return static_cast<size_t>(n) * ((run->mixed ? 5 * 4 + 4 : 5 * 8 + 4) + psd);
}

size_t ckpt_size(h1d_run const *run)
{
    size_t b = sizeof(CkptHeader) + sizeof(double) * 6 * run->M + sizeof(double) * 4 * run->M * run->p.n_cold;
    for (int s = 0; s < run->p.n_kinetic; ++s)
        b += particle_bytes(run, s, run->sp[s].n);
    return b;
}

} // namespace

extern "C" {

int h1d_checkpoint_size(h1d_run *run, size_t *bytes)
{
    if (!run || !bytes)
        return H1D_ERR_INVALID_ARG;
    for (int s = 0; s < run->p.n_kinetic; ++s) { // exact counts (absorbed particles trimmed)
        int64_t n = 0;
        TRY(h1d_particle_count(run, s, &n));
    }
    *bytes = ckpt_size(run);
    return H1D_OK;
}

int h1d_checkpoint_save(h1d_run *run, void *buffer, size_t capacity, size_t *written)
{
    size_t need = 0;
    TRY(h1d_checkpoint_size(run, &need));
    if (!buffer || capacity < need)
        return set_err(run, H1D_ERR_INVALID_ARG, fmt("h1d_checkpoint_save: the buffer needs %zu bytes", need));
    if (run->fields_dirty)
        TRY(prepare_fields(run)); // ghost cells as the first step would fill them
    CkptHeader hd{};
    std::memcpy(hd.magic, CKPT_MAGIC, sizeof hd.magic);
    hd.version = CKPT_VERSION, hd.precision = static_cast<uint32_t>(run->p.precision);
    hd.signature = params_signature(run->p), hd.step = run->step, hd.Nx = run->Nx;
    hd.n_kinetic = run->p.n_kinetic, hd.n_cold = run->p.n_cold;
    for (int s = 0; s < run->p.n_kinetic; ++s)
        hd.n[s] = run->sp[s].n;
    auto *out = static_cast<unsigned char *>(buffer);
    std::memcpy(out, &hd, sizeof hd);
    size_t off = sizeof hd;
    auto   d2h = [&](void const *src, size_t bytes) -> cudaError_t {
        cudaError_t const e = bytes ? cudaMemcpyAsync(out + off, src, bytes, cudaMemcpyDeviceToHost, run->stream) : cudaSuccess;
        off += bytes;
        return e;
    };
    long const M = run->M;
    CU(d2h(run->B[run->fcur], sizeof(double) * 3 * M));
    CU(d2h(run->E[run->fcur], sizeof(double) * 3 * M));
    for (int c = 0; c < run->p.n_cold; ++c) {
        CU(d2h(run->cold[c].n, sizeof(double) * M));
        CU(d2h(run->cold[c].nV[run->cold[c].cur], sizeof(double) * 3 * M));
    }
    for (int s = 0; s < run->p.n_kinetic; ++s) {
        SpeciesState const &S = run->sp[s];
        size_t const        n = static_cast<size_t>(S.n);
        if (run->mixed) {
            CU(d2h(S.pos[S.cur], 4 * n));
            for (int k = 0; k < 4; ++k)
                CU(d2h(S.fbuf[S.cur][k], 4 * n));
        } else {
            for (int k = 0; k < 5; ++k)
                CU(d2h(S.buf[S.cur][k], 8 * n));
        }
        CU(d2h(S.pid[S.cur], 4 * n));
        if (evolves_psd(run->p.kinetic[s]))
            for (int k = 0; k < 2; ++k)
                CU(run->mixed ? d2h(S.fpsd[S.cur][k], 4 * n) : d2h(S.psd[S.cur][k], 8 * n));
    }
    CU(cudaStreamSynchronize(run->stream));
    if (written)
        *written = off;
    return H1D_OK;
}

int h1d_checkpoint_load(h1d_run *run, void const *buffer, size_t size)
{
    if (!run || !buffer || size < sizeof(CkptHeader))
        return set_err(run, H1D_ERR_INVALID_ARG, "h1d_checkpoint_load: no checkpoint");
    CkptHeader hd;
    std::memcpy(&hd, buffer, sizeof hd);
    if (std::memcmp(hd.magic, CKPT_MAGIC, sizeof hd.magic) != 0 || hd.version != CKPT_VERSION)
        return set_err(run, H1D_ERR_INVALID_ARG, "h1d_checkpoint_load: not a checkpoint of this library version");
    if (hd.signature != params_signature(run->p) || hd.Nx != run->Nx || hd.n_kinetic != run->p.n_kinetic
        || hd.n_cold != run->p.n_cold)
        return set_err(run, H1D_ERR_INVALID_ARG, "h1d_checkpoint_load: signature verification failed");
    size_t need = sizeof hd + sizeof(double) * 6 * run->M + sizeof(double) * 4 * run->M * run->p.n_cold;
    for (int s = 0; s < run->p.n_kinetic; ++s) {
        if (hd.n[s] < 0 || hd.n[s] > (int64_t{ 1 } << 31) - 1)
            return set_err(run, H1D_ERR_INVALID_ARG, "h1d_checkpoint_load: corrupt particle count");
        need += particle_bytes(run, s, hd.n[s]);
    }
    if (size < need)
        return set_err(run, H1D_ERR_INVALID_ARG, "h1d_checkpoint_load: truncated checkpoint");
    CU(cudaStreamSynchronize(run->stream));
    auto const *in  = static_cast<unsigned char const *>(buffer);
    size_t      off = sizeof hd;
    auto        h2d = [&](void *dst, size_t bytes) -> cudaError_t {
        cudaError_t const e = bytes ? cudaMemcpyAsync(dst, in + off, bytes, cudaMemcpyHostToDevice, run->stream) : cudaSuccess;
        off += bytes;
        return e;
    };
    long const M = run->M;
    CU(h2d(run->B[run->fcur], sizeof(double) * 3 * M));
    CU(h2d(run->E[run->fcur], sizeof(double) * 3 * M));
    for (int c = 0; c < run->p.n_cold; ++c) {
        ColdState &C = run->cold[c];
        CU(h2d(C.n, sizeof(double) * M));
        CU(h2d(C.nV[C.cur], sizeof(double) * 3 * M));
        CU(cudaMemcpyAsync(C.nV[1 - C.cur], C.nV[C.cur], sizeof(double) * 3 * M, cudaMemcpyDeviceToDevice, run->stream));
    }
    for (int s = 0; s < run->p.n_kinetic; ++s) {
        SpeciesState &S = run->sp[s];
        TRY(ensure_capacity(run, s, hd.n[s]));
        S.cur = 0, S.n = hd.n[s];
        size_t const n = static_cast<size_t>(S.n);
        if (run->mixed) {
            CU(h2d(S.pos[0], 4 * n));
            for (int k = 0; k < 4; ++k)
                CU(h2d(S.fbuf[0][k], 4 * n));
        } else {
            for (int k = 0; k < 5; ++k)
                CU(h2d(S.buf[0][k], 8 * n));
        }
        CU(h2d(S.pid[0], 4 * n));
        if (evolves_psd(run->p.kinetic[s]))
            for (int k = 0; k < 2; ++k)
                CU(run->mixed ? h2d(S.fpsd[0][k], 4 * n) : h2d(S.psd[0][k], 8 * n));
        CU(cudaMemsetAsync(S.dep, 0, sizeof(double) * 16 * M, run->stream)); // no deposit in flight
        S.since_sort = 1 << 30;
    }
    CU(cudaStreamSynchronize(run->stream));
    run->step          = hd.step;
    run->recurring     = false; // the next advance starts like the reference's after a snapshot load
    run->fields_dirty  = true;
    run->moments_stale = true;
    run->gen++;
    return H1D_OK;
}

int h1d_step_count(h1d_run *run, int64_t *step)
{
    if (!run || !step)
        return H1D_ERR_INVALID_ARG;
    *step = run->step;
    return H1D_OK;
}

} // extern "C"
