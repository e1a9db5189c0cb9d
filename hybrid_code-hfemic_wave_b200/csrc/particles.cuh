// Particle kernels of the hybrid_1d hot path (FP64).
//
// One fused pass per species and CAM-CL step does what the reference does in four loops over
// the particle deque (src/hybrid_1d/Core/Domain_CAMCL.cc:69-82):
//   PartSpecies::update_vel   interp of E and dB at x^N, mirror-field B, Boris push   (PartSpecies.cc:105-109, 161-176)
//   PartSpecies::collect_part deposit of n and nV at x^N with v^{N+1/2}                (PartSpecies.cc:115-128, 210-224)
//   PartSpecies::update_pos   x^{N+1} = x^N + v.e^1 dt, travel check                   (PartSpecies.cc:110-114, 147-159)
//   Delegate::boundary_pass   periodic wrap / reflection (+ gyro-phase)               (Delegate.cc:51-74, 101-156)
//   PartSpecies::collect_part deposit of n and nV at x^{N+1}                          (PartSpecies.cc:115-128, 210-224)
// Particles are structure-of-arrays and cell-sorted (sort.cuh), so the particles of a warp span a
// few cells.  Each warp deposits into a window of PIPE_W cells held in shared memory as
// lane-private columns; a window is summed over its 32 columns and added to the global moment
// arrays (one atomic per cell and quantity) only when it has to move.  Moments are accumulated
// unscaled; the 1/Nc factor of collect_part is applied by the field kernel.
#pragma once

#include "device_common.cuh"
#include "h1d_gpu.h"
#include "tma.cuh"

namespace h1d {

enum { BCK_PERIODIC = 0, BCK_REFLECTING = 1, BCK_ABSORBING = 2 };

struct PushArgs {
    double        *q1, *vx, *vy, *vz;
    double        *w; // writable only for absorption (w = 0 marks a removed particle)
    int32_t const *pid;
    int64_t        n;
    int            Nx;
    double const  *EB; // per cell {Ex, Ey, Ez, dBx, dBy, dBz}: E and B averaged onto the half grid
                       // (PartSpecies.cc:27-34), pointer at interior cell 0
    double        *dep[2][4]; // [deposit at x^N | x^{N+1}][n, nVx, nVy, nVz], at cell 0
    double        *nvv[6];    // collect_all's xx, yy, zz, xy, yz, zx sums at cell 0 (NVV launches only)
    double         half_min, full_min, full_max, full_len;
    double         xi, xi2, xiD1, D1, inv_D1, O0, Oc, dt, travel_scale, xiO0_Oc;
    BorisK         boris;
    unsigned      *status;
    unsigned long long *fallbacks; // deposits outside their warp's window (diagnostic)
    uint64_t       seed, counter;
    int            species, randomize, homogeneous_poly;
    int            move_steps; // 1: CAM-CL full step; 2: PC half step, push, half step; 0: deposit only
    int            deposit_mask; // bit0: deposit at x^N, bit1: deposit at the end position
    int            write_back;   // 0 for the PC predictor (particles are not kept)
    // evolving weights (push_kernel<..., PSD = true>): Particle::PSD arrays and the equilibrium
    // f0 of PartSpecies::impl_update_weight (PartSpecies.cc:178-208)
    double        *real_f, *marker;
    double         nu_dt;          // psd_refresh_frequency * dt
    double         vth1, vth1_cubed, T2_T1;
    double         vc[4];          // constants of the distribution `vdf` (equilibrium_f0)
    int            vdf;            // H1D_VDF_*
    int            psd_refresh;    // nu != 0
    int            delta_f;        // weight = (real_f - f0) / marker, else real_f / marker
};

template <int O>
__device__ __forceinline__ bool stencil_ok(Shape<O> const &sh, int Nx)
{
    return sh.i0 >= -PAD && sh.i0 + O < Nx + PAD;
}

// x^N -> x^N + v.e^1 dt (CurviBasis.h:65-69: contravariant q1-velocity = v_x cos^2 / D1)
template <bool MIRROR>
__device__ __forceinline__ double contr_vx(PushArgs const &a, double q1, double vx)
{
    if constexpr (MIRROR) {
        double s, c;
        sincos_taylor(a.xiD1 * q1, s, c);
        return (a.inv_D1 * (c * c)) * vx;
    } else {
        return a.inv_D1 * vx;
    }
}

template <bool MIRROR>
__device__ __forceinline__ double move(PushArgs const &a, double &q1, double vx, double dt)
{
    double moved = contr_vx<MIRROR>(a, q1, vx) * dt;
    q1 += moved;
    moved *= a.travel_scale;
    return moved;
}

// particle boundary pass for one particle; returns false if the particle left the system
template <int BC>
__device__ __forceinline__ bool boundary(PushArgs const &a, double &q1, d3 &v, int32_t pid, uint64_t counter)
{
    if constexpr (BC == BCK_PERIODIC) {
        if (q1 < a.full_min)
            q1 += a.full_len;
        else if (q1 >= a.full_max)
            q1 -= a.full_len;
        return true;
    } else if constexpr (BC == BCK_REFLECTING) {
        bool const left = q1 < a.full_min, right = q1 >= a.full_max;
        if (left || right) {
            double const ext = left ? a.full_min : a.full_max;
            q1 += 2 * (ext - q1);
            v.x = v.x - 2 * v.x; // v -= 2 (v.e1) e1 with e1 = x^
            if (a.randomize) {
                double s, c;
                sincos_half_turn(gyrophase(a.seed, counter, (uint64_t)a.species, (uint64_t)pid), s, c);
                double const vy = v.y, vz = v.z;
                v.y = vy * c - vz * s;
                v.z = vy * s + vz * c;
            }
        }
        return true;
    } else {
        return q1 >= a.full_min && q1 < a.full_max;
    }
}

// background mirror field at the particle with its gyro-radius offset (PartSpecies.cc:169-174;
// MFABasis.h:72-75; MirrorGeometry.h:68-71; MirrorGeometry.cc:34-47).  With c = cos(xi D1 q1), s = sin(xi D1 q1):
// B/B0 = 1/c^2, x = tan/xi, rL = (-vz, vy) c^2/Oc, so the transverse components
// -xi^2 x rL O0 reduce to (xi O0/Oc) s c (vz, -vy).  Also returns c^2 for the move.
template <bool MIRROR>
__device__ __forceinline__ d3 background_B(PushArgs const &a, double q1, d3 v, double &c2)
{
    if constexpr (MIRROR) {
        double s, c;
        sincos_taylor(a.xiD1 * q1, s, c);
        c2               = c * c;
        double const ksc = a.xiO0_Oc * (s * c);
        return { a.O0 / c2, ksc * v.z, -ksc * v.y };
    } else {
        c2 = 1;
        return { a.O0, 0, 0 };
    }
}

// The equilibrium f0(v, q1) of a species' distribution (VDF::real_f0), with cs = cos(xi D1 q1).
// cart_to_mfa is the identity on the field line (MFABasis.h:98-100), so v is field-aligned; every
// f0 is n0(q1) times a velocity distribution normalised to one.
//  - bi-Maxwellian (MaxwellianVDF.cc:33-43, 67-81): n0 = eta = 1 / (T + (1 - T) cs^2), T = T2OT1_eq
//    (T2_T1), T2OT1 = T eta; f0 = n0 exp(-x1^2) pi^-1/2 exp(-x_perp^2 / T2OT1) / (pi T2OT1) / vth1^3,
//    x = v / vth1.
//  - loss-cone (LossconeVDF.cc:46-117): vc = {beta_eq, X = xth2_eq^2, beta_eq X}; eta as above with
//    X, eta_b with beta_eq X, n0 = (eta - beta_eq eta_b) / (1 - beta_eq), xth2^2 = X eta,
//    beta = beta_eq eta_b / eta (kept 1e-10 away from 1); the perpendicular factor is
//    (exp(-y) - exp(-y / beta)) / (pi xth2^2 (1 - beta)) with y = x_perp^2 / xth2^2.
//  - partial shell (PartialShellVDF.cc:78-93, 125-140): vc = {zeta, xs, A(xs), B(zeta)}; n0 = cs^zeta;
//    f0 = n0 exp(-(x - xs)^2) / A sin^zeta(alpha) / B / (2 pi vth^3), x = |v| / vth,
//    cos(alpha) = x1 / x.
//  - counter-beam (CounterBeamVDF.cc:99-132): vc = {nu0, xs, A(xs), B(nu0)}; nu = nu0 / cs
//    (B/B0 = 1/cs^2), n0 = B(nu) / B(nu0) and the pitch-angle factor
//    exp(-sin^2(alpha) / nu^2) / B(nu): their product needs no B(nu), so
//    f0 = exp(-(x - xs)^2) / A exp(-sin^2(alpha) cs^2 / nu0^2) / B(nu0) / (2 pi vth^3).
__device__ __forceinline__ double equilibrium_f0(PushArgs const &a, d3 v, double cs)
{
    constexpr double PI = 3.141592653589793, HALF_2_SQRTPI = 1.1283791670955126 * .5;
    double const     x1 = v.x / a.vth1, x2 = v.y / a.vth1, x3 = v.z / a.vth1;
    if (a.vdf == H1D_VDF_LOSSCONE) {
        double const X = a.vc[1], bX = a.vc[2], beq = a.vc[0];
        double const eta   = 1 / (X + (1 - X) * cs * cs);
        double const eta_b = 1 / (bX + (1 - bX) * cs * cs);
        double       beta  = beq * eta_b / eta;
        if (fabs(beta - 1) < 1e-10)
            beta += copysign(1e-10, beta - 1);
        double const n0 = (eta - beq * eta_b) / (1 - beq);
        double const x2s = X * eta;
        double const y   = (x2 * x2 + x3 * x3) / x2s;
        double const f1  = exp(-x1 * x1) * HALF_2_SQRTPI;
        double const f2  = (exp(-y) - exp(-y / beta)) / (PI * x2s * (1 - beta));
        return n0 * ((f1 * f2) / a.vth1_cubed);
    }
    if (a.vdf == H1D_VDF_PARTIAL_SHELL || a.vdf == H1D_VDF_COUNTER_BEAM) {
        double const x  = sqrt(x1 * x1 + x2 * x2 + x3 * x3);
        double const t  = x - a.vc[1];
        double const fv = exp(-t * t) / a.vc[2];
        double const u  = x1 / x; // cos(alpha)
        if (a.vdf == H1D_VDF_PARTIAL_SHELL) {
            bool const   iso = a.vc[0] == 0;
            double const fa  = (iso ? 1 : pow((1 - u) * (1 + u), .5 * a.vc[0])) / a.vc[3];
            double const n0  = iso ? 1 : pow(cs, a.vc[0]);
            return n0 * (.5 * fv * fa / (PI * a.vth1_cubed));
        }
        double const fa = exp(-((1 - u) * (1 + u)) * (cs * cs) / (a.vc[0] * a.vc[0])) / a.vc[3];
        return fv * fa / (2 * PI * a.vth1_cubed);
    }
    double const eta   = 1 / (a.T2_T1 + (1 - a.T2_T1) * cs * cs);
    double const T2OT1 = a.T2_T1 * eta;
    double const f1    = exp(-x1 * x1) * HALF_2_SQRTPI;
    double const f2    = exp(-(x2 * x2 + x3 * x3) / T2OT1) / (PI * T2OT1);
    return (1 * eta) * ((f1 * f2) / a.vth1_cubed);
}
// PartSpecies::impl_update_weight for one particle after its velocity update: the new weight,
// with real_f relaxed toward f0 when the PSD is refreshed
__device__ __forceinline__ double update_weight(PushArgs const &a, d3 v, double q1, double &real_f, double marker)
{
    double cs = 1;
    if (a.xi != 0) {
        double sn;
        sincos_taylor(a.xiD1 * q1, sn, cs);
    }
    double const f0 = equilibrium_f0(a, v, cs);
    if (a.psd_refresh)
        real_f = (real_f + a.nu_dt * f0) / (1 + a.nu_dt);
    return a.delta_f ? (real_f - f0) / marker : real_f / marker;
}

// E and dB interpolated at the particle (GridArray.h:110-119) from the interleaved cell records
template <int O>
__device__ __forceinline__ void interp_EB(double const *eb, Shape<O> const &sh, d3 &E, d3 &B)
{
    E = { 0, 0, 0 };
    B = { 0, 0, 0 };
#pragma unroll
    for (int j = 0; j <= O; ++j) {
        double2 const *p = reinterpret_cast<double2 const *>(eb + 6 * (sh.i0 + j));
        double2 const  x = __ldg(p), y = __ldg(p + 1), z = __ldg(p + 2);
        double const   w = sh.w[j];
        E.x += x.x * w, E.y += x.y * w, E.z += y.x * w;
        B.x += y.y * w, B.y += z.x * w, B.z += z.y * w;
    }
}

// ------------------------------------------------------------------------------------------------
// The particle pass.  Warp-specialised pipeline per CTA: one producer warp streams the CTA's
// contiguous run of chunks (PIPE_CHUNK particles each) global -> shared with 1-D TMA bulk copies
// completing on mbarriers (PIPE_STAGES deep) and bulk-stores the updated particles back;
// PIPE_CONSUMER_WARPS warps compute.  A consumer warp owns 32 x PIPE_PPT consecutive (cell-sorted)
// particles of each chunk and, per particle: pushes at x^N, moves, applies the boundary, writes
// the result beside the inputs, and deposits at x^N (with the pre-boundary velocity) and at the
// end position into its shared-memory window.
//
// CAM-CL (move_steps == 1): push at x^N, deposit, move, BC, deposit.
// Predictor-corrector (move_steps == 2, Domain_PC.cc:110-124, 169-181): half move, BC, push at
// the half-step position, half move, BC, deposit.  move_steps == 0: deposit only
// (Domain_PC.cc:36-44).
// ------------------------------------------------------------------------------------------------
// The pipeline's shape: particles per chunk (128 or 256: one or two per consumer lane), stages,
// CTAs per SM and cells per deposit window; a build may set them with -DH1D_FP64_<NAME>=value.
#ifndef H1D_FP64_CHUNK
#define H1D_FP64_CHUNK 256
#endif
#ifndef H1D_FP64_STAGES
#define H1D_FP64_STAGES 2
#endif
#ifndef H1D_FP64_CTAS
#define H1D_FP64_CTAS 3
#endif
#ifndef H1D_FP64_W
#define H1D_FP64_W 6
#endif
constexpr int PIPE_CONSUMER_WARPS = 4;
constexpr int PIPE_THREADS        = 32 * (PIPE_CONSUMER_WARPS + 1);
constexpr int PIPE_CHUNK          = H1D_FP64_CHUNK;
constexpr int PIPE_PPT            = PIPE_CHUNK / (32 * PIPE_CONSUMER_WARPS);
constexpr int PIPE_STAGES         = H1D_FP64_STAGES;
constexpr int PIPE_CTAS_PER_SM    = H1D_FP64_CTAS;
constexpr int PIPE_W              = H1D_FP64_W; // cells per deposit window: 4 quantities x W cells, flushed over 32 lanes
static_assert(PIPE_PPT == 1 || PIPE_PPT == 2, "one or two particles per consumer lane and chunk");
static_assert(4 * PIPE_W <= 32 && PIPE_W >= 4, "a window flush reduce-scatters at most 32 values; a cubic stencil fits");

// a stage holds one chunk; the consumers overwrite it in place with the new state, which the
// producer then stores.  With evolving weights (PSD) a stage also holds real_f and marker, and
// the pipeline is one stage shorter so that two CTAs still fit an SM.
template <bool PSD>
struct PipeStageT {
    double  q1[PIPE_CHUNK], vx[PIPE_CHUNK], vy[PIPE_CHUNK], vz[PIPE_CHUNK], w[PIPE_CHUNK];
    int32_t pid[PIPE_CHUNK];
    double  real_f[PSD ? PIPE_CHUNK : 2], marker[PSD ? PIPE_CHUNK : 2];
};
using PipeStage = PipeStageT<false>;
template <bool PSD>
struct PipeLayout {
    static constexpr int    STAGES     = PIPE_STAGES;
    static constexpr size_t BAR_OFFSET = sizeof(PipeStageT<PSD>) * STAGES;
    static constexpr size_t COL_OFFSET = BAR_OFFSET + 128;
};
constexpr size_t PIPE_COL_BYTES  = sizeof(double2) * PIPE_CONSUMER_WARPS * 2 * PIPE_W * 2 * 32;
constexpr size_t PIPE_SMEM       = PipeLayout<false>::COL_OFFSET + PIPE_COL_BYTES;
constexpr size_t PIPE_SMEM_PSD   = PipeLayout<true>::COL_OFFSET + PIPE_COL_BYTES;
static_assert(2 * PIPE_STAGES * sizeof(uint64_t) <= 128, "barriers fit before the columns");
static_assert(2 * (PIPE_SMEM_PSD + 1024) <= 233472, "two CTAs with evolving weights fit an SM");
// a launch that also forms collect_all's second moments (NVV, the last step of an advance_by)
// holds a second window per warp: three double2 columns per cell; two CTAs fit an SM
constexpr size_t PIPE_NVV_BYTES = sizeof(double2) * 3 * PIPE_CONSUMER_WARPS * PIPE_W * 32;
constexpr size_t PIPE_SMEM_NVV  = PipeLayout<false>::COL_OFFSET + PIPE_COL_BYTES + PIPE_NVV_BYTES;
static_assert(2 * (PIPE_SMEM_NVV + 1024) <= 233472, "two CTAs of a second-moment launch fit an SM");

__device__ __forceinline__ uint32_t round16(uint32_t b) { return (b + 15u) & ~15u; }

// warp reduce-scatter by recursive halving of V (16 or 32) values: after log2(V) exchange rounds
// (V/2 + V/4 + ... shuffles) and a butterfly over the remaining lane bits, lane l holds the warp
// total of value (l >> (5 - log2 V))
template <int V>
__device__ __forceinline__ double reduce_scatter(double (&x)[V], int lane)
{
    static_assert(V == 16 || V == 32, "V must be 16 or 32");
#pragma unroll
    for (int h = V / 2, m = 16; h >= 1; h >>= 1, m >>= 1) {
        bool const up = (lane & m) != 0;
#pragma unroll
        for (int j = 0; j < h; ++j) {
            double const send = up ? x[j] : x[j + h];
            double const keep = up ? x[j + h] : x[j];
            x[j]              = keep + __shfl_xor_sync(0xffffffffu, send, m);
        }
    }
    double v = x[0];
    if constexpr (V == 16)
        v += __shfl_xor_sync(0xffffffffu, v, 1);
    return v;
}

// A warp's deposit window of PIPE_W cells from `base`: lane-private columns, for deposit d (at
// x^N / at the end position) and cell c two double2 {n, nVx}, {nVy, nVz}, lane-contiguous so a
// warp's access is conflict-free whatever the cells of its lanes.
struct ColWindow64 {
    static constexpr int NONE = -0x40000000;
    double2             *col;
    int                  base;

    __device__ __forceinline__ double2 &at(int d, int c, int h, int lane) { return col[((d * PIPE_W + c) * 2 + h) * 32 + lane]; }
    __device__ __forceinline__ void     zero(int lane)
    {
#pragma unroll
        for (int d = 0; d < 2; ++d)
#pragma unroll
            for (int c = 0; c < PIPE_W; ++c)
                at(d, c, 0, lane) = make_double2(0, 0), at(d, c, 1, lane) = make_double2(0, 0);
    }
    template <int O>
    __device__ __forceinline__ void add(int d, Shape<O> const &sh, double const (&vw)[4], int lane)
    {
        int const r = sh.i0 - base;
#pragma unroll
        for (int j = 0; j <= O; ++j) {
            double2 &e0 = at(d, r + j, 0, lane);
            double2 &e1 = at(d, r + j, 1, lane);
            double2  a0 = e0, a1 = e1;
            a0.x = fma(vw[0], sh.w[j], a0.x), a0.y = fma(vw[1], sh.w[j], a0.y);
            a1.x = fma(vw[2], sh.w[j], a1.x), a1.y = fma(vw[3], sh.w[j], a1.y);
            e0 = a0, e1 = a1;
        }
    }
    __device__ __forceinline__ void flush_one(int d, int lane, PushArgs const &a)
    {
        double x[32];
#pragma unroll
        for (int c = 0; c < PIPE_W; ++c) {
            double2 const u = at(d, c, 0, lane), v = at(d, c, 1, lane);
            x[4 * c] = u.x, x[4 * c + 1] = u.y, x[4 * c + 2] = v.x, x[4 * c + 3] = v.y;
            at(d, c, 0, lane) = make_double2(0, 0), at(d, c, 1, lane) = make_double2(0, 0);
        }
#pragma unroll
        for (int k = 4 * PIPE_W; k < 32; ++k)
            x[k] = 0.0;
        double const t = reduce_scatter<32>(x, lane); // lane l: value l = 4 * cell + quantity
        if (t != 0.0) {
            int const cell = base + (lane >> 2);
            if (cell >= -PAD && cell < a.Nx + PAD)
                atomicAdd(a.dep[d][lane & 3] + cell, t);
            else
                atomicOr(a.status, ST_OUT_OF_RANGE);
        }
    }
    __device__ __forceinline__ void flush(int lane, PushArgs const &a)
    {
        if (base == NONE)
            return;
        if (a.deposit_mask & 1)
            flush_one(0, lane, a);
        if (a.deposit_mask & 2)
            flush_one(1, lane, a);
    }
};

// collect_all's second moments w v_i v_j of the deposit at the end position (NVV launches): per
// warp, cell and lane the double2 columns {xx, yy}, {zz, xy}, {yz, zx}, over the cells of the
// warp's main window (same base, flushed and moved with it)
struct NvvWindow64 {
    double2 *col;

    __device__ __forceinline__ double2 &at(int c, int h, int lane) { return col[(c * 3 + h) * 32 + lane]; }
    __device__ __forceinline__ void     zero(int lane)
    {
#pragma unroll
        for (int c = 0; c < PIPE_W; ++c)
#pragma unroll
            for (int h = 0; h < 3; ++h)
                at(c, h, lane) = make_double2(0, 0);
    }
    template <int O>
    __device__ __forceinline__ void add(int base, Shape<O> const &sh, double const (&v)[6], int lane)
    {
        int const r = sh.i0 - base;
#pragma unroll
        for (int j = 0; j <= O; ++j)
#pragma unroll
            for (int h = 0; h < 3; ++h) {
                double2 &e = at(r + j, h, lane);
                double2  t = e;
                t.x = fma(v[2 * h], sh.w[j], t.x), t.y = fma(v[2 * h + 1], sh.w[j], t.y);
                e   = t;
            }
    }
    // the columns summed over the warp and added to the moment sums: {xx, yy, zz, xy} of the
    // PIPE_W cells in one 32-value reduce-scatter (lane l < 4 PIPE_W: value l = 4 c + q), {yz, zx}
    // in a 16-value one (lanes 2 k, 2 k + 1: value k = 2 c + q)
    __device__ __forceinline__ void flush(int base, int lane, PushArgs const &a)
    {
        if (base == ColWindow64::NONE)
            return;
        double x[32], y[16];
#pragma unroll
        for (int k = 0; k < 32; ++k)
            x[k] = 0.0;
#pragma unroll
        for (int k = 0; k < 16; ++k)
            y[k] = 0.0;
#pragma unroll
        for (int c = 0; c < PIPE_W; ++c) {
            double2 const u = at(c, 0, lane), v = at(c, 1, lane), w = at(c, 2, lane);
            x[4 * c] = u.x, x[4 * c + 1] = u.y, x[4 * c + 2] = v.x, x[4 * c + 3] = v.y;
            y[2 * c] = w.x, y[2 * c + 1] = w.y;
#pragma unroll
            for (int h = 0; h < 3; ++h)
                at(c, h, lane) = make_double2(0, 0);
        }
        double const t0 = reduce_scatter<32>(x, lane);
        double const t1 = reduce_scatter<16>(y, lane);
        unsigned     bad = 0;
        if (lane < 4 * PIPE_W && t0 != 0.0) {
            int const cell = base + (lane >> 2);
            if (cell >= -PAD && cell < a.Nx + PAD)
                atomicAdd(a.nvv[lane & 3] + cell, t0);
            else
                bad = ST_OUT_OF_RANGE;
        }
        int const k = lane >> 1;
        if ((lane & 1) == 0 && k < 2 * PIPE_W && t1 != 0.0) {
            int const cell = base + (k >> 1);
            if (cell >= -PAD && cell < a.Nx + PAD)
                atomicAdd(a.nvv[4 + (k & 1)] + cell, t1);
            else
                bad = ST_OUT_OF_RANGE;
        }
        if (bad)
            atomicOr(a.status, bad);
    }
};

template <int O>
__device__ __forceinline__ void nvv_direct(PushArgs const &a, Shape<O> const &sh, double const (&v)[6])
{
#pragma unroll
    for (int j = 0; j <= O; ++j)
#pragma unroll
        for (int q = 0; q < 6; ++q)
            atomicAdd(a.nvv[q] + sh.i0 + j, v[q] * sh.w[j]);
}

template <int O>
__device__ __forceinline__ void deposit_direct(PushArgs const &a, int d, Shape<O> const &sh, double const (&vw)[4])
{
    atomicAdd(a.fallbacks, 1ull);
#pragma unroll
    for (int j = 0; j <= O; ++j)
#pragma unroll
        for (int q = 0; q < 4; ++q)
            atomicAdd(a.dep[d][q] + sh.i0 + j, vw[q] * sh.w[j]);
}

// The groups of particles one launch of the pass covers: a run's species (one group per launch)
// or the species of many runs of an ensemble (up to MAXG per launch).  The launch's chunks are
// numbered consecutively over the groups; a CTA takes a contiguous range of them, and its warps
// flush their deposit windows and status bits whenever the range crosses into the next group.
// The table travels as the kernel's parameter block (at most 32 KB).
template <int MAXG>
struct PushGroups {
    static constexpr int MAX = MAXG;
    int      n;
    int64_t  chunk0[MAXG + 1]; // first chunk of each group; chunk0[n] = number of chunks
    PushArgs g[MAXG];
};

template <int MAXG>
__device__ __forceinline__ int group_of(PushGroups<MAXG> const &G, int64_t chunk, int from)
{
    if constexpr (MAXG == 1) {
        return 0;
    } else {
        int g = from < 0 ? 0 : from;
        while (g + 1 < G.n && chunk >= G.chunk0[g + 1])
            ++g;
        return g;
    }
}

template <int O, bool MIRROR, int BC, int MAXG, bool PSD = false, bool NVV = false>
__global__ void __launch_bounds__(PIPE_THREADS, NVV ? 2 : PIPE_CTAS_PER_SM) push_kernel(PushGroups<MAXG> const __grid_constant__ G)
{
    constexpr int      SPAN        = PIPE_W - 1 - O; // largest stencil base offset inside the window
    constexpr int      PIPE_STAGES = PipeLayout<PSD>::STAGES;
    using Stage                    = PipeStageT<PSD>;
    extern __shared__ __align__(128) unsigned char smraw[];
    Stage        *stage = reinterpret_cast<Stage *>(smraw);
    uint64_t     *full  = reinterpret_cast<uint64_t *>(smraw + PipeLayout<PSD>::BAR_OFFSET);
    uint64_t     *empty = full + PIPE_STAGES;
    int const     warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    int64_t const nchunks = G.chunk0[G.n];
    int64_t const per     = (nchunks + gridDim.x - 1) / gridDim.x;
    int64_t const c0      = static_cast<int64_t>(blockIdx.x) * per;
    int64_t const mine    = c0 < nchunks ? min(per, nchunks - c0) : 0;

    if (threadIdx.x == 0) {
        for (int s = 0; s < PIPE_STAGES; ++s) {
            mbar_init(&full[s], 1);
            mbar_init(&empty[s], PIPE_CONSUMER_WARPS);
        }
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    __syncthreads();

    if (warp == PIPE_CONSUMER_WARPS) { // ---------------- producer ----------------
        if (lane == 0) {
            int gl = -1, gr = -1; // groups of the chunk being loaded / retired
            int      s  = 0; // i % PIPE_STAGES
            uint32_t ph = 0; // (i / PIPE_STAGES) & 1; both kept incrementally, without a 64-bit division per chunk
            for (int64_t i = 0; i < mine + PIPE_STAGES; ++i, s = s + 1 == PIPE_STAGES ? 0 : s + 1, ph ^= s == 0 ? 1u : 0u) {
                if (i >= PIPE_STAGES && i - PIPE_STAGES < mine) { // retire the chunk held by stage s
                    int64_t const   j = i - PIPE_STAGES;
                    gr                = group_of(G, c0 + j, gr);
                    PushArgs const &a = G.g[gr];
                    if (!mbar_wait(&empty[s], ph ^ 1u)) { // the phase of chunk j = i - PIPE_STAGES
                        atomicOr(a.status, ST_TIMEOUT);
                        break;
                    }
                    if (a.write_back) {
                        int64_t const  start = (c0 + j - G.chunk0[gr]) * PIPE_CHUNK;
                        uint32_t const cnt   = static_cast<uint32_t>(min(static_cast<int64_t>(PIPE_CHUNK), a.n - start));
                        uint32_t const b8    = round16(cnt * 8);
                        bulk_store(a.q1 + start, stage[s].q1, b8);
                        bulk_store(a.vx + start, stage[s].vx, b8);
                        bulk_store(a.vy + start, stage[s].vy, b8);
                        bulk_store(a.vz + start, stage[s].vz, b8);
                        if (BC == BCK_ABSORBING || PSD)
                            bulk_store(a.w + start, stage[s].w, b8);
                        if (PSD)
                            bulk_store(a.real_f + start, stage[s].real_f, b8);
                        bulk_commit();
                    }
                    bulk_wait_read_all();
                }
                if (i < mine) {
                    gl                   = group_of(G, c0 + i, gl);
                    PushArgs const &a    = G.g[gl];
                    bool const      lpid = a.randomize != 0;
                    int64_t const   start = (c0 + i - G.chunk0[gl]) * PIPE_CHUNK;
                    uint32_t const  cnt   = static_cast<uint32_t>(min(static_cast<int64_t>(PIPE_CHUNK), a.n - start));
                    uint32_t const  b8 = round16(cnt * 8), b4 = round16(cnt * 4);
                    mbar_arrive_expect_tx(&full[s], (PSD ? 7 : 5) * b8 + (lpid ? b4 : 0));
                    bulk_load(stage[s].q1, a.q1 + start, b8, &full[s]);
                    bulk_load(stage[s].vx, a.vx + start, b8, &full[s]);
                    bulk_load(stage[s].vy, a.vy + start, b8, &full[s]);
                    bulk_load(stage[s].vz, a.vz + start, b8, &full[s]);
                    bulk_load(stage[s].w, a.w + start, b8, &full[s]);
                    if (lpid)
                        bulk_load(stage[s].pid, a.pid + start, b4, &full[s]);
                    if (PSD) {
                        bulk_load(stage[s].real_f, a.real_f + start, b8, &full[s]);
                        bulk_load(stage[s].marker, a.marker + start, b8, &full[s]);
                    }
                }
            }
            bulk_wait_all();
        }
        return;
    }

    // ---------------- consumers ----------------
    ColWindow64 win;
    win.col  = reinterpret_cast<double2 *>(smraw + PipeLayout<PSD>::COL_OFFSET) + warp * 2 * PIPE_W * 2 * 32;
    NvvWindow64 nvw{};
    if constexpr (NVV) {
        nvw.col = reinterpret_cast<double2 *>(smraw + PipeLayout<PSD>::COL_OFFSET + PIPE_COL_BYTES) + warp * PIPE_W * 3 * 32;
        nvw.zero(lane);
    }
    win.base = ColWindow64::NONE;
    win.zero(lane);
    unsigned bad = 0;
    int      gc  = -1; // current group
    int      s  = 0; // i % PIPE_STAGES
    uint32_t ph = 0; // (i / PIPE_STAGES) & 1
    for (int64_t i = 0; i < mine; ++i, s = s + 1 == PIPE_STAGES ? 0 : s + 1, ph ^= s == 0 ? 1u : 0u) {
        int const gi = group_of(G, c0 + i, gc);
        if (gi != gc) { // entering the next group: settle the previous group's window and status
            if (gc >= 0) {
                PushArgs const &ap = G.g[gc];
                win.flush(lane, ap);
                if constexpr (NVV)
                    nvw.flush(win.base, lane, ap);
                bad = __reduce_or_sync(0xffffffffu, bad);
                if (bad && lane == 0)
                    atomicOr(ap.status, bad);
                bad = 0;
            }
            win.base = ColWindow64::NONE;
            gc       = gi;
        }
        PushArgs const &a        = G.g[gc];
        bool const      load_pid = a.randomize != 0;
        if (!mbar_wait(&full[s], ph)) {
            bad |= ST_TIMEOUT;
            break;
        }
        int64_t const start = (c0 + i - G.chunk0[gc]) * PIPE_CHUNK;
        int const     cnt   = static_cast<int>(min(static_cast<int64_t>(PIPE_CHUNK), a.n - start));
        Stage        &P     = stage[s];
        int const     w0    = warp * 32 * PIPE_PPT;

        // slots past `cnt` hold stale finite data and are processed but never deposited or stored
        // the lane's particles are pushed first, then one window check covers all their deposits
        Shape<O> ds0[PIPE_PPT], ds1[PIPE_PPT];
        d3       dv0[PIPE_PPT], dv1[PIPE_PPT];
        double   dw0[PIPE_PPT], dw1[PIPE_PPT];
        bool     dd0[PIPE_PPT], dd1[PIPE_PPT];
#pragma unroll
        for (int k = 0; k < PIPE_PPT; ++k) {
            int const    idx   = w0 + k * 32 + lane;
            bool const   live  = idx < cnt;
            double       q1    = P.q1[idx];
            d3           v     = { P.vx[idx], P.vy[idx], P.vz[idx] };
            double       w     = P.w[idx];
            double       w_in  = w;
            int32_t      pid   = load_pid ? P.pid[idx] : 0;
            bool         alive = true;
            if (a.move_steps == 2) {
                double const moved = move<MIRROR>(a, q1, v.x, 0.5 * a.dt);
                if (live && !(fabs(moved) < 1.0)) // long(moved * scale) != 0 (PartSpecies.cc:156)
                    bad |= ST_MOVED_TOO_FAR;
                alive = boundary<BC>(a, q1, v, pid, a.counter);
                if (!alive)
                    w = 0, q1 = a.full_min + 0.5, v = { 0, 0, 0 };
            }
            Shape<O> const sh0    = make_shape<O>(q1 - a.half_min);
            bool const     in0    = finite_pos(q1) && stencil_ok(sh0, a.Nx);
            d3             v_push = v;
            if (in0) {
                if (alive && a.move_steps != 0) {
                    d3 E, dB;
                    interp_EB<O>(a.EB, sh0, E, dB);
                    double   c2;
                    d3 const B = background_B<MIRROR>(a, q1, v, c2) + dB;
                    v          = boris_push(a.boris, v, B, E);
                    if constexpr (PSD) { // the weight at the new velocity and the push position
                        double rf     = P.real_f[idx];
                        w             = update_weight(a, v, q1, rf, P.marker[idx]);
                        w_in          = w;
                        P.real_f[idx] = rf;
                    }
                    // contravariant q1-velocity v_x cos^2 / D1 at the position of the push (CurviBasis.h:65-69)
                    double moved = (a.inv_D1 * c2) * v.x * (a.move_steps == 2 ? 0.5 * a.dt : a.dt);
                    q1 += moved;
                    moved *= a.travel_scale;
                    if (live && !(fabs(moved) < 1.0))
                        bad |= ST_MOVED_TOO_FAR;
                    v_push = v;
                    alive  = boundary<BC>(a, q1, v, pid, a.counter + (a.move_steps == 2 ? 1 : 0));
                    if (!alive)
                        w = 0, q1 = a.full_min + 0.5, v = { 0, 0, 0 };
                }
            } else if (live) {
                bad |= ST_OUT_OF_RANGE;
            }
            P.q1[idx]  = q1;
            P.vx[idx]  = v.x;
            P.vy[idx]  = v.y;
            P.vz[idx]  = v.z;
            if (BC == BCK_ABSORBING || PSD)
                P.w[idx] = w;

            ds0[k] = sh0;
            ds1[k] = make_shape<O>(q1 - a.half_min);
            dd0[k] = live && in0 && (a.deposit_mask & 1);
            dd1[k] = live && (a.deposit_mask & 2) && w != 0.0 && finite_pos(q1) && stencil_ok(ds1[k], a.Nx);
            dv0[k] = v_push, dw0[k] = w_in;
            dv1[k] = v, dw1[k] = w;
        }
        {
            int lo = 0x7fffffff, hi = -0x7fffffff;
#pragma unroll
            for (int k = 0; k < PIPE_PPT; ++k) {
                if (dd0[k])
                    lo = min(lo, ds0[k].i0), hi = max(hi, ds0[k].i0);
                if (dd1[k])
                    lo = min(lo, ds1[k].i0), hi = max(hi, ds1[k].i0);
            }
            bool const outside = lo <= hi && (lo < win.base || hi > win.base + SPAN);
            bool       all_in  = true; // every deposit of the lane inside the window
            if (__any_sync(0xffffffffu, outside)) { // move the window onto this batch
                win.flush(lane, a);
                if constexpr (NVV)
                    nvw.flush(win.base, lane, a);
                int const mlo = __reduce_min_sync(0xffffffffu, lo);
                int const mhi = __reduce_max_sync(0xffffffffu, hi);
                int const gap = SPAN - (mhi - mlo);
                win.base      = gap > 0 ? mlo - gap / 2 : mlo;
                all_in        = lo > hi || (lo >= win.base && hi <= win.base + SPAN);
            }
            // collect_all's w v_i v_j at the end position (PartSpecies.cc:236-239)
            auto nvv_terms = [&](int k, double (&t)[6]) {
                d3 const v = dv1[k];
                t[0] = (v.x * v.x) * dw1[k], t[1] = (v.y * v.y) * dw1[k], t[2] = (v.z * v.z) * dw1[k];
                t[3] = (v.x * v.y) * dw1[k], t[4] = (v.y * v.z) * dw1[k], t[5] = (v.z * v.x) * dw1[k];
            };
            if (all_in) { // the usual case: no check per deposit
#pragma unroll
                for (int k = 0; k < PIPE_PPT; ++k) {
                    if (dd0[k]) {
                        double const vw[4] = { dw0[k], dv0[k].x * dw0[k], dv0[k].y * dw0[k], dv0[k].z * dw0[k] };
                        win.add<O>(0, ds0[k], vw, lane);
                    }
                    if (dd1[k]) {
                        double const vw[4] = { dw1[k], dv1[k].x * dw1[k], dv1[k].y * dw1[k], dv1[k].z * dw1[k] };
                        win.add<O>(1, ds1[k], vw, lane);
                        if constexpr (NVV) {
                            double t[6];
                            nvv_terms(k, t);
                            nvw.add<O>(win.base, ds1[k], t, lane);
                        }
                    }
                }
            } else {
#pragma unroll
                for (int k = 0; k < PIPE_PPT; ++k) {
                    if (dd0[k]) {
                        double const vw[4] = { dw0[k], dv0[k].x * dw0[k], dv0[k].y * dw0[k], dv0[k].z * dw0[k] };
                        if (ds0[k].i0 >= win.base && ds0[k].i0 <= win.base + SPAN)
                            win.add<O>(0, ds0[k], vw, lane);
                        else
                            deposit_direct<O>(a, 0, ds0[k], vw);
                    }
                    if (dd1[k]) {
                        double const vw[4] = { dw1[k], dv1[k].x * dw1[k], dv1[k].y * dw1[k], dv1[k].z * dw1[k] };
                        bool const   inside = ds1[k].i0 >= win.base && ds1[k].i0 <= win.base + SPAN;
                        if (inside)
                            win.add<O>(1, ds1[k], vw, lane);
                        else
                            deposit_direct<O>(a, 1, ds1[k], vw);
                        if constexpr (NVV) {
                            double t[6];
                            nvv_terms(k, t);
                            if (inside)
                                nvw.add<O>(win.base, ds1[k], t, lane);
                            else
                                nvv_direct<O>(a, ds1[k], t);
                        }
                    }
                }
            }
        }
        fence_proxy_async_smem();
        __syncwarp();
        if (lane == 0)
            mbar_arrive(&empty[s]);
    }
    if (gc >= 0) {
        PushArgs const &a = G.g[gc];
        win.flush(lane, a);
        if constexpr (NVV)
            nvw.flush(win.base, lane, a);
        bad = __reduce_or_sync(0xffffffffu, bad);
        if (bad && lane == 0)
            atomicOr(a.status, bad);
    }
}

} // namespace h1d
