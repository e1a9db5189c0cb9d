// Particle kernels outside the particle pass: collect_all of n, nV and nvv for the recorders
// (PartSpecies::impl_collect_all, PartSpecies.cc:225-244) in both precisions, the FP64 <->
// mixed-precision conversions of upload and download, and the cell keys and gather of the
// mixed-precision cell sort.  Compiled in the library's main translation unit only.
#pragma once

#include "particles_mixed.cuh"

namespace h1d {

// PartSpecies::impl_collect_all (PartSpecies.cc:225-244): n, nV and nvv with CIC, unscaled, from
// cell-sorted particles (moments_kernel below).

struct MomentArgs {
    double const  *q1, *vx, *vy, *vz, *w;
    int64_t        n;
    int            ppt, Nx;
    int            vec; // every array 16-byte aligned: vector loads
    double         half_min;
    double        *out[10]; // n, nVx, nVy, nVz, xx, yy, zz, xy, yz, zx at cell 0
    unsigned      *status;
};
struct MomentArgsMixed {
    int32_t const *pos; // fixed-point positions (pos_cell, pos_off)
    float const   *vx, *vy, *vz, *w;
    int64_t        n;
    int            ppt, Nx, fbits;
    float          inv_scale;
    int            vec; // every array 16-byte aligned: vector loads
    double        *out[10];
    unsigned      *status;
};

// the arithmetic of a lane's collect_all sums: FP64 for FP64 particles; FP32 for mixed-precision
// particles (a lane sums at most 16 FP32 particles per cell; warp sums and atomics are FP64)
template <class Args> struct MomReal {
    using type = double;
};
template <> struct MomReal<MomentArgsMixed> {
    using type = float;
};
// one particle as the collect_all loop needs it: CIC stencil, weight and velocity
template <class R> struct MomParticle {
    int  i0;
    R    s0, s1, w, vx, vy, vz;
    bool ok;
};
// NP consecutive particles of a lane, loaded with 16-byte vector loads (NP = 4 FP32 / 2 FP64)
template <class Args> struct MomTile;
template <> struct MomTile<MomentArgs> {
    static constexpr int NP = 2;
    double2              q1, vx, vy, vz, w;
};
template <> struct MomTile<MomentArgsMixed> {
    static constexpr int NP = 4;
    int4                 pos;
    float4               vx, vy, vz, w;
};
__device__ __forceinline__ double el2(double2 const &v, int j) { return j ? v.y : v.x; }
__device__ __forceinline__ float  el4(float4 const &v, int j) { return j == 0 ? v.x : j == 1 ? v.y : j == 2 ? v.z : v.w; }
__device__ __forceinline__ int    el4(int4 const &v, int j) { return j == 0 ? v.x : j == 1 ? v.y : j == 2 ? v.z : v.w; }

// the tile at particle i (a multiple of NP); past the end it repeats the last particle (never used)
__device__ __forceinline__ MomTile<MomentArgs> mom_load(MomentArgs const &a, int64_t i)
{
    MomTile<MomentArgs> t;
    if (a.vec && i + 1 < a.n) {
        t.q1 = *reinterpret_cast<double2 const *>(a.q1 + i), t.vx = *reinterpret_cast<double2 const *>(a.vx + i);
        t.vy = *reinterpret_cast<double2 const *>(a.vy + i), t.vz = *reinterpret_cast<double2 const *>(a.vz + i);
        t.w  = *reinterpret_cast<double2 const *>(a.w + i);
    } else {
        int64_t const j0 = min(i, a.n - 1), j1 = min(i + 1, a.n - 1);
        t.q1 = make_double2(a.q1[j0], a.q1[j1]), t.vx = make_double2(a.vx[j0], a.vx[j1]);
        t.vy = make_double2(a.vy[j0], a.vy[j1]), t.vz = make_double2(a.vz[j0], a.vz[j1]);
        t.w  = make_double2(a.w[j0], a.w[j1]);
    }
    return t;
}
__device__ __forceinline__ MomTile<MomentArgsMixed> mom_load(MomentArgsMixed const &a, int64_t i)
{
    MomTile<MomentArgsMixed> t;
    if (a.vec && i + 3 < a.n) {
        t.pos  = *reinterpret_cast<int4 const *>(a.pos + i);
        t.vx   = *reinterpret_cast<float4 const *>(a.vx + i), t.vy = *reinterpret_cast<float4 const *>(a.vy + i);
        t.vz   = *reinterpret_cast<float4 const *>(a.vz + i), t.w = *reinterpret_cast<float4 const *>(a.w + i);
    } else {
        int64_t const j[4] = { min(i, a.n - 1), min(i + 1, a.n - 1), min(i + 2, a.n - 1), min(i + 3, a.n - 1) };
        t.pos  = make_int4(a.pos[j[0]], a.pos[j[1]], a.pos[j[2]], a.pos[j[3]]);
        t.vx   = make_float4(a.vx[j[0]], a.vx[j[1]], a.vx[j[2]], a.vx[j[3]]);
        t.vy   = make_float4(a.vy[j[0]], a.vy[j[1]], a.vy[j[2]], a.vy[j[3]]);
        t.vz   = make_float4(a.vz[j[0]], a.vz[j[1]], a.vz[j[2]], a.vz[j[3]]);
        t.w    = make_float4(a.w[j[0]], a.w[j[1]], a.w[j[2]], a.w[j[3]]);
    }
    return t;
}
__device__ __forceinline__ MomParticle<double> mom_particle(MomentArgs const &a, MomTile<MomentArgs> const &t, int j)
{
    double const   q1 = el2(t.q1, j);
    Shape<1> const sh = make_shape<1>(q1 - a.half_min);
    return { sh.i0, sh.w[0], sh.w[1], el2(t.w, j), el2(t.vx, j), el2(t.vy, j), el2(t.vz, j),
             finite_pos(q1) && stencil_ok(sh, a.Nx) };
}
__device__ __forceinline__ MomParticle<float> mom_particle(MomentArgsMixed const &a, MomTile<MomentArgsMixed> const &t, int j)
{
    int32_t const   X  = el4(t.pos, j);
    ShapeF<1> const sh = make_shape_f<1>(pos_cell(X, a.fbits), pos_off(X, a.fbits, a.inv_scale));
    return { sh.i0, sh.w[0], sh.w[1], el4(t.w, j), el4(t.vx, j), el4(t.vy, j), el4(t.vz, j), stencil_ok_f(sh, a.Nx) };
}

constexpr int MOM_THREADS = 128;
// resident blocks per SM: FP32 lane sums fit five blocks in 96 registers without spills (0.235 ->
// about 0.165 ms per collect_all of 16.4M particles, against three blocks of FP64 sums); six
// spill and are slower
constexpr int MOM_MIN_BLOCKS_MIXED = 5;
// particles per lane of a collect_all warp: a multiple of 4 (whole rounds of either tile) from 4
// to 16, growing with the particles per cell
inline int mom_ppt(double ppc)
{
    int const k = static_cast<int>(ppc / 128);
    return k < 4 ? 4 : k > 16 ? 16 : k & ~3;
}

// collect_all by cells.  A lane takes ppt consecutive (cell-sorted) particles and sums, per
// quantity, the total T of its particles in one cell c, the part L that CIC gives the left
// neighbour c - 1 and the part R it gives the right neighbour c + 1; cell c receives T - L - R.
// The sums go to the moments when the lane reaches another cell (rare: a lane's particles are
// consecutive in cell order) and once at the end, one warp sum per distinct cell among the lanes.
__device__ __forceinline__ void mom_add(double *const (&out)[10], int q, int cell, int Nx, double v, unsigned &bad)
{
    if (v == 0.0)
        return;
    if (cell >= -PAD && cell < Nx + PAD)
        atomicAdd(out[q] + cell, v);
    else
        bad |= ST_OUT_OF_RANGE;
}

// resident blocks of MOM_THREADS per SM the register budget is set for
template <class Args> constexpr int mom_min_blocks = 4;
template <> constexpr int mom_min_blocks<MomentArgsMixed> = MOM_MIN_BLOCKS_MIXED;

template <class Args>
__global__ void __launch_bounds__(MOM_THREADS, mom_min_blocks<Args>) moments_kernel(Args a)
{
    constexpr int NP   = MomTile<Args>::NP;
    constexpr int NONE = 0x40000000;
    int const     lane   = threadIdx.x & 31;
    int64_t const warp   = (static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x) >> 5;
    int64_t const chunk0 = warp * 32 * a.ppt;
    if (chunk0 >= a.n)
        return;
    int64_t const first = chunk0 + static_cast<int64_t>(lane) * a.ppt; // this lane's particles
    using Real          = typename MomReal<Args>::type;
    Real          T[10], L[10], R[10];
#pragma unroll
    for (int q = 0; q < 10; ++q)
        T[q] = L[q] = R[q] = 0;
    int      rc  = NONE; // the cell T, L and R belong to
    unsigned bad = 0;
    auto     cur = mom_load(a, first);
    for (int k = 0; k < a.ppt / NP; ++k) {
        int64_t const i0  = first + NP * k;
        auto const    nxt = mom_load(a, i0 + NP); // next particles in flight
#pragma unroll
        for (int j = 0; j < NP; ++j) {
            if (i0 + j >= a.n)
                break;
            auto const p = mom_particle(a, cur, j);
            if (!p.ok) {
                bad |= ST_OUT_OF_RANGE;
                continue;
            }
            bool const up = p.s1 >= Real(0.5); // the particle's cell is i0 + 1, its left neighbour gets s0
            int const  c  = p.i0 + (up ? 1 : 0);
            if (c != rc) {
                if (rc != NONE) {
#pragma unroll
                    for (int q = 0; q < 10; ++q) {
                        double const t = T[q], l = L[q], r = R[q];
                        mom_add(a.out, q, rc, a.Nx, t - l - r, bad);
                        mom_add(a.out, q, rc - 1, a.Nx, l, bad);
                        mom_add(a.out, q, rc + 1, a.Nx, r, bad);
                        T[q] = L[q] = R[q] = 0;
                    }
                }
                rc = c;
            }
            Real const left = up ? p.s0 : Real(0), right = up ? Real(0) : p.s1;
            Real const v[10] = { p.w,               p.vx * p.w,        p.vy * p.w,        p.vz * p.w,
                                   (p.vx * p.vx) * p.w, (p.vy * p.vy) * p.w, (p.vz * p.vz) * p.w, (p.vx * p.vy) * p.w,
                                   (p.vy * p.vz) * p.w, (p.vz * p.vx) * p.w };
#pragma unroll
            for (int q = 0; q < 10; ++q) {
                T[q] += v[q];
                L[q] = fma(v[q], left, L[q]);
                R[q] = fma(v[q], right, R[q]);
            }
        }
        cur = nxt;
    }
    // one warp sum per distinct cell among the lanes; lane 3q + m adds quantity q's share m
    for (unsigned pending = __ballot_sync(0xffffffffu, rc != NONE); pending;) {
        int const  key  = __shfl_sync(0xffffffffu, rc, __ffs(pending) - 1);
        bool const mine = rc == key;
#pragma unroll
        for (int q = 0; q < 10; ++q) {
            double const t = warp_sum(mine ? static_cast<double>(T[q]) : 0.0);
            double const l = warp_sum(mine ? static_cast<double>(L[q]) : 0.0);
            double const r = warp_sum(mine ? static_cast<double>(R[q]) : 0.0);
            if (lane == 3 * q)
                mom_add(a.out, q, key, a.Nx, t - l - r, bad);
            else if (lane == 3 * q + 1)
                mom_add(a.out, q, key - 1, a.Nx, l, bad);
            else if (lane == 3 * q + 2)
                mom_add(a.out, q, key + 1, a.Nx, r, bad);
        }
        pending &= ~__ballot_sync(0xffffffffu, mine);
    }
    bad = __reduce_or_sync(0xffffffffu, bad);
    if (bad && lane == 0)
        atomicOr(a.status, bad);
}

// FP64 host-layout particles <-> mixed-precision particles (upload and download), one component at
// a time so that the FP64 staging buffer holds a single array: position q1 <-> the fixed-point
// X = round((q1 - q1min) 2^F), and velocity / weight components FP64 <-> FP32.  The grid is
// [0, len) with len = Nx 2^F; a position q1 <= q1max that rounds up to len (within half a step of
// q1max, one ulp below it where q1 - q1min itself rounds to Nx, or q1max itself, where a wrap or
// reflection of the boundary pass can round) becomes the last position len - 1, inside the grid.
__device__ __forceinline__ int32_t q1_to_pos(double q1, double full_min, double scale, int32_t len)
{
    double const y  = (q1 - full_min) * scale;
    bool const   ok = y > -1073741824.0 && y < 2147483520.0; // NaN and lost positions map outside the grid
    if (!ok)
        return -0x40000000;
    int32_t const X      = static_cast<int32_t>(__double2ll_rn(y));
    bool const    inside = q1 <= full_min + static_cast<double>(len) / scale; // q1 <= q1max, exactly
    return X >= len && inside ? len - 1 : X;
}
__global__ void q1_to_pos_kernel(double const *q1, int64_t n, double full_min, double scale, int32_t len, int32_t *pos)
{
    int64_t const i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i < n)
        pos[i] = q1_to_pos(q1[i], full_min, scale, len);
}
__global__ void to_f32_kernel(double const *src, int64_t n, float *dst)
{
    int64_t const i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i < n)
        dst[i] = static_cast<float>(src[i]);
}
// one component at a time, so that the caller's FP64 staging buffer holds a single array: the
// position (exact in FP64) from `pos`, or an FP32 component from `src`
__global__ void from_mixed_kernel(int32_t const *pos, float const *src, int64_t n, double full_min, double inv_scale,
                                  double *dst)
{
    int64_t const i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i >= n)
        return;
    dst[i] = pos ? full_min + static_cast<double>(pos[i]) * inv_scale : static_cast<double>(src[i]);
}

// ------------------------------------------------------------------------------------------------
// Device loader of a bi-Maxwellian species (PartSpecies::populate with MaxwellianVDF::load,
// VDF/MaxwellianVDF.cc:115-134, q1_of_N :55-65, eta :33-43).  Particle i uses the radical
// inverses in bases 2, 3 and 5 of the sequence index offset + i and two counter-based uniforms (the
// splitmix64 finalizer of the species key and 2i + 1, 2i + 2).  Every arithmetic step is the one
// the host loader (loader.py) performs, in the same order and without contraction, so the two
// agree up to the device's tan/atan/cos/log/sin.
// ------------------------------------------------------------------------------------------------
constexpr uint64_t POP_GOLDEN = 0x9E3779B97F4A7C15ULL;

inline uint64_t populate_key(uint64_t seed, uint64_t s)
{
    return mix64(mix64(seed ^ 0x243F6A8885A308D3ULL) + s * POP_GOLDEN);
}
inline uint64_t populate_offset(uint64_t key) { return 1 + (mix64(key ^ 0x13198A2E03707344ULL) >> 24); }

struct PopulateArgs {
    int64_t  n;
    uint64_t key, offset;
    double   N_loc, N_len, xiD1, T2m1, sqrtT2, sDxXi, T2, oneMinusT2, vth1, q1min, q1max_in, full_min;
    int      homogeneous;
    double  *q1, *vx, *vy, *vz, *w;                 // FP64 storage, or
    int32_t *pos;                                    // mixed-precision storage
    float   *fvx, *fvy, *fvz, *fw;
    double   scale;                                  // 2^F of the fixed-point positions
    int32_t  len;                                    // Nx 2^F, the end of the fixed-point grid
};

__device__ __forceinline__ double radical_inverse_dev(uint64_t k, unsigned base)
{
    if (base == 2)
        return __dmul_rn(static_cast<double>(__brevll(k) >> 11), 0x1p-53);
    double       out = 0, f = __ddiv_rn(1.0, static_cast<double>(base));
    double const b   = static_cast<double>(base);
    while (k) {
        out = __dadd_rn(out, __dmul_rn(static_cast<double>(k % base), f));
        k /= base;
        f = __ddiv_rn(f, b);
    }
    return out;
}

__device__ __forceinline__ double pop_uniform(uint64_t key, uint64_t i, uint64_t j)
{
    double const eps = 1e-15;
    double const u   = __dmul_rn(static_cast<double>(mix64(key + (i * 2 + j) * POP_GOLDEN) >> 11), 0x1p-53);
    return __dadd_rn(eps, __dmul_rn(1 - 2 * eps, u));
}

__global__ void populate_kernel(PopulateArgs a)
{
    int64_t const i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i >= a.n)
        return;
    double const   eps = 1e-15, one_m = 1 - 2 * eps, two_pi = 2 * 3.141592653589793;
    uint64_t const idx = a.offset + static_cast<uint64_t>(i);
    double const   u2  = __dadd_rn(eps, __dmul_rn(one_m, radical_inverse_dev(idx, 2)));
    double const   u3  = __dadd_rn(eps, __dmul_rn(one_m, radical_inverse_dev(idx, 3)));
    double const   u5  = __dadd_rn(eps, __dmul_rn(one_m, radical_inverse_dev(idx, 5)));
    double const   N   = __dadd_rn(__dmul_rn(u2, a.N_len), a.N_loc);
    double         q1;
    if (a.homogeneous) {
        double const x = __dmul_rn(a.xiD1, N);
        double       t = __dmul_rn(__dmul_rn(x, x), a.T2m1);
        t              = __dadd_rn(1.0, __ddiv_rn(t, 3.0));
        q1             = __dmul_rn(N, t);
    } else {
        q1 = __ddiv_rn(atan(__ddiv_rn(tan(__dmul_rn(a.sDxXi, N)), a.sqrtT2)), a.xiD1);
    }
    q1                  = fmin(fmax(q1, a.q1min), a.q1max_in);
    double const U1     = pop_uniform(a.key, static_cast<uint64_t>(i), 1);
    double const U2     = pop_uniform(a.key, static_cast<uint64_t>(i), 2);
    double const c      = cos(__dmul_rn(a.xiD1, q1));
    double const eta    = __ddiv_rn(1.0, __dadd_rn(a.T2, __dmul_rn(__dmul_rn(a.oneMinusT2, c), c)));
    double const T2OT1  = __dmul_rn(a.T2, eta);
    double const x1     = __dmul_rn(sqrt(-log(U1)), sin(__dmul_rn(two_pi, u3)));
    double const tmp    = sqrt(__dmul_rn(-log(U2), T2OT1));
    double const x2     = __dmul_rn(cos(__dmul_rn(two_pi, u5)), tmp);
    double const x3     = __dmul_rn(sin(__dmul_rn(two_pi, u5)), tmp);
    double const vx = __dmul_rn(x1, a.vth1), vy = __dmul_rn(x2, a.vth1), vz = __dmul_rn(x3, a.vth1);
    if (a.q1) {
        a.q1[i] = q1, a.vx[i] = vx, a.vy[i] = vy, a.vz[i] = vz, a.w[i] = 1.0;
    } else {
        a.pos[i] = q1_to_pos(q1, a.full_min, a.scale, a.len);
        a.fvx[i] = static_cast<float>(vx), a.fvy[i] = static_cast<float>(vy), a.fvz[i] = static_cast<float>(vz);
        a.fw[i] = 1.0f;
    }
}


// ------------------------------------------------------------------------------------------------
// VHistogramRecorder::local_counting (Recorder/VHistogramRecorder.cc:289-306): gyro-averaged
// velocity histogram of the particles in [ext_lo, ext_hi), relative to the bulk velocity nV/n of
// the recorded moments at the particle (Shape<1>), binned as the recorder's Indexer does
// (:88-100).  Rounded operations (no contraction) so that the bins equal the host's.  Per bin:
// marker count, weight sum, real_f / marker sum (1 per full-f particle); the host normalises.
// ------------------------------------------------------------------------------------------------
struct VHistArgs {
    double const  *q1, *vx, *vy, *vz, *w;        // FP64 storage (+ real_f, marker when the weights evolve), or
    double const  *real_f, *marker;
    int32_t const *pos;                          // mixed-precision storage
    float const   *fvx, *fvy, *fvz, *fw, *freal_f, *fmarker;
    double         inv_scale;                    // 2^-F of the fixed-point positions
    int64_t        n;
    double         half_min, full_min, ext_lo, ext_hi, v1min, v1len, v2min, v2len;
    int            v1dim, v2dim;
    double const  *mom; // finalized moments: n (M), nV (3M), GridArray layout
    long           M;
    double        *out; // 3 x v1dim x v2dim
    unsigned long long *count;
};

__global__ void vhist_kernel(VHistArgs a)
{
    int64_t const k = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (k >= a.n)
        return;
    double q1, vx, vy, vz, w;
    if (a.q1) {
        q1 = a.q1[k], vx = a.vx[k], vy = a.vy[k], vz = a.vz[k], w = a.w[k];
    } else {
        q1 = a.full_min + static_cast<double>(a.pos[k]) * a.inv_scale;
        vx = a.fvx[k], vy = a.fvy[k], vz = a.fvz[k], w = a.fw[k];
    }
    if (!(q1 >= a.ext_lo && q1 < a.ext_hi))
        return;
    atomicAdd(a.count, 1ull);
    Shape<1> const sh = make_shape<1>(q1 - a.half_min);
    if (sh.i0 < -PAD || sh.i0 + 1 >= a.M - PAD)
        return;
    double n = 0, V[3] = { 0, 0, 0 };
#pragma unroll
    for (int j = 0; j <= 1; ++j) {
        long const i = sh.i0 + j + PAD;
        n            = __dadd_rn(n, __dmul_rn(a.mom[i], sh.w[j]));
#pragma unroll
        for (int c = 0; c < 3; ++c)
            V[c] = __dadd_rn(V[c], __dmul_rn(a.mom[a.M + 3 * i + c], sh.w[j]));
    }
#pragma unroll
    for (int c = 0; c < 3; ++c)
        V[c] = n < 1e-15 ? 0.0 : __ddiv_rn(V[c], n);
    double const v1 = vx - V[0], py = vy - V[1], pz = vz - V[2];
    double const v2 = __dsqrt_rn(__dadd_rn(__dmul_rn(py, py), __dmul_rn(pz, pz)));
    double const f1 = floor(__ddiv_rn(__dmul_rn(v1 - a.v1min, static_cast<double>(a.v1dim)), a.v1len));
    double const f2 = floor(__ddiv_rn(__dmul_rn(v2 - a.v2min, static_cast<double>(a.v2dim)), a.v2len));
    if (f1 >= 0 && f1 < a.v1dim && f2 >= 0 && f2 < a.v2dim) {
        double *o = a.out + 3 * (static_cast<int64_t>(f1) * a.v2dim + static_cast<int64_t>(f2));
        atomicAdd(o, 1.0);
        atomicAdd(o + 1, w);
        // real_f / marker; without evolving weights real_f = w and marker = 1 (the upload convention)
        double const rm = a.real_f  ? __ddiv_rn(a.real_f[k], a.marker[k])
                          : a.freal_f ? static_cast<double>(a.freal_f[k]) / static_cast<double>(a.fmarker[k])
                                      : w;
        atomicAdd(o + 2, rm);
    }
}

} // namespace h1d
