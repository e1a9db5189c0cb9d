// Device-side building blocks of the hybrid_1d hot path for sm_100a.
//
// Shape functions, Boris push and the mirror-field geometry follow
//   Shape<1..3>            src/LibPIC/PIC/Shape.h:29-35, 77-99, 149-176
//   BorisPush              src/LibPIC/PIC/BorisPush.h:25-30, 57-73, 99-102
//   CurviBasis / MFABasis  src/LibPIC/PIC/Geometry/CurviBasis.h:40-69, MFABasis.h:37-80
//   MirrorGeometry         src/LibPIC/PIC/Geometry/MirrorGeometry.cc:34-47
// of kyungguk1/hybrid_code-hfemic_wave.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

namespace h1d {

constexpr int PAD = 3;
// floats per cell of the FP32 push record {Ex, Ey, Ez, dBx, dBy, dBz, 0, 0}: two 16-byte loads per node
constexpr int EBF_STRIDE = 8;

// device status word bits; read by the host after each advance
enum : unsigned {
    ST_MOVED_TOO_FAR = 1u << 0, // |dq1| >= allowed fraction of a cell (PartSpecies.cc:147-159)
    ST_OUT_OF_RANGE  = 1u << 1, // a particle's stencil fell outside the padded grid (non-finite or lost particle)
    ST_NAN           = 1u << 2,
    ST_SORT_OVERFLOW = 1u << 3,
    ST_TIMEOUT       = 1u << 4, // a bounded wait on a pipeline barrier gave up
};

struct d3 {
    double x, y, z;
};
__device__ __forceinline__ d3 make_d3(double x, double y, double z) { return d3{ x, y, z }; }
__device__ __forceinline__ d3 operator+(d3 a, d3 b) { return { a.x + b.x, a.y + b.y, a.z + b.z }; }
__device__ __forceinline__ d3 operator-(d3 a, d3 b) { return { a.x - b.x, a.y - b.y, a.z - b.z }; }
__device__ __forceinline__ d3 operator*(d3 a, double s) { return { a.x * s, a.y * s, a.z * s }; }
__device__ __forceinline__ d3 cross(d3 A, d3 B)
{
    return { A.y * B.z - A.z * B.y, A.z * B.x - A.x * B.z, A.x * B.y - A.y * B.x };
}
__device__ __forceinline__ d3 ld3(double const *g, long i) { return { g[3 * i], g[3 * i + 1], g[3 * i + 2] }; }
__device__ __forceinline__ void st3(double *g, long i, d3 v) { g[3 * i] = v.x, g[3 * i + 1] = v.y, g[3 * i + 2] = v.z; }

// Exact floor / round-half-away-from-zero / ceil of |x| < 2^30 with their integer value, on the
// FP64 pipe instead of the conversion unit: t = x + 1.5*2^52 holds x rounded to the nearest
// integer (ties to even) in its low mantissa word, and t - 1.5*2^52 is that integer as a double;
// one comparison then corrects the rounding direction.
struct IntReal {
    int    i;
    double d;
};
__device__ __forceinline__ IntReal rint_magic(double x)
{
    double const M = 6755399441055744.0;
    double const t = __dadd_rn(x, M);
    return { __double2loint(t), __dsub_rn(t, M) };
}
__device__ __forceinline__ IntReal floor_ir(double x)
{
    IntReal r = rint_magic(x);
    if (r.d > x)
        r.i -= 1, r.d -= 1.0;
    return r;
}
__device__ __forceinline__ IntReal ceil_ir(double x)
{
    IntReal r = rint_magic(x);
    if (r.d < x)
        r.i += 1, r.d += 1.0;
    return r;
}
__device__ __forceinline__ IntReal round_ir(double x) // std::round: halves away from zero
{
    IntReal      r = rint_magic(x);
    double const f = x - r.d; // exact
    if (f == 0.5 && x > 0)
        r.i += 1, r.d += 1.0;
    else if (f == -0.5 && x < 0)
        r.i -= 1, r.d -= 1.0;
    return r;
}

// sin and cos of |x| <= pi/2 from their Taylor series through x^23 and x^24 (truncation error
// below 1e-20), Horner in x^2; no range reduction is needed because |xi D1 q1| < pi/2 holds on the
// whole domain (ParamSet.cc:25-29)
__device__ __forceinline__ void sincos_taylor(double x, double &s, double &c)
{
    double const x2 = x * x;
    double       ps = -3.868170170630684e-23;
    ps              = fma(ps, x2, 1.9572941063391263e-20);
    ps              = fma(ps, x2, -8.22063524662433e-18);
    ps              = fma(ps, x2, 2.8114572543455206e-15);
    ps              = fma(ps, x2, -7.647163731819816e-13);
    ps              = fma(ps, x2, 1.6059043836821613e-10);
    ps              = fma(ps, x2, -2.505210838544172e-08);
    ps              = fma(ps, x2, 2.7557319223985893e-06);
    ps              = fma(ps, x2, -0.0001984126984126984);
    ps              = fma(ps, x2, 0.008333333333333333);
    ps              = fma(ps, x2, -0.16666666666666666);
    s               = fma(ps * x2, x, x);
    double pc       = 1.6117375710961184e-24;
    pc              = fma(pc, x2, -8.896791392450574e-22);
    pc              = fma(pc, x2, 4.110317623312165e-19);
    pc              = fma(pc, x2, -1.5619206968586225e-16);
    pc              = fma(pc, x2, 4.779477332387385e-14);
    pc              = fma(pc, x2, -1.1470745597729725e-11);
    pc              = fma(pc, x2, 2.08767569878681e-09);
    pc              = fma(pc, x2, -2.755731922398589e-07);
    pc              = fma(pc, x2, 2.48015873015873e-05);
    pc              = fma(pc, x2, -0.001388888888888889);
    pc              = fma(pc, x2, 0.041666666666666664);
    pc              = fma(pc, x2, -0.5);
    c               = fma(pc, x2, 1.0);
}

// Shape<Order>: base index i0 and weights w[0..Order]
template <int O>
struct Shape {
    int    i0;
    double w[O + 1];
};
template <int O>
__device__ __forceinline__ Shape<O> make_shape(double x)
{
    Shape<O> s;
    if constexpr (O == 1) {
        IntReal const f = floor_ir(x);
        s.i0            = f.i;
        s.w[1]          = x - f.d;
        s.w[0]          = 1 - s.w[1];
    } else if constexpr (O == 2) {
        IntReal const r = round_ir(x);
        s.i0            = r.i - 1;
        double t        = r.d - x;
        s.w[1]          = 0.75 - t * t;
        t += 0.5;
        s.w[0] = 0.5 * (t * t);
        s.w[2] = 1 - (s.w[0] + s.w[1]);
    } else {
        IntReal const c = ceil_ir(x);
        s.i0            = c.i - 2;
        double const i0 = c.d - 2;
        double       t  = 2 + (i0 - x);
        s.w[0]          = (1. / 6) * (t * t * t);
        t               = 2 - ((i0 + 3) - x);
        s.w[3]          = (1. / 6) * (t * t * t);
        t               = x - (i0 + 1);
        s.w[1]          = (1. / 6) * (4 + 3 * t * t * (t - 2));
        s.w[2]          = 1 - (s.w[0] + s.w[1] + s.w[3]);
    }
    return s;
}
// positions further than this from the grid are lost particles (NaN and Inf included)
__device__ __forceinline__ bool finite_pos(double x) { return x > -1073741824.0 && x < 1073741824.0; }

// Boris push constants (BorisPush.h:25-30)
struct BorisK {
    double dtOc_2O0, cDtOc_2O0;
};
__host__ __device__ inline BorisK boris_make(double dt, double c, double O0, double Oc)
{
    double const dt_2 = 0.5 * dt;
    BorisK       k;
    k.dtOc_2O0  = Oc * dt_2 / O0;
    k.cDtOc_2O0 = c * k.dtOc_2O0;
    return k;
}
__device__ __forceinline__ d3 boris_push(BorisK const &k, d3 v, d3 B, d3 E)
{
    B          = B * k.dtOc_2O0;
    E          = E * k.cDtOc_2O0;
    v          = v + E;
    d3 const u = v + cross(v, B);
    // 2 / d as twice the correctly rounded reciprocal: scaling by two is exact, so the result is
    // the same rounded quotient, with a shorter dependent chain than a division (d >= 1)
    double const s = 2 * __drcp_rn(1 + (B.x * B.x + B.y * B.y + B.z * B.z));
    v              = v + cross(u, B * s);
    return v + E;
}

// 64-bit warp all-reduce (butterfly)
__device__ __forceinline__ double warp_sum(double v)
{
#pragma unroll
    for (int o = 16; o > 0; o >>= 1)
        v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

// counter-based draw in [-pi, pi) for the gyro-phase of reflected particles; replaces the
// std::random_device-seeded generator of Delegate::randomize_gyrophase (Delegate.cc:146-156)
__host__ __device__ inline uint64_t mix64(uint64_t z)
{
    z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ULL;
    z = (z ^ (z >> 27)) * 0x94d049bb133111ebULL;
    return z ^ (z >> 31);
}
// sin and cos of an angle in [-pi, pi) (a gyrophase): one half-turn brought onto |x| <= pi/2 for
// sincos_taylor, so the particle pass carries no general range reduction
__device__ __forceinline__ void sincos_half_turn(double x, double &s, double &c)
{
    constexpr double PI   = 3.141592653589793;
    bool const       flip = fabs(x) > 0.5 * PI;
    sincos_taylor(flip ? x - copysign(PI, x) : x, s, c);
    if (flip)
        s = -s, c = -c;
}

__host__ __device__ inline double gyrophase(uint64_t seed, uint64_t counter, uint64_t species, uint64_t pid)
{
    uint64_t h = mix64(seed + 0x9e3779b97f4a7c15ULL);
    h          = mix64(h ^ (counter * 0xd1b54a32d192ed03ULL));
    h          = mix64(h ^ (species * 0x8cb92ba72f3d8dd7ULL) ^ pid);
    double const u = static_cast<double>(h >> 11) * (1.0 / 9007199254740992.0);
    return -3.14159265358979323846 + u * (2 * 3.14159265358979323846);
}

} // namespace h1d
