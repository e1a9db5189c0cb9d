// Device-side building blocks of the hybrid_1d hot path for sm_100a.
//
// Shape functions, Boris push and the mirror-field geometry follow
//   Shape<1..3>            src/LibPIC/PIC/Shape.h:29-35, 77-99, 149-176
//   BorisPush              src/LibPIC/PIC/BorisPush.h:25-30, 57-73, 99-102
//   CurviBasis / MFABasis  src/LibPIC/PIC/Geometry/CurviBasis.h:40-69, MFABasis.h:252-290
//   MirrorGeometry         src/LibPIC/PIC/Geometry/MirrorGeometry.cc:199-212
// of kyungguk1/hybrid_code-hfemic_wave.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

namespace h1d {

constexpr int PAD = 3;

// device status word bits; read by the host after each advance
enum : unsigned {
    ST_MOVED_TOO_FAR = 1u << 0, // |dq1| >= allowed fraction of a cell (PartSpecies.cc:252-264)
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
        double const f = floor(x);
        s.i0           = static_cast<int>(f);
        s.w[1]         = x - f;
        s.w[0]         = 1 - s.w[1];
    } else if constexpr (O == 2) {
        double const r = round(x); // half away from zero, as std::round
        s.i0           = static_cast<int>(r) - 1;
        double t       = r - x;
        s.w[1]         = 0.75 - t * t;
        t += 0.5;
        s.w[0] = 0.5 * (t * t);
        s.w[2] = 1 - (s.w[0] + s.w[1]);
    } else {
        double const c = ceil(x);
        s.i0           = static_cast<int>(c) - 2;
        double const i0 = c - 2;
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
    double const s = 2 / (1 + (B.x * B.x + B.y * B.y + B.z * B.z));
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
// std::random_device-seeded generator of Delegate::randomize_gyrophase (Delegate.cc:229-239)
__host__ __device__ inline uint64_t mix64(uint64_t z)
{
    z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ULL;
    z = (z ^ (z >> 27)) * 0x94d049bb133111ebULL;
    return z ^ (z >> 31);
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
