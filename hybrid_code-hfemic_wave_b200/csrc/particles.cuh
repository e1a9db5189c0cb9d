// Particle kernels of the hybrid_1d hot path (FP64).
//
// One fused pass per species and CAM-CL step does what the reference does in four loops over
// the particle deque (src/hybrid_1d/Core/Domain_CAMCL.cc:69-82):
//   PartSpecies::update_vel   interp of E and dB at x^N, mirror-field B, Boris push   (PartSpecies.cc:266-281)
//   PartSpecies::collect_part deposit of n and nV at x^N with v^{N+1/2}                (PartSpecies.cc:315-329)
//   PartSpecies::update_pos   x^{N+1} = x^N + v.e^1 dt, travel check                   (PartSpecies.cc:252-264)
//   Delegate::boundary_pass   periodic wrap / reflection (+ gyro-phase)               (Delegate.cc:116-228)
//   PartSpecies::collect_part deposit of n and nV at x^{N+1}                          (PartSpecies.cc:315-329)
// Particles are structure-of-arrays and cell-sorted (sort.cuh), so the 32 x ppt particles of a
// warp span a couple of cells.  Each lane accumulates its deposits in registers over a small
// warp-uniform window of cells; the window is reduced across the warp once per warp-chunk and
// added to the global moment arrays with one atomic per (cell, quantity).  Particles that fall
// outside the window (rare: drift since the last sort, periodic wrap) add their stencil with
// direct atomics.  Moments are accumulated unscaled; the 1/Nc factor of collect_part is applied
// by the field kernel.
#pragma once

#include "device_common.cuh"

namespace h1d {

enum { BCK_PERIODIC = 0, BCK_REFLECTING = 1, BCK_ABSORBING = 2 };

struct PushArgs {
    double        *q1, *vx, *vy, *vz;
    double        *w; // writable only for absorption (w = 0 marks a removed particle)
    int32_t const *pid;
    int64_t        n;
    int            ppt; // particles per lane per warp-chunk
    int            Nx;
    double const  *E;  // AoS double3, pointer at interior cell 0 (ghost cells at negative index)
    double const  *Bh; // B averaged onto the half grid (PartSpecies.cc:132-139), same layout
    double        *dep[2][4]; // [deposit at x^N | x^{N+1}][n, nVx, nVy, nVz], at cell 0
    double         half_min, full_min, full_max, full_len;
    double         xi, xi2, xiD1, D1, inv_D1, O0, Oc, dt, travel_scale;
    BorisK         boris;
    unsigned      *status;
    uint64_t       seed, counter;
    int            species, randomize, homogeneous_poly;
    int            move_steps; // 1: CAM-CL full step; 2: PC half step, push, half step
    int            deposit_mask; // bit0: deposit at x^N, bit1: deposit at the end position
    int            write_back;   // 0 for the PC predictor (particles are not kept)
};

template <int O, int S>
struct Acc {
    double v[4][S];
};

template <int O, int S>
__device__ __forceinline__ void acc_zero(Acc<O, S> &a)
{
#pragma unroll
    for (int q = 0; q < 4; ++q)
#pragma unroll
        for (int s = 0; s < S; ++s)
            a.v[q][s] = 0;
}

// deposit one particle: register window if its stencil fits, else direct atomics
template <int O, int S, int D>
__device__ __forceinline__ void deposit(Acc<O, S> &acc, int base, Shape<O> const &sh, double w, d3 v,
                                        PushArgs const &a)
{
    double const vw[4] = { w, v.x * w, v.y * w, v.z * w };
    int const    r     = sh.i0 - base;
    if (r >= 0 && r <= S - O - 1) {
#pragma unroll
        for (int s = 0; s < S; ++s) {
            double ws = 0;
#pragma unroll
            for (int j = 0; j <= O; ++j)
                ws = (s - r == j) ? sh.w[j] : ws;
#pragma unroll
            for (int q = 0; q < 4; ++q)
                acc.v[q][s] = fma(vw[q], ws, acc.v[q][s]);
        }
    } else {
#pragma unroll
        for (int j = 0; j <= O; ++j)
#pragma unroll
            for (int q = 0; q < 4; ++q)
                atomicAdd(a.dep[D][q] + sh.i0 + j, vw[q] * sh.w[j]);
    }
}

template <int O, int S, int D>
__device__ __forceinline__ void flush(Acc<O, S> const &acc, int base, int lane, PushArgs const &a)
{
    constexpr int tag = D;
#pragma unroll
    for (int q = 0; q < 4; ++q)
#pragma unroll
        for (int s = 0; s < S; ++s) {
            double const v = warp_sum(acc.v[q][s]);
            if (lane == ((tag * 4 + q) * S + s) % 32 && v != 0.0) {
                int const cell = base + s;
                if (cell >= -PAD && cell < a.Nx + PAD)
                    atomicAdd(a.dep[D][q] + cell, v);
                else
                    atomicOr(a.status, ST_OUT_OF_RANGE);
            }
        }
}

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
        double const c = cos(a.xiD1 * q1);
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
                sincos(gyrophase(a.seed, counter, (uint64_t)a.species, (uint64_t)pid), &s, &c);
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

// background mirror field at the particle with its gyro-radius offset
// (PartSpecies.cc:274-279; MFABasis.h:287-290; MirrorGeometry.cc:199-212)
template <bool MIRROR>
__device__ __forceinline__ d3 background_B(PushArgs const &a, double q1, d3 v)
{
    if constexpr (MIRROR) {
        double s, c;
        sincos(a.xiD1 * q1, &s, &c);
        double const ic  = 1 / c;
        double const Ocl = a.Oc * (ic * ic);
        double const rLy = -v.z / Ocl;
        double const rLz = +v.y / Ocl;
        double       x;
        if (a.homogeneous_poly) {
            double const D1q1 = q1 * a.D1;
            x                 = D1q1 * (1 + a.xi * a.xi * D1q1 * D1q1 / 3);
        } else {
            x = (s * ic) / a.xi;
        }
        return { (1 + a.xi2 * (x * x)) * a.O0, -a.xi2 * x * rLy * a.O0, -a.xi2 * x * rLz * a.O0 };
    } else {
        return { a.O0, 0, 0 };
    }
}

template <int O>
__device__ __forceinline__ d3 interp(double const *g, Shape<O> const &sh)
{
    d3 y = { 0, 0, 0 };
#pragma unroll
    for (int j = 0; j <= O; ++j) {
        d3 const f = ld3(g, sh.i0 + j);
        y.x += f.x * sh.w[j];
        y.y += f.y * sh.w[j];
        y.z += f.z * sh.w[j];
    }
    return y;
}

// One pass of a species: CAM-CL (move_steps == 1): push at x^N, deposit, move, BC, deposit.
// Predictor-corrector (move_steps == 2, Domain_PC.cc:110-124, 169-181): half move, BC,
// push at the half-step position, half move, BC, deposit.
template <int O, bool MIRROR, int BC>
__global__ void __launch_bounds__(256) push_kernel(PushArgs a)
{
    constexpr int R = 2;
    constexpr int S = O + 1 + R;
    int const     lane   = threadIdx.x & 31;
    int64_t const warp   = (static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x) >> 5;
    int64_t const chunk0 = warp * 32 * a.ppt;
    if (chunk0 >= a.n)
        return;

    // warp-uniform window base from the first particle of every lane
    int first = 0x7fffffff;
    if (chunk0 + lane < a.n) {
        Shape<O> const sh = make_shape<O>(a.q1[chunk0 + lane] - a.half_min);
        first             = sh.i0;
    }
    int const base = __reduce_min_sync(0xffffffffu, first) - 1;

    Acc<O, S> acc0, acc1;
    acc_zero(acc0);
    acc_zero(acc1);
    unsigned bad = 0;

    for (int k = 0; k < a.ppt; ++k) {
        int64_t const idx = chunk0 + static_cast<int64_t>(k) * 32 + lane;
        if (idx >= a.n)
            break;
        double   q1 = a.q1[idx];
        d3       v  = { a.vx[idx], a.vy[idx], a.vz[idx] };
        double   w  = a.w[idx];
        int32_t  pid = a.pid[idx];
        bool     alive = true;

        if (a.move_steps == 2) { // PC: first half step
            double const moved = move<MIRROR>(a, q1, v.x, 0.5 * a.dt);
            if (static_cast<long long>(moved) != 0)
                bad |= ST_MOVED_TOO_FAR;
            alive = boundary<BC>(a, q1, v, pid, a.counter);
            if (!alive) { // absorbed: park the particle with zero weight; the next sort drops it
                w  = 0;
                q1 = a.full_min + 0.5;
                v  = { 0, 0, 0 };
            }
        }
        Shape<O> const sh = make_shape<O>(q1 - a.half_min);
        if (!stencil_ok(sh, a.Nx) || !(q1 == q1)) {
            bad |= ST_OUT_OF_RANGE;
            continue;
        }
        if (alive) {
            d3 const B = background_B<MIRROR>(a, q1, v) + interp<O>(a.Bh, sh);
            d3 const E = interp<O>(a.E, sh);
            v          = boris_push(a.boris, v, B, E);
        }
        if (a.deposit_mask & 1)
            deposit<O, S, 0>(acc0, base, sh, alive ? w : 0.0, v, a);
        if (alive) {
            double const moved = move<MIRROR>(a, q1, v.x, a.move_steps == 2 ? 0.5 * a.dt : a.dt);
            if (static_cast<long long>(moved) != 0)
                bad |= ST_MOVED_TOO_FAR;
            alive = boundary<BC>(a, q1, v, pid, a.counter + (a.move_steps == 2 ? 1 : 0));
            if (!alive) {
                w  = 0;
                q1 = a.full_min + 0.5;
                v  = { 0, 0, 0 };
            }
        }
        if (a.deposit_mask & 2) {
            Shape<O> const sh2 = make_shape<O>(q1 - a.half_min);
            if (!stencil_ok(sh2, a.Nx) || !(q1 == q1))
                bad |= ST_OUT_OF_RANGE;
            else
                deposit<O, S, 1>(acc1, base, sh2, w, v, a);
        }
        if (a.write_back) {
            a.q1[idx] = q1;
            a.vx[idx] = v.x;
            a.vy[idx] = v.y;
            a.vz[idx] = v.z;
            if (BC == BCK_ABSORBING)
                a.w[idx] = w;
        }
    }
    if (a.deposit_mask & 1)
        flush<O, S, 0>(acc0, base, lane, a);
    if (a.deposit_mask & 2)
        flush<O, S, 1>(acc1, base, lane, a);
    bad = __reduce_or_sync(0xffffffffu, bad);
    if (bad && lane == 0)
        atomicOr(a.status, bad);
}

// PartSpecies::impl_collect_all (PartSpecies.cc:330-349): n, nV and nvv with CIC, unscaled
struct MomentArgs {
    double const  *q1, *vx, *vy, *vz, *w;
    int64_t        n;
    int            ppt, Nx;
    double         half_min;
    double        *out[10]; // n, nVx, nVy, nVz, xx, yy, zz, xy, yz, zx at cell 0
    unsigned      *status;
};

__global__ void __launch_bounds__(256) moments_kernel(MomentArgs a)
{
    constexpr int S = 4; // CIC + window of 2
    int const     lane   = threadIdx.x & 31;
    int64_t const warp   = (static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x) >> 5;
    int64_t const chunk0 = warp * 32 * a.ppt;
    if (chunk0 >= a.n)
        return;
    int first = 0x7fffffff;
    if (chunk0 + lane < a.n)
        first = make_shape<1>(a.q1[chunk0 + lane] - a.half_min).i0;
    int const base = __reduce_min_sync(0xffffffffu, first) - 1;
    double    acc[10][S];
#pragma unroll
    for (int q = 0; q < 10; ++q)
#pragma unroll
        for (int s = 0; s < S; ++s)
            acc[q][s] = 0;
    unsigned bad = 0;
    for (int k = 0; k < a.ppt; ++k) {
        int64_t const idx = chunk0 + static_cast<int64_t>(k) * 32 + lane;
        if (idx >= a.n)
            break;
        double const   q1 = a.q1[idx], vx = a.vx[idx], vy = a.vy[idx], vz = a.vz[idx], w = a.w[idx];
        Shape<1> const sh = make_shape<1>(q1 - a.half_min);
        if (!stencil_ok(sh, a.Nx) || !(q1 == q1)) {
            bad |= ST_OUT_OF_RANGE;
            continue;
        }
        double const val[10] = { w,           vx * w,      vy * w,      vz * w,      (vx * vx) * w,
                                 (vy * vy) * w, (vz * vz) * w, (vx * vy) * w, (vy * vz) * w, (vz * vx) * w };
        int const    r       = sh.i0 - base;
        if (r >= 0 && r <= S - 2) {
#pragma unroll
            for (int s = 0; s < S; ++s) {
                double const ws = (s == r) ? sh.w[0] : (s == r + 1) ? sh.w[1] : 0.0;
#pragma unroll
                for (int q = 0; q < 10; ++q)
                    acc[q][s] = fma(val[q], ws, acc[q][s]);
            }
        } else {
#pragma unroll
            for (int j = 0; j <= 1; ++j)
#pragma unroll
                for (int q = 0; q < 10; ++q)
                    atomicAdd(a.out[q] + sh.i0 + j, val[q] * sh.w[j]);
        }
    }
#pragma unroll
    for (int q = 0; q < 10; ++q)
#pragma unroll
        for (int s = 0; s < S; ++s) {
            double const v = warp_sum(acc[q][s]);
            if (lane == (q * S + s) % 32 && v != 0.0) {
                int const cell = base + s;
                if (cell >= -PAD && cell < a.Nx + PAD)
                    atomicAdd(a.out[q] + cell, v);
                else
                    bad |= ST_OUT_OF_RANGE;
            }
        }
    bad = __reduce_or_sync(0xffffffffu, bad);
    if (bad && lane == 0)
        atomicOr(a.status, bad);
}

} // namespace h1d
