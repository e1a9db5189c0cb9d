// Small grid kernels: ghost fill on the first advance, the post-process of advance_by
// (collect_all scaling and boundary_gather, ColdSpecies::collect_all) and the energy reductions
// of EnergyRecorder::dump.
#pragma once

#include "device_common.cuh"
#include "h1d_gpu.h"
#include "launchers.h"

namespace h1d {

__global__ void fill_kernel(double *a, int64_t n, double v)
{
    int64_t const i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i < n)
        a[i] = v;
}
__global__ void fill_f_kernel(float *a, int64_t n, float v)
{
    int64_t const i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i < n)
        a[i] = v;
}
__global__ void iota_kernel(int32_t *pid, int64_t n)
{
    int64_t const i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i < n)
        pid[i] = static_cast<int32_t>(i);
}

__device__ __forceinline__ int wrap(int i, int Nx) { return i < 0 ? i + Nx : i >= Nx ? i - Nx : i; }

// the periodic ghost fill of an interleaved array of `nc` components per cell (a at interior cell
// 0): the boundary_pass a delegate applies to a grid array (Delegate.cc:76-87), e.g. to the cold
// fluid's mom0_full / mom1_full at the start of a predictor-corrector run (Domain_PC.cc:46)
// (the ghosts of `dst` from the interior of `src`, which may be the same array)
__global__ void ghost_fill_kernel(double *dst, double const *src, int nc, int Nx)
{
    int const k = static_cast<int>(threadIdx.x); // PAD ghost cells on each side
    if (k >= PAD)
        return;
    for (int c = 0; c < nc; ++c) {
        dst[nc * (k - PAD) + c] = src[nc * (Nx - PAD + k) + c];
        dst[nc * (Nx + k) + c]  = src[nc * k + c];
    }
}

// boundary_pass of E and B (periodic ghost fill, Delegate.cc:76-87) and the push record
// {E, B on the half grid} (PartSpecies.cc:27-34; the last ghost's half-grid B stays NaN)
__global__ void prep_fields_kernel(double *B, double *E, double *EB, float *EBf, int Nx)
{
    int const i = static_cast<int>(blockIdx.x * blockDim.x + threadIdx.x) - PAD;
    if (i >= Nx + PAD)
        return;
    d3 const e = ld3(E, wrap(i, Nx));
    double  *p = EB + 6 * i;
    p[0] = e.x, p[1] = e.y, p[2] = e.z;
    if (i < Nx + PAD - 1) {
        d3 const b1 = ld3(B, wrap(i + 1, Nx)), b0 = ld3(B, wrap(i, Nx));
        d3 const bh = (b1 + b0) * 0.5;
        p[3] = bh.x, p[4] = bh.y, p[5] = bh.z;
    } else {
        p[3] = p[4] = p[5] = __longlong_as_double(0x7ff8000000000000LL);
    }
    if (EBf)
        for (int c = 0; c < 6; ++c)
            EBf[EBF_STRIDE * i + c] = static_cast<float>(p[c]);
    if (i < 0 || i >= Nx) {
        st3(B, i, ld3(B, wrap(i, Nx)));
        st3(E, i, e);
    }
}

// collect_all scaling by 1/Nc (PartSpecies.cc:241-243) and boundary_gather of the three moments
// (SubdomainDelegate.cc:115-181).  raw: 10 arrays of M (n, nV xyz, nvv xx yy zz xy yz zx);
// out: GridArray layout n[M], nV[3M], nvv[6M].
// delta-f species (eq != null): + the equilibrium n0 (M) and nvv0 (6M) x m_moment_weighting_factor
// (PartSpecies.cc:129-143), before the ghost fold as in the reference
__global__ void finalize_kinetic_kernel(double const *raw, double const *eq, double *out, int Nx, double s1)
{
    int const M = Nx + 2 * PAD;
    int const i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= M)
        return;
    double *n = out, *nV = out + M, *nvv = out + 4 * M;
    n[i]      = raw[i] * s1;
    for (int c = 0; c < 3; ++c)
        nV[3 * i + c] = raw[(1 + c) * M + i] * s1;
    for (int c = 0; c < 6; ++c)
        nvv[6 * i + c] = raw[(4 + c) * M + i] * s1;
    if (eq) {
        n[i] = n[i] + eq[i] * 1.0;
        for (int c = 0; c < 6; ++c)
            nvv[6 * i + c] = nvv[6 * i + c] + eq[M + 6 * i + c] * 1.0;
    }
}
// the ghost fold of the finalized moments, one thread per component (n; nV xyz; nvv x 6)
__global__ void fold_moments_kernel(double *out, int Nx, int reflecting)
{
    int const t = threadIdx.x;
    if (t >= 10)
        return;
    int const M  = Nx + 2 * PAD;
    int const nc = t == 0 ? 1 : t < 4 ? 3 : 6;
    int const c  = t == 0 ? 0 : t < 4 ? t - 1 : t - 4;
    double   *a  = t == 0 ? out : t < 4 ? out + M : out + 4 * M;
    if (reflecting) {
        for (int i = 0; i < PAD; ++i) { // cells -3 -> -2 -> -1 -> 0
            a[nc * (i + 1) + c] += a[nc * i + c];
            a[nc * i + c] = 0;
        }
        for (int i = M - 1; i >= Nx + PAD; --i) {
            a[nc * (i - 1) + c] += a[nc * i + c];
            a[nc * i + c] = 0;
        }
    }
    double left[PAD], right[PAD];
    for (int k = 0; k < PAD; ++k)
        left[k] = a[nc * k + c], right[k] = a[nc * (Nx + PAD + k) + c];
    for (int k = 0; k < PAD; ++k)
        a[nc * (Nx + k) + c] += left[k];
    for (int k = 0; k < PAD; ++k)
        a[nc * (PAD + k) + c] += right[k];
}

// ColdSpecies::collect_all (ColdSpecies.cc:48-77): moments x weight on the interior,
// zero ghosts, nvv = (nV/n) nV
__global__ void finalize_cold_kernel(double const *n_full, double const *nV_full, double *out, int Nx, double w)
{
    int const M = Nx + 2 * PAD;
    double   *n = out, *nV = out + M, *nvv = out + 4 * M;
    for (int i = threadIdx.x; i < M; i += blockDim.x) {
        bool const interior = i >= PAD && i < Nx + PAD;
        double const ni     = interior ? n_full[i] * w : 0.0;
        d3 const     v      = interior ? ld3(nV_full, i) * w : d3{ 0, 0, 0 };
        n[i]                = ni;
        st3(nV, i, v);
        double t[6] = { 0, 0, 0, 0, 0, 0 };
        if (interior) {
            t[0] = t[3] = v.x / ni;
            t[1] = t[4] = v.y / ni;
            t[2] = t[5] = v.z / ni;
            t[0] *= v.x, t[1] *= v.y, t[2] *= v.z;
            t[3] *= v.y, t[4] *= v.z, t[5] *= v.x;
        }
        for (int c = 0; c < 6; ++c)
            nvv[6 * i + c] = t[c];
    }
}

__device__ double block_sum(double v, double *sh)
{
    v = warp_sum(v);
    if ((threadIdx.x & 31) == 0)
        sh[threadIdx.x >> 5] = v;
    __syncthreads();
    double r = 0;
    if (threadIdx.x < 32) {
        r = threadIdx.x < (blockDim.x >> 5) ? sh[threadIdx.x] : 0.0;
        r = warp_sum(r);
    }
    __syncthreads();
    return r;
}

// EnergyRecorder::dump (EnergyRecorder.cc:98-140); MFA components equal Cartesian ones here
__global__ void energy_kernel(EnergyArgs a)
{
    __shared__ double sh[32];
    double const      denom = 2 * static_cast<double>(a.Nx);
    for (int f = 0; f < 2; ++f) {
        double const *g = f ? a.E : a.B;
        for (int c = 0; c < 3; ++c) {
            double acc = 0;
            for (int i = threadIdx.x; i < a.Nx; i += blockDim.x)
                acc += g[3 * i + c] * g[3 * i + c];
            double const s = block_sum(acc, sh);
            if (threadIdx.x == 0)
                a.out[3 * f + c] = s / denom;
        }
    }
    for (int s = 0; s < a.ns; ++s)
        for (int c = 0; c < 3; ++c) {
            double lab = 0, pla = 0;
            for (int i = threadIdx.x; i < a.Nx; i += blockDim.x) {
                double const n = a.n[s][i];
                if (n < 1e-15)
                    continue;
                double const t = a.nvv[s][6 * i + c], v = a.nV[s][3 * i + c];
                lab += t;
                pla += t - v * v / n;
            }
            double const L = block_sum(lab, sh), P = block_sum(pla, sh);
            if (threadIdx.x == 0) {
                a.out[6 + 6 * s + c]     = L * a.factor[s];
                a.out[6 + 6 * s + 3 + c] = P * a.factor[s];
            }
        }
}

// ExternalSource::update / collect (Core/ExternalSource.cc:12-66): the moment<1> of every external
// source at time t, deposited with Shape<1> at its points inside the half-grid extent; one block,
// the points in order on one thread (the reference's order), no contraction (this unit).
__global__ void source_kernel(SourceArgs a)
{
    for (int e = 0; e < a.ne; ++e)
        for (int c = 0; c < 3; ++c)
            for (int i = threadIdx.x; i < a.M; i += blockDim.x)
                a.J[e][c][i - PAD] = 0;
    __syncthreads();
    if (threadIdx.x != 0)
        return;
    for (int e = 0; e < a.ne; ++e) {
        h1d_source_desc const &d = a.d[e];
        // envelope (ExternalSource.cc:44-67) with the ramp slopes of ExternalSource.hh:29-32
        double const eps       = 1e-15;
        double const slope_in  = 3.141592653589793 / (d.ease_in > eps ? d.ease_in : 1.0);
        double const slope_out = 3.141592653589793 / (d.ease_out > eps ? d.ease_out : 1.0);
        double       tt        = a.t - d.start;
        double       env;
        if (tt < -d.ease_in)
            env = 0;
        else if (tt < 0)
            env = .5 * (1 + cos(slope_in * tt));
        else if (tt < d.duration)
            env = 1;
        else if ((tt -= d.duration) < d.ease_out)
            env = .5 * (1 + cos(slope_out * tt));
        else
            env = 0;
        for (int i = 0; i < d.n_points; ++i) {
            double const pos = d.pos[i];
            if (!(pos >= a.half_min && pos < a.half_min + a.half_len))
                continue;
            Shape<1> const sx    = make_shape<1>(pos - a.half_min);
            double const   phase = -d.omega * (a.t - d.start);
            double const   cs = cos(phase), sn = sin(phase);
            double const   f  = env * a.weighting;
            for (int c = 0; c < 3; ++c) {
                double const v = (d.J0re[i][c] * cs - d.J0im[i][c] * sn) * f;
                a.J[e][c][sx.i0] += v * sx.w[0];
                a.J[e][c][sx.i0 + 1] += v * sx.w[1];
            }
        }
    }
}

} // namespace h1d
