// Mixed-precision particle pass: the same cycle as push_kernel (particles.cuh) with
//   - position as one int32 in fixed point: x = q1 - q1min (full grid, in cells) times 2^F, F =
//     31 - ceil(log2(Nx + 2)) fraction bits (18 at Nx = 4096), so the cell is X >> F and the
//     in-cell offset the low F bits; the shape weights come from the offset, a move is an exact
//     integer addition of the displacement rounded to 2^-F cell, and the resolution is the same
//     anywhere on the grid;
//   - FP32 velocity, weight, field interpolation, mirror geometry and Boris push;
//   - FP32 deposits into per-lane shared-memory columns of a per-warp window of cells, summed
//     into the FP64 moment arrays per cell when the window moves.
// The field cycle that consumes the moments stays FP64.  Traffic: read position, v, w (20 B),
// write position, v (16 B) per particle-step.
#pragma once

#include "particles.cuh"

namespace h1d {

struct PushArgsMixed {
    int32_t     *pos; // fixed-point position (pos_cell, pos_off)
    float       *vx, *vy, *vz, *w;
    int32_t const *pid;
    int64_t      n;
    int          Nx;
    float const *EB; // per cell {Ex, Ey, Ez, dBx, dBy, dBz, 0, 0} in FP32 (EBF_STRIDE), at interior cell 0
    double      *dep[2][4];
    double      *nvv[6]; // collect_all's xx, yy, zz, xy, yz, zx sums at cell 0 (NVV launches only)
    float        full_min, xiD1, inv_D1, O0, dt, travel_scale, xiO0_Oc, dtOc_2O0, cDtOc_2O0;
    int          fbits;            // F, the fraction bits of a position
    float        scale, inv_scale; // 2^F, 2^-F
    unsigned    *status;
    unsigned long long *fallbacks;
    uint64_t     seed, counter;
    int          species, randomize;
    int          move_steps, deposit_mask, write_back;
    // evolving weights (push_kernel_mixed<..., PSD = true>): FP32 Particle::PSD arrays and the
    // equilibrium distribution of PartSpecies::impl_update_weight, as in PushArgs
    float       *real_f, *marker;
    float        nu_dt, vth1, vth1_cubed, T2_T1;
    float        vc[4];
    int          vdf, psd_refresh, delta_f;
};

struct f3 {
    float x, y, z;
};
__device__ __forceinline__ f3 operator+(f3 a, f3 b) { return { a.x + b.x, a.y + b.y, a.z + b.z }; }
__device__ __forceinline__ f3 operator*(f3 a, float s) { return { a.x * s, a.y * s, a.z * s }; }
__device__ __forceinline__ f3 crossf(f3 A, f3 B) { return { A.y * B.z - A.z * B.y, A.z * B.x - A.x * B.z, A.x * B.y - A.y * B.x }; }

// pairs of FP32 values (a lane's two particles) on the packed FP32 pipe of sm_100
__device__ __forceinline__ float2 bc(float s) { return make_float2(s, s); }
__device__ __forceinline__ float2 padd(float2 a, float2 b) { return __fadd2_rn(a, b); }
__device__ __forceinline__ float2 pmul(float2 a, float2 b) { return __fmul2_rn(a, b); }
__device__ __forceinline__ float2 pfma(float2 a, float2 b, float2 c) { return __ffma2_rn(a, b, c); }
__device__ __forceinline__ float2 pneg(float2 a) { return make_float2(-a.x, -a.y); }
__device__ __forceinline__ float &el(float2 &p, int k) { return k ? p.y : p.x; }
__device__ __forceinline__ float  el(float2 const &p, int k) { return k ? p.y : p.x; }
struct p3 {
    float2 x, y, z;
};
__device__ __forceinline__ p3 padd3(p3 a, p3 b) { return { padd(a.x, b.x), padd(a.y, b.y), padd(a.z, b.z) }; }
// A x B, each component as one multiply and one fused multiply-subtract
__device__ __forceinline__ p3 pcross(p3 A, p3 B)
{
    return { pfma(A.y, B.z, pneg(pmul(A.z, B.y))), pfma(A.z, B.x, pneg(pmul(A.x, B.z))),
             pfma(A.x, B.y, pneg(pmul(A.y, B.x))) };
}

// shape weights from the in-cell offset: x - q1min_half = cell - 1/2 + off (Shape.h:24-176)
template <int O>
struct ShapeF {
    int   i0;
    float w[O + 1];
};
template <int O>
__device__ __forceinline__ ShapeF<O> make_shape_f(int cell, float off)
{
    ShapeF<O> s;
    if constexpr (O == 1) {
        bool const up = off >= 0.5f;
        s.i0          = up ? cell : cell - 1;
        s.w[1]        = up ? off - 0.5f : off + 0.5f;
        s.w[0]        = 1.0f - s.w[1];
    } else if constexpr (O == 2) {
        s.i0           = cell - 1;
        float const t  = 0.5f - off;
        float const u  = 1.0f - off;
        s.w[0]         = 0.5f * (u * u);
        s.w[1]         = 0.75f - t * t;
        s.w[2]         = 0.5f * (off * off);
    } else {
        bool const  up = off > 0.5f;
        s.i0           = up ? cell - 1 : cell - 2;
        float const u  = up ? off - 0.5f : off + 0.5f; // x - (i0 + 1)
        float const v  = 1.0f - u;
        float const u2 = u * u, u3 = u2 * u;
        s.w[0]         = (1.0f / 6) * (v * v * v);
        s.w[1]         = (1.0f / 6) * (4.0f - 6.0f * u2 + 3.0f * u3);
        s.w[3]         = (1.0f / 6) * u3;
        s.w[2]         = 1.0f - (s.w[0] + s.w[1] + s.w[3]);
    }
    return s;
}
// the shape of a fixed-point position X (make_shape_f of its cell and offset).  For CIC the
// position relative to the half grid, X - 2^(F-1), gives the base cell (arithmetic shift) and the
// weight of the upper cell (its low F bits) in one integer step; the weights are the same floats.
template <int O>
__device__ __forceinline__ ShapeF<O> make_shape_fx(int32_t X, int F, float inv_scale)
{
    if constexpr (O == 1) {
        int32_t const H = static_cast<int32_t>(static_cast<uint32_t>(X) - (1u << (F - 1)));
        ShapeF<1>     s;
        s.i0   = H >> F;
        s.w[1] = static_cast<float>(H & ((1 << F) - 1)) * inv_scale;
        s.w[0] = 1.0f - s.w[1];
        return s;
    } else {
        return make_shape_f<O>(X >> F, static_cast<float>(X & ((1 << F) - 1)) * inv_scale);
    }
}
template <int O>
__device__ __forceinline__ bool stencil_ok_f(ShapeF<O> const &sh, int Nx)
{
    return sh.i0 >= -PAD && sh.i0 + O < Nx + PAD;
}

// sin and cos of |x| <= pi/2 in FP32 from their Taylor series through x^13 and x^14
__device__ __forceinline__ void sincos_taylor_f(float x, float &s, float &c)
{
    float const x2 = x * x;
    float       ps = -1.6059043836821613e-10f;
    ps             = fmaf(ps, x2, 2.505210838544172e-08f);
    ps             = fmaf(ps, x2, -2.7557319223985893e-06f);
    ps             = fmaf(ps, x2, 0.0001984126984126984f);
    ps             = fmaf(ps, x2, -0.008333333333333333f);
    ps             = fmaf(ps, x2, 0.16666666666666666f);
    s              = fmaf(-ps * x2, x, x);
    float pc       = 1.1470745597729725e-11f;
    pc             = fmaf(pc, x2, -2.08767569878681e-09f);
    pc             = fmaf(pc, x2, 2.755731922398589e-07f);
    pc             = fmaf(pc, x2, -2.48015873015873e-05f);
    pc             = fmaf(pc, x2, 0.001388888888888889f);
    pc             = fmaf(pc, x2, -0.041666666666666664f);
    pc             = fmaf(pc, x2, 0.5f);
    c              = fmaf(-pc, x2, 1.0f);
}

// sincos_taylor_f of a pair
__device__ __forceinline__ void sincos_taylor_f2(float2 x, float2 &s, float2 &c)
{
    float2 const x2 = pmul(x, x);
    float2       ps = bc(-1.6059043836821613e-10f);
    ps              = pfma(ps, x2, bc(2.505210838544172e-08f));
    ps              = pfma(ps, x2, bc(-2.7557319223985893e-06f));
    ps              = pfma(ps, x2, bc(0.0001984126984126984f));
    ps              = pfma(ps, x2, bc(-0.008333333333333333f));
    ps              = pfma(ps, x2, bc(0.16666666666666666f));
    s               = pfma(pneg(pmul(ps, x2)), x, x);
    float2 pc       = bc(1.1470745597729725e-11f);
    pc              = pfma(pc, x2, bc(-2.08767569878681e-09f));
    pc              = pfma(pc, x2, bc(2.755731922398589e-07f));
    pc              = pfma(pc, x2, bc(-2.48015873015873e-05f));
    pc              = pfma(pc, x2, bc(0.001388888888888889f));
    pc              = pfma(pc, x2, bc(-0.041666666666666664f));
    pc              = pfma(pc, x2, bc(0.5f));
    c               = pfma(pneg(pc), x2, bc(1.0f));
}

// a fixed-point position: its full-grid cell and its offset in the cell, [0, 1) exactly
__device__ __forceinline__ int   pos_cell(int32_t X, int F) { return X >> F; }
__device__ __forceinline__ float pos_off(int32_t X, int F, float inv_scale)
{
    return static_cast<float>(X & ((1 << F) - 1)) * inv_scale;
}
// move by dq cells (|dq| < 1 is checked by the caller): an integer addition of dq rounded to 2^-F
__device__ __forceinline__ void move_pos(int32_t &X, float dq, float scale) { X += __float2int_rn(dq * scale); }

template <int BC>
__device__ __forceinline__ bool boundary_mixed(PushArgsMixed const &a, int32_t &X, f3 &v, int32_t pid, uint64_t counter)
{
    int32_t const len = a.Nx << a.fbits; // the domain [0, Nx) in fixed point
    if constexpr (BC == BCK_PERIODIC) {
        if (X < 0)
            X += len;
        else if (X >= len)
            X -= len;
        return true;
    } else if constexpr (BC == BCK_REFLECTING) {
        bool const left = X < 0, right = X >= len;
        if (left || right) { // q1 -> 2 q1_boundary - q1 (Delegate.cc:116-145)
            if (left)        // x -> -x
                X = -X;
            else // x -> 2 Nx - x; x = Nx exactly stays inside, at the last position of the grid
                X = X > len ? len - (X - len) : len - 1;
            v.x = -v.x;
            if (a.randomize) {
                float s, c;
                float const x    = static_cast<float>(gyrophase(a.seed, counter, (uint64_t)a.species, (uint64_t)pid));
                bool const  flip = fabsf(x) > 1.5707963f; // one half-turn onto |x| <= pi/2 for the series
                sincos_taylor_f(flip ? x - copysignf(3.14159265f, x) : x, s, c);
                if (flip)
                    s = -s, c = -c;
                float const vy = v.y, vz = v.z;
                v.y = vy * c - vz * s;
                v.z = vy * s + vz * c;
            }
        }
        return true;
    } else {
        return X >= 0 && X < len;
    }
}

// ------------------------------------------------------------------------------------------------
// The pass.  Same warp-specialised TMA pipeline as push_kernel (particles.cuh) with chunks of
// MIX_CHUNK particles.  A consumer warp owns 32 x MIX_PPT particles of a chunk and does everything
// in one loop: push, move, boundary, and both deposits.  Deposits go to a per-warp window of
// MIX_W cells held in shared memory as lane-private float4 columns {n, nVx, nVy, nVz}: lane l adds
// its particle to column l of cell (i0 - base + j), so any mix of cells within a warp costs the
// same (no divergence, no bank conflicts), and lanes never collide.  When a particle's stencil
// falls outside the window the warp flushes it (per cell and quantity a warp reduce-scatter over
// the 32 columns, then one FP64 atomic) and re-centres it on the current particles; particles
// still outside deposit with direct atomics.  The CTA's particles are cell-sorted and contiguous,
// so the window moves a few times per CTA.
// ------------------------------------------------------------------------------------------------
constexpr int MIX_CHUNK = 256;
constexpr int MIX_PPT   = MIX_CHUNK / (32 * PIPE_CONSUMER_WARPS);
static_assert(MIX_PPT == 2, "a lane pushes one pair of particles per chunk");
constexpr int MIX_W     = 8; // 4 quantities x 8 cells = the 32 lanes of a flush
static_assert(4 * MIX_W == 32, "a window flush reduce-scatters exactly 32 values");

// a stage holds one chunk; the consumers overwrite it in place with the new state, which the
// producer then stores.  With evolving weights (PSD) a stage also holds real_f and marker and the
// pipeline is one stage shorter, so that four CTAs still fit an SM.
template <bool PSD>
struct PipeStageMixedT {
    int32_t pos[MIX_CHUNK];
    float   vx[MIX_CHUNK], vy[MIX_CHUNK], vz[MIX_CHUNK], w[MIX_CHUNK];
    int32_t pid[MIX_CHUNK];
    float   real_f[PSD ? MIX_CHUNK : 4], marker[PSD ? MIX_CHUNK : 4];
};
using PipeStageMixed = PipeStageMixedT<false>;
constexpr int    PIPE_STAGES_MIXED      = 3;
constexpr int    PIPE_CTAS_PER_SM_MIXED = 4;
// A launch that also forms collect_all's second moments (NVV, the last step of an advance_by)
// holds a second window per warp and is one stage shorter, so that three CTAs fit an SM.
template <bool PSD, bool NVV = false>
struct MixLayout {
    static constexpr int    STAGES     = PSD || NVV ? PIPE_STAGES_MIXED - 1 : PIPE_STAGES_MIXED;
    static constexpr size_t BAR_OFFSET = sizeof(PipeStageMixedT<PSD>) * STAGES;
    static constexpr size_t COL_OFFSET = BAR_OFFSET + 128; // barriers, then 16-byte aligned columns
};
constexpr size_t MIX_COL_BYTES        = sizeof(float4) * PIPE_CONSUMER_WARPS * 2 * MIX_W * 32;
constexpr size_t MIX_NVV_BYTES        = (sizeof(float4) + sizeof(float2)) * PIPE_CONSUMER_WARPS * MIX_W * 32;
constexpr size_t PIPE_SMEM_MIXED      = MixLayout<false>::COL_OFFSET + MIX_COL_BYTES;
constexpr size_t PIPE_SMEM_MIXED_PSD  = MixLayout<true>::COL_OFFSET + MIX_COL_BYTES;
constexpr size_t PIPE_SMEM_MIXED_NVV  = MixLayout<false, true>::COL_OFFSET + MIX_COL_BYTES + MIX_NVV_BYTES;
static_assert(3 * (PIPE_SMEM_MIXED_NVV + 1024) <= 233472, "three CTAs of a second-moment launch fit an SM");
static_assert(2 * PIPE_STAGES_MIXED * sizeof(uint64_t) <= 128, "barriers fit before the columns");
static_assert(PIPE_CTAS_PER_SM_MIXED * (PIPE_SMEM_MIXED_PSD + 1024) <= 233472, "four CTAs with evolving weights fit an SM");

// PartSpecies::impl_update_weight in FP32 for one particle after its velocity update (as
// update_weight and equilibrium_f0, particles.cuh): f0 of the equilibrium distribution at velocity
// v and at the push position (c2 = cos^2(xi D1 q1)), then real_f and the weight
__device__ __forceinline__ float update_weight_f(PushArgsMixed const &a, f3 v, float c2, float &real_f, float marker)
{
    constexpr float PI = 3.14159265358979f, INV_SQRTPI = 0.5641895835477563f;
    float const     x1 = v.x / a.vth1, x2 = v.y / a.vth1, x3 = v.z / a.vth1;
    float           f0;
    if (a.vdf == H1D_VDF_LOSSCONE) {
        float const X = a.vc[1], bX = a.vc[2], beq = a.vc[0];
        float const eta   = 1.0f / (X + (1.0f - X) * c2);
        float const eta_b = 1.0f / (bX + (1.0f - bX) * c2);
        float       beta  = beq * eta_b / eta;
        if (fabsf(beta - 1.0f) < 1e-6f) // beta = 1 is a removable singularity; FP32 resolves 1e-6
            beta = beta < 1.0f ? 1.0f - 1e-6f : 1.0f + 1e-6f;
        float const x2s = X * eta;
        float const y   = (x2 * x2 + x3 * x3) / x2s;
        float const f2  = (expf(-y) - expf(-y / beta)) / (PI * x2s * (1.0f - beta));
        f0 = ((eta - beq * eta_b) / (1.0f - beq)) * ((expf(-x1 * x1) * INV_SQRTPI * f2) / a.vth1_cubed);
    } else if (a.vdf == H1D_VDF_PARTIAL_SHELL || a.vdf == H1D_VDF_COUNTER_BEAM) {
        float const x  = sqrtf(x1 * x1 + x2 * x2 + x3 * x3);
        float const t  = x - a.vc[1];
        float const fv = expf(-t * t) / a.vc[2];
        float const u  = x1 / x;
        float const s2 = (1.0f - u) * (1.0f + u); // sin^2(alpha)
        if (a.vdf == H1D_VDF_PARTIAL_SHELL) {
            bool const iso = a.vc[0] == 0.0f;
            // sin^zeta(alpha) cs^zeta = (s2 c2)^(zeta/2)
            float const fa = iso ? 1.0f : powf(s2 * c2, 0.5f * a.vc[0]);
            f0 = 0.5f * fv * fa / (a.vc[3] * PI * a.vth1_cubed);
        } else {
            f0 = fv * expf(-s2 * c2 / (a.vc[0] * a.vc[0])) / (a.vc[3] * 2.0f * PI * a.vth1_cubed);
        }
    } else {
        float const eta   = 1.0f / (a.T2_T1 + (1.0f - a.T2_T1) * c2);
        float const T2OT1 = a.T2_T1 * eta;
        float const f1    = expf(-x1 * x1) * INV_SQRTPI;
        float const f2    = expf(-(x2 * x2 + x3 * x3) / T2OT1) / (PI * T2OT1);
        f0 = eta * ((f1 * f2) / a.vth1_cubed);
    }
    if (a.psd_refresh)
        real_f = (real_f + a.nu_dt * f0) / (1.0f + a.nu_dt);
    return a.delta_f ? (real_f - f0) / marker : real_f / marker;
}

// a warp's deposit window: columns [d][c][lane] (d: deposit at x^N / at the end position)
struct ColWindow {
    static constexpr int NONE = -0x40000000;
    float4              *col;
    int                  base;

    __device__ __forceinline__ float4 &at(int d, int c, int lane) { return col[(d * MIX_W + c) * 32 + lane]; }
    __device__ __forceinline__ void    zero(int lane)
    {
#pragma unroll
        for (int d = 0; d < 2; ++d)
#pragma unroll
            for (int c = 0; c < MIX_W; ++c)
                at(d, c, lane) = make_float4(0.f, 0.f, 0.f, 0.f);
    }
    template <int O>
    __device__ __forceinline__ void add(int d, ShapeF<O> const &sh, float4 vw, int lane)
    {
        int const r = sh.i0 - base;
#pragma unroll
        for (int j = 0; j <= O; ++j) {
            float4 &e = at(d, r + j, lane);
            float4  t = e;
            t.x = fmaf(vw.x, sh.w[j], t.x), t.y = fmaf(vw.y, sh.w[j], t.y);
            t.z = fmaf(vw.z, sh.w[j], t.z), t.w = fmaf(vw.w, sh.w[j], t.w);
            e   = t;
        }
    }
    // sum the 32 columns of every (cell, quantity) of deposit d, add to the moments, clear
    __device__ __forceinline__ void flush_one(int d, int lane, PushArgsMixed const &a)
    {
        float x[32];
#pragma unroll
        for (int c = 0; c < MIX_W; ++c) {
            float4 const v = at(d, c, lane);
            x[4 * c] = v.x, x[4 * c + 1] = v.y, x[4 * c + 2] = v.z, x[4 * c + 3] = v.w;
            at(d, c, lane) = make_float4(0.f, 0.f, 0.f, 0.f);
        }
#pragma unroll
        for (int h = 16; h >= 1; h >>= 1) {
            bool const up = (lane & h) != 0;
#pragma unroll
            for (int j = 0; j < h; ++j) {
                float const send = up ? x[j] : x[j + h];
                float const keep = up ? x[j + h] : x[j];
                x[j]             = keep + __shfl_xor_sync(0xffffffffu, send, h);
            }
        }
        if (x[0] != 0.0f) { // lane l holds the total of value l = 4 * cell + quantity
            int const cell = base + (lane >> 2);
            if (cell >= -PAD && cell < a.Nx + PAD)
                atomicAdd(a.dep[d][lane & 3] + cell, static_cast<double>(x[0]));
            else
                atomicOr(a.status, ST_OUT_OF_RANGE);
        }
    }
    __device__ __forceinline__ void flush(int lane, PushArgsMixed const &a)
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
// warp and cell, lane-private columns {xx, yy, zz, xy} (float4) and {yz, zx} (float2), over the
// cells of the warp's main window (same base, flushed and moved with it)
struct NvvWindow {
    float4 *c4;
    float2 *c2;

    __device__ __forceinline__ float4 &a4(int c, int lane) { return c4[c * 32 + lane]; }
    __device__ __forceinline__ float2 &a2(int c, int lane) { return c2[c * 32 + lane]; }
    __device__ __forceinline__ void    zero(int lane)
    {
#pragma unroll
        for (int c = 0; c < MIX_W; ++c)
            a4(c, lane) = make_float4(0.f, 0.f, 0.f, 0.f), a2(c, lane) = make_float2(0.f, 0.f);
    }
    template <int O>
    __device__ __forceinline__ void add(int base, ShapeF<O> const &sh, float const (&v)[6], int lane)
    {
        int const r = sh.i0 - base;
#pragma unroll
        for (int j = 0; j <= O; ++j) {
            float4 &e = a4(r + j, lane);
            float2 &f = a2(r + j, lane);
            float4  t = e;
            float2  u = f;
            t.x = fmaf(v[0], sh.w[j], t.x), t.y = fmaf(v[1], sh.w[j], t.y);
            t.z = fmaf(v[2], sh.w[j], t.z), t.w = fmaf(v[3], sh.w[j], t.w);
            u.x = fmaf(v[4], sh.w[j], u.x), u.y = fmaf(v[5], sh.w[j], u.y);
            e = t, f = u;
        }
    }
    // the columns summed over the warp and added to the moment sums: {xx, yy, zz, xy} of the MIX_W
    // cells as one 32-value reduce-scatter (lane l: value 4 c + q), {yz, zx} as a 16-value one
    // (lanes 2 k and 2 k + 1: value k = 2 c + q)
    __device__ __forceinline__ void flush(int base, int lane, PushArgsMixed const &a)
    {
        if (base == ColWindow::NONE)
            return;
        float x[32], y[16];
#pragma unroll
        for (int c = 0; c < MIX_W; ++c) {
            float4 const t = a4(c, lane);
            float2 const u = a2(c, lane);
            x[4 * c] = t.x, x[4 * c + 1] = t.y, x[4 * c + 2] = t.z, x[4 * c + 3] = t.w;
            y[2 * c] = u.x, y[2 * c + 1] = u.y;
            a4(c, lane) = make_float4(0.f, 0.f, 0.f, 0.f), a2(c, lane) = make_float2(0.f, 0.f);
        }
#pragma unroll
        for (int h = 16; h >= 1; h >>= 1) {
            bool const up = (lane & h) != 0;
#pragma unroll
            for (int j = 0; j < h; ++j) {
                float const send = up ? x[j] : x[j + h];
                float const keep = up ? x[j + h] : x[j];
                x[j]             = keep + __shfl_xor_sync(0xffffffffu, send, h);
            }
        }
#pragma unroll
        for (int h = 8, m = 16; h >= 1; h >>= 1, m >>= 1) {
            bool const up = (lane & m) != 0;
#pragma unroll
            for (int j = 0; j < h; ++j) {
                float const send = up ? y[j] : y[j + h];
                float const keep = up ? y[j + h] : y[j];
                y[j]             = keep + __shfl_xor_sync(0xffffffffu, send, m);
            }
        }
        float const yz = y[0] + __shfl_xor_sync(0xffffffffu, y[0], 1);
        unsigned    bad = 0;
        if (x[0] != 0.0f) {
            int const cell = base + (lane >> 2);
            if (cell >= -PAD && cell < a.Nx + PAD)
                atomicAdd(a.nvv[lane & 3] + cell, static_cast<double>(x[0]));
            else
                bad = ST_OUT_OF_RANGE;
        }
        if ((lane & 1) == 0 && yz != 0.0f) {
            int const k = lane >> 1, cell = base + (k >> 1);
            if (cell >= -PAD && cell < a.Nx + PAD)
                atomicAdd(a.nvv[4 + (k & 1)] + cell, static_cast<double>(yz));
            else
                bad = ST_OUT_OF_RANGE;
        }
        if (bad)
            atomicOr(a.status, bad);
    }
};

// the second moments of a particle outside the window, by direct atomics
template <int O>
__device__ __forceinline__ void nvv_direct(PushArgsMixed const &a, ShapeF<O> const &sh, float const (&v)[6])
{
#pragma unroll
    for (int j = 0; j <= O; ++j)
#pragma unroll
        for (int q = 0; q < 6; ++q)
            atomicAdd(a.nvv[q] + sh.i0 + j, static_cast<double>(v[q] * sh.w[j]));
}

// the groups of one launch, as PushGroups in particles.cuh
template <int MAXG>
struct PushGroupsMixed {
    static constexpr int MAX = MAXG;
    int           n;
    int64_t       chunk0[MAXG + 1];
    PushArgsMixed g[MAXG];
};

template <int MAXG>
__device__ __forceinline__ int group_of(PushGroupsMixed<MAXG> const &G, int64_t chunk, int from)
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

// direct atomics for a stencil outside the window
template <int O>
__device__ __forceinline__ void deposit_direct(PushArgsMixed const &a, int d, ShapeF<O> const &sh, float4 vw)
{
    atomicAdd(a.fallbacks, 1ull);
#pragma unroll
    for (int j = 0; j <= O; ++j) {
        double *const p = a.dep[d][0] + sh.i0 + j;
        atomicAdd(p, static_cast<double>(vw.x * sh.w[j]));
        atomicAdd(a.dep[d][1] + sh.i0 + j, static_cast<double>(vw.y * sh.w[j]));
        atomicAdd(a.dep[d][2] + sh.i0 + j, static_cast<double>(vw.z * sh.w[j]));
        atomicAdd(a.dep[d][3] + sh.i0 + j, static_cast<double>(vw.w * sh.w[j]));
    }
}

template <int O, bool MIRROR, int BC, int MAXG, bool PSD = false, bool NVV = false>
__global__ void __launch_bounds__(PIPE_THREADS, PIPE_CTAS_PER_SM_MIXED)
    push_kernel_mixed(PushGroupsMixed<MAXG> const __grid_constant__ G)
{
    using Layout           = MixLayout<PSD, NVV>;
    constexpr int   STAGES = Layout::STAGES;
    constexpr int   SPAN   = MIX_W - 1 - O; // largest stencil base offset inside the window
    using Stage            = PipeStageMixedT<PSD>;
    extern __shared__ __align__(128) unsigned char smraw[];
    Stage          *stage = reinterpret_cast<Stage *>(smraw);
    uint64_t       *full  = reinterpret_cast<uint64_t *>(smraw + Layout::BAR_OFFSET);
    uint64_t       *empty = full + STAGES;
    int const       warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    int64_t const   nchunks = G.chunk0[G.n];
    int64_t const   per     = (nchunks + gridDim.x - 1) / gridDim.x;
    int64_t const   c0      = static_cast<int64_t>(blockIdx.x) * per;
    int64_t const   mine    = c0 < nchunks ? min(per, nchunks - c0) : 0;

    if (threadIdx.x == 0) {
        for (int s = 0; s < STAGES; ++s) {
            mbar_init(&full[s], 1);
            mbar_init(&empty[s], PIPE_CONSUMER_WARPS);
        }
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    __syncthreads();

    if (warp == PIPE_CONSUMER_WARPS) { // ---------------- producer ----------------
        if (lane == 0) {
            int gl = -1, gr = -1;
            int      s  = 0; // i % STAGES
            uint32_t ph = 0; // (i / STAGES) & 1; both kept incrementally, without a 64-bit division per chunk
            for (int64_t i = 0; i < mine + STAGES; ++i, s = s + 1 == STAGES ? 0 : s + 1, ph ^= s == 0 ? 1u : 0u) {
                if (i >= STAGES && i - STAGES < mine) {
                    int64_t const        j = i - STAGES;
                    gr                     = group_of(G, c0 + j, gr);
                    PushArgsMixed const &a = G.g[gr];
                    if (!mbar_wait(&empty[s], ph ^ 1u)) { // the phase of chunk j = i - STAGES
                        atomicOr(a.status, ST_TIMEOUT);
                        break;
                    }
                    if (a.write_back) {
                        int64_t const  start = (c0 + j - G.chunk0[gr]) * MIX_CHUNK;
                        uint32_t const cnt   = static_cast<uint32_t>(min(static_cast<int64_t>(MIX_CHUNK), a.n - start));
                        uint32_t const b4    = round16(cnt * 4);
                        bulk_store(a.pos + start, stage[s].pos, b4);
                        bulk_store(a.vx + start, stage[s].vx, b4);
                        bulk_store(a.vy + start, stage[s].vy, b4);
                        bulk_store(a.vz + start, stage[s].vz, b4);
                        if (BC == BCK_ABSORBING || PSD)
                            bulk_store(a.w + start, stage[s].w, b4);
                        if (PSD)
                            bulk_store(a.real_f + start, stage[s].real_f, b4);
                        bulk_commit();
                    }
                    bulk_wait_read_all();
                }
                if (i < mine) {
                    gl                     = group_of(G, c0 + i, gl);
                    PushArgsMixed const &a = G.g[gl];
                    bool const     lpid  = a.randomize != 0;
                    int64_t const  start = (c0 + i - G.chunk0[gl]) * MIX_CHUNK;
                    uint32_t const cnt   = static_cast<uint32_t>(min(static_cast<int64_t>(MIX_CHUNK), a.n - start));
                    uint32_t const b4    = round16(cnt * 4);
                    mbar_arrive_expect_tx(&full[s], (5 + (lpid ? 1 : 0) + (PSD ? 2 : 0)) * b4);
                    bulk_load(stage[s].pos, a.pos + start, b4, &full[s]);
                    bulk_load(stage[s].vx, a.vx + start, b4, &full[s]);
                    bulk_load(stage[s].vy, a.vy + start, b4, &full[s]);
                    bulk_load(stage[s].vz, a.vz + start, b4, &full[s]);
                    bulk_load(stage[s].w, a.w + start, b4, &full[s]);
                    if (lpid)
                        bulk_load(stage[s].pid, a.pid + start, b4, &full[s]);
                    if (PSD) {
                        bulk_load(stage[s].real_f, a.real_f + start, b4, &full[s]);
                        bulk_load(stage[s].marker, a.marker + start, b4, &full[s]);
                    }
                }
            }
            bulk_wait_all();
        }
        return;
    }

    // ---------------- consumers ----------------
    ColWindow win;
    win.col  = reinterpret_cast<float4 *>(smraw + Layout::COL_OFFSET) + warp * 2 * MIX_W * 32;
    NvvWindow nvw{};
    if constexpr (NVV) {
        unsigned char *const nb = smraw + Layout::COL_OFFSET + MIX_COL_BYTES;
        nvw.c4 = reinterpret_cast<float4 *>(nb) + warp * MIX_W * 32;
        nvw.c2 = reinterpret_cast<float2 *>(nb + sizeof(float4) * PIPE_CONSUMER_WARPS * MIX_W * 32) + warp * MIX_W * 32;
        nvw.zero(lane);
    }
    win.base = ColWindow::NONE;
    win.zero(lane);
    unsigned bad = 0;
    int      gc  = -1;
    int      s  = 0; // i % STAGES
    uint32_t ph = 0; // (i / STAGES) & 1
    for (int64_t i = 0; i < mine; ++i, s = s + 1 == STAGES ? 0 : s + 1, ph ^= s == 0 ? 1u : 0u) {
        int const gi = group_of(G, c0 + i, gc);
        if (gi != gc) { // entering the next group: settle the previous group's window and status
            if (gc >= 0) {
                PushArgsMixed const &ap = G.g[gc];
                win.flush(lane, ap);
                if constexpr (NVV)
                    nvw.flush(win.base, lane, ap);
                bad = __reduce_or_sync(0xffffffffu, bad);
                if (bad && lane == 0)
                    atomicOr(ap.status, bad);
                bad = 0;
            }
            win.base = ColWindow::NONE;
            gc       = gi;
        }
        PushArgsMixed const &a        = G.g[gc];
        bool const           load_pid = a.randomize != 0;
        if (!mbar_wait(&full[s], ph)) {
            bad |= ST_TIMEOUT;
            break;
        }
        int64_t const   start = (c0 + i - G.chunk0[gc]) * MIX_CHUNK;
        int const       cnt   = static_cast<int>(min(static_cast<int64_t>(MIX_CHUNK), a.n - start));
        Stage          &P     = stage[s];
        int const       w0    = warp * 32 * MIX_PPT;

        // The lane's two particles are adjacent (i2, i2 + 1) and pushed as a pair on the packed
        // FP32 pipe (one f32x2 instruction per operation of both); then one window check covers
        // all their deposits.
        int const  i2      = w0 + 2 * lane;
        bool const live[2] = { i2 < cnt, i2 + 1 < cnt }; // slots past cnt hold stale data: pushed, never stored or deposited
        int2 const x_in    = *reinterpret_cast<int2 const *>(P.pos + i2);
        int32_t    X[2]    = { x_in.x, x_in.y };
        int32_t const half = int32_t{ 1 } << (a.fbits - 1); // a removed particle: cell 0, offset 1/2
        p3         v       = { *reinterpret_cast<float2 const *>(P.vx + i2), *reinterpret_cast<float2 const *>(P.vy + i2),
                               *reinterpret_cast<float2 const *>(P.vz + i2) };
        float2       w    = *reinterpret_cast<float2 const *>(P.w + i2);
        float2       w_in = w;
        int2 const   pid  = load_pid ? *reinterpret_cast<int2 const *>(P.pid + i2) : make_int2(0, 0);
        bool         alive[2] = { true, true };
        if (a.move_steps == 2) { // predictor-corrector: half move and boundary before the push
#pragma unroll
            for (int k = 0; k < 2; ++k) {
                float dq = a.inv_D1 * el(v.x, k) * (0.5f * a.dt);
                if constexpr (MIRROR) {
                    float s_, c_;
                    sincos_taylor_f(a.xiD1 * (static_cast<float>(pos_cell(X[k], a.fbits)) + a.full_min
                                              + pos_off(X[k], a.fbits, a.inv_scale)),
                                    s_, c_);
                    dq *= c_ * c_;
                }
                if (live[k] && !(fabsf(dq * a.travel_scale) < 1.0f))
                    bad |= ST_MOVED_TOO_FAR;
                f3 vk = { el(v.x, k), el(v.y, k), el(v.z, k) };
                move_pos(X[k], dq, a.scale);
                alive[k] = boundary_mixed<BC>(a, X[k], vk, k ? pid.y : pid.x, a.counter);
                if (!alive[k])
                    el(w, k) = 0.0f, X[k] = half, vk = { 0, 0, 0 };
                el(v.x, k) = vk.x, el(v.y, k) = vk.y, el(v.z, k) = vk.z;
            }
        }
        ShapeF<O> ds0[2], ds1[2];
        bool      in0[2], push[2];
        p3        E = { { 0, 0 }, { 0, 0 }, { 0, 0 } }, dB = E;
        int       cell[2];
        float2    off;
#pragma unroll
        for (int k = 0; k < 2; ++k) { // E and dB at the particles, each into its half of the pairs
            if constexpr (MIRROR) // the position itself, for the background field
                cell[k] = pos_cell(X[k], a.fbits), el(off, k) = pos_off(X[k], a.fbits, a.inv_scale);
            ds0[k] = make_shape_fx<O>(X[k], a.fbits, a.inv_scale);
            in0[k]  = stencil_ok_f(ds0[k], a.Nx);
            push[k] = in0[k] && alive[k] && a.move_steps != 0;
            if (!in0[k] && live[k])
                bad |= ST_OUT_OF_RANGE;
            // a particle that is not pushed reads the records of cells 0..O instead of its own (its
            // velocity is not updated below), so the loads need no branch
            int const ib = push[k] ? ds0[k].i0 : 0;
#pragma unroll
            for (int j = 0; j <= O; ++j) {
                float const *q  = a.EB + EBF_STRIDE * (ib + j);
                float4 const x0 = __ldg(reinterpret_cast<float4 const *>(q));
                float4 const x1 = __ldg(reinterpret_cast<float4 const *>(q + 4));
                float const  wj = ds0[k].w[j];
                el(E.x, k) += x0.x * wj, el(E.y, k) += x0.y * wj, el(E.z, k) += x0.z * wj;
                el(dB.x, k) += x0.w * wj, el(dB.y, k) += x1.x * wj, el(dB.z, k) += x1.y * wj;
            }
        }
        // the Boris push of both particles (as in boris_push, device_common.cuh)
        float2 c2 = { 1.0f, 1.0f };
        p3     B;
        if constexpr (MIRROR) { // background field, as in background_B (particles.cuh)
            float2 const x = { a.xiD1 * (static_cast<float>(cell[0]) + a.full_min + off.x),
                               a.xiD1 * (static_cast<float>(cell[1]) + a.full_min + off.y) };
            float2       s_, c_;
            sincos_taylor_f2(x, s_, c_);
            c2               = pmul(c_, c_);
            float2 const ksc = pmul(bc(a.xiO0_Oc), pmul(s_, c_));
            B                = { { __fdividef(a.O0, c2.x), __fdividef(a.O0, c2.y) }, pmul(ksc, v.z), pneg(pmul(ksc, v.y)) };
        } else {
            B = { bc(a.O0), { 0.0f, 0.0f }, { 0.0f, 0.0f } };
        }
        float2 const hB = bc(a.dtOc_2O0), hE = bc(a.cDtOc_2O0);
        B               = { pmul(padd(B.x, dB.x), hB), pmul(padd(B.y, dB.y), hB), pmul(padd(B.z, dB.z), hB) };
        E               = { pmul(E.x, hE), pmul(E.y, hE), pmul(E.z, hE) };
        p3 const vm     = { padd(v.x, E.x), padd(v.y, E.y), padd(v.z, E.z) };
        p3 const u      = padd3(vm, pcross(vm, B));
        float2 const d  = pfma(B.x, B.x, pfma(B.y, B.y, pfma(B.z, B.z, bc(1.0f))));
        float2 const sb = { __fdividef(2.0f, d.x), __fdividef(2.0f, d.y) };
        p3 const     Bs = { pmul(B.x, sb), pmul(B.y, sb), pmul(B.z, sb) };
        p3 const     vp = padd3(padd3(vm, pcross(u, Bs)), E);
        float2 const dq = pmul(pmul(bc(a.inv_D1), c2), pmul(vp.x, bc(a.move_steps == 2 ? 0.5f * a.dt : a.dt)));
        p3           v_push = v;
        float4       dv0[2], dv1[2];
        bool         dd0[2], dd1[2];
#pragma unroll
        for (int k = 0; k < 2; ++k) {
            if (push[k]) {
                if (live[k] && !(fabsf(el(dq, k) * a.travel_scale) < 1.0f))
                    bad |= ST_MOVED_TOO_FAR;
                f3 vk      = { el(vp.x, k), el(vp.y, k), el(vp.z, k) };
                if constexpr (PSD) { // the weight at the new velocity and the push position
                    float rf       = P.real_f[i2 + k];
                    el(w, k)       = update_weight_f(a, vk, el(c2, k), rf, P.marker[i2 + k]);
                    el(w_in, k)    = el(w, k);
                    P.real_f[i2 + k] = rf;
                }
                el(v_push.x, k) = vk.x, el(v_push.y, k) = vk.y, el(v_push.z, k) = vk.z;
                move_pos(X[k], el(dq, k), a.scale);
                alive[k] = boundary_mixed<BC>(a, X[k], vk, k ? pid.y : pid.x, a.counter + (a.move_steps == 2 ? 1 : 0));
                if (!alive[k])
                    el(w, k) = 0.0f, X[k] = half, vk = { 0, 0, 0 };
                el(v.x, k) = vk.x, el(v.y, k) = vk.y, el(v.z, k) = vk.z;
            }
            ds1[k] = make_shape_fx<O>(X[k], a.fbits, a.inv_scale);
            dd0[k] = live[k] && in0[k] && (a.deposit_mask & 1);
            dd1[k] = live[k] && (a.deposit_mask & 2) && el(w, k) != 0.0f && stencil_ok_f(ds1[k], a.Nx);
        }
        *reinterpret_cast<int2 *>(P.pos + i2)   = make_int2(X[0], X[1]);
        *reinterpret_cast<float2 *>(P.vx + i2)  = v.x;
        *reinterpret_cast<float2 *>(P.vy + i2)  = v.y;
        *reinterpret_cast<float2 *>(P.vz + i2)  = v.z;
        if (BC == BCK_ABSORBING || PSD)
            *reinterpret_cast<float2 *>(P.w + i2) = w;
        {
            p3 const m0 = { pmul(v_push.x, w_in), pmul(v_push.y, w_in), pmul(v_push.z, w_in) };
            p3 const m1 = { pmul(v.x, w), pmul(v.y, w), pmul(v.z, w) };
#pragma unroll
            for (int k = 0; k < 2; ++k) {
                dv0[k] = make_float4(el(w_in, k), el(m0.x, k), el(m0.y, k), el(m0.z, k));
                dv1[k] = make_float4(el(w, k), el(m1.x, k), el(m1.y, k), el(m1.z, k));
            }
        }
        {
            int lo = 0x7fffffff, hi = -0x7fffffff;
#pragma unroll
            for (int k = 0; k < 2; ++k) {
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
            auto nvv_terms = [&](int k, float (&t)[6]) {
                float const vx = el(v.x, k), vy = el(v.y, k), vz = el(v.z, k), wk = el(w, k);
                t[0] = (vx * vx) * wk, t[1] = (vy * vy) * wk, t[2] = (vz * vz) * wk;
                t[3] = (vx * vy) * wk, t[4] = (vy * vz) * wk, t[5] = (vz * vx) * wk;
            };
            if (all_in) { // the usual case: no check per deposit
#pragma unroll
                for (int k = 0; k < 2; ++k) {
                    if (dd0[k])
                        win.add<O>(0, ds0[k], dv0[k], lane);
                    if (dd1[k]) {
                        win.add<O>(1, ds1[k], dv1[k], lane);
                        if constexpr (NVV) {
                            float t[6];
                            nvv_terms(k, t);
                            nvw.add<O>(win.base, ds1[k], t, lane);
                        }
                    }
                }
            } else {
#pragma unroll
                for (int k = 0; k < 2; ++k) {
                    if (dd0[k]) {
                        if (ds0[k].i0 >= win.base && ds0[k].i0 <= win.base + SPAN)
                            win.add<O>(0, ds0[k], dv0[k], lane);
                        else
                            deposit_direct<O>(a, 0, ds0[k], dv0[k]);
                    }
                    if (dd1[k]) {
                        bool const inside = ds1[k].i0 >= win.base && ds1[k].i0 <= win.base + SPAN;
                        if (inside)
                            win.add<O>(1, ds1[k], dv1[k], lane);
                        else
                            deposit_direct<O>(a, 1, ds1[k], dv1[k]);
                        if constexpr (NVV) {
                            float t[6];
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
        PushArgsMixed const &a = G.g[gc];
        win.flush(lane, a);
        if constexpr (NVV)
            nvw.flush(win.base, lane, a);
        bad = __reduce_or_sync(0xffffffffu, bad);
        if (bad && lane == 0)
            atomicOr(a.status, bad);
    }
}

} // namespace h1d
