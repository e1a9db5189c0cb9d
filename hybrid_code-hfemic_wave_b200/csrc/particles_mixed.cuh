// Mixed-precision particle pass: the same cycle as push_kernel (particles.cuh) with
//   - position as an int32 full-grid cell plus an FP32 offset in [0, 1), so the shape weights
//     come from the in-cell offset and keep ~1e-7 cell resolution anywhere on the grid;
//   - FP32 velocity, weight, field interpolation, mirror geometry and Boris push;
//   - FP32 per-warp deposit windows, summed into the FP64 moment arrays per cell.
// The field cycle that consumes the moments stays FP64.  Traffic: read cell, offset, v, w
// (24 B), write cell, offset, v (20 B) per particle-step.
#pragma once

#include "particles.cuh"

namespace h1d {

struct PushArgsMixed {
    int32_t     *cell;
    float       *off, *vx, *vy, *vz, *w;
    int32_t const *pid;
    int64_t      n;
    int          Nx;
    float const *EB; // per cell {Ex, Ey, Ez, dBx, dBy, dBz} in FP32, pointer at interior cell 0
    double      *dep[2][4];
    float        full_min, xiD1, inv_D1, O0, dt, travel_scale, xiO0_Oc, dtOc_2O0, cDtOc_2O0;
    unsigned    *status;
    unsigned long long *fallbacks;
    uint64_t     seed, counter;
    int          species, randomize;
    int          move_steps, deposit_mask, write_back;
};

struct f3 {
    float x, y, z;
};
__device__ __forceinline__ f3 operator+(f3 a, f3 b) { return { a.x + b.x, a.y + b.y, a.z + b.z }; }
__device__ __forceinline__ f3 operator*(f3 a, float s) { return { a.x * s, a.y * s, a.z * s }; }
__device__ __forceinline__ f3 crossf(f3 A, f3 B) { return { A.y * B.z - A.z * B.y, A.z * B.x - A.x * B.z, A.x * B.y - A.y * B.x }; }

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

template <int O, int S>
struct AccF {
    float v[4][S];
};

template <int O, int S, int R>
__device__ __forceinline__ void deposit_at_f(AccF<O, S> &acc, ShapeF<O> const &sh, float const (&vw)[4])
{
#pragma unroll
    for (int j = 0; j <= O; ++j)
#pragma unroll
        for (int q = 0; q < 4; ++q)
            acc.v[q][R + j] = fmaf(vw[q], sh.w[j], acc.v[q][R + j]);
}

template <int O, int R, int D>
struct WindowF {
    static constexpr int S    = O + 1 + R;
    static constexpr int NONE = -0x40000000;
    AccF<O, S> acc;
    int        base;

    __device__ __forceinline__ void zero()
    {
#pragma unroll
        for (int q = 0; q < 4; ++q)
#pragma unroll
            for (int s = 0; s < S; ++s)
                acc.v[q][s] = 0.0f;
    }
    __device__ __forceinline__ void init()
    {
        zero();
        base = NONE;
    }
    // FP32 reduce-scatter across the warp (recursive halving of V = 16 or 32 values, as
    // reduce_scatter in particles.cuh), then one FP64 atomic per (cell, quantity)
    __device__ __forceinline__ void flush(int lane, PushArgsMixed const &a)
    {
        constexpr int V  = 4 * S <= 16 ? 16 : 32;
        constexpr int SH = V == 16 ? 1 : 0;
        static_assert(4 * S <= 32, "window too wide");
        float x[V];
#pragma unroll
        for (int q = 0; q < 4; ++q)
#pragma unroll
            for (int s = 0; s < S; ++s)
                x[q * S + s] = acc.v[q][s];
#pragma unroll
        for (int k = 4 * S; k < V; ++k)
            x[k] = 0.0f;
#pragma unroll
        for (int h = V / 2, m = 16; h >= 1; h >>= 1, m >>= 1) {
            bool const up = (lane & m) != 0;
#pragma unroll
            for (int j = 0; j < h; ++j) {
                float const send = up ? x[j] : x[j + h];
                float const keep = up ? x[j + h] : x[j];
                x[j]             = keep + __shfl_xor_sync(0xffffffffu, send, m);
            }
        }
        float v = x[0];
        if constexpr (V == 16)
            v += __shfl_xor_sync(0xffffffffu, v, 1);
        int const vi = lane >> SH;
        if ((lane & SH) == 0 && vi < 4 * S && v != 0.0f) {
            int const q = vi / S, cell = base + vi % S;
            if (cell >= -PAD && cell < a.Nx + PAD)
                atomicAdd(a.dep[D][q] + cell, static_cast<double>(v));
            else
                atomicOr(a.status, ST_OUT_OF_RANGE);
        }
    }
    __device__ __forceinline__ void prepare(bool valid, int i0, int lane, PushArgsMixed const &a)
    {
        bool const outside = valid && (i0 > base + R || i0 < base);
        if (__any_sync(0xffffffffu, outside)) {
            if (base != NONE)
                flush(lane, a);
            zero();
            base = __reduce_min_sync(0xffffffffu, valid ? i0 : 0x7fffffff);
        }
    }
    __device__ __forceinline__ void add(ShapeF<O> const &sh, float w, f3 v, PushArgsMixed const &a)
    {
        float const vw[4] = { w, v.x * w, v.y * w, v.z * w };
        int const   r     = sh.i0 - base;
        if (r == 0)
            deposit_at_f<O, S, 0>(acc, sh, vw);
        else if (r == 1)
            deposit_at_f<O, S, 1>(acc, sh, vw);
        else if (R >= 2 && r == 2)
            deposit_at_f<O, S, (R >= 2 ? 2 : 0)>(acc, sh, vw);
        else if (R >= 3 && r == 3)
            deposit_at_f<O, S, (R >= 3 ? 3 : 0)>(acc, sh, vw);
        else {
            atomicAdd(a.fallbacks, 1ull);
#pragma unroll
            for (int j = 0; j <= O; ++j)
#pragma unroll
                for (int q = 0; q < 4; ++q)
                    atomicAdd(a.dep[D][q] + sh.i0 + j, static_cast<double>(vw[q] * sh.w[j]));
        }
    }
    __device__ __forceinline__ void finish(int lane, PushArgsMixed const &a)
    {
        if (base != NONE)
            flush(lane, a);
    }
};

// move by dq cells (|dq| < 1 is checked by the caller); returns the new (cell, off)
__device__ __forceinline__ void move_cell(int &cell, float &off, float dq)
{
    float o = off + dq;
    if (o >= 1.0f)
        cell += 1, o -= 1.0f;
    else if (o < 0.0f)
        cell -= 1, o += 1.0f;
    off = o < 1.0f ? o : 0.99999994f;
}

template <int BC>
__device__ __forceinline__ bool boundary_mixed(PushArgsMixed const &a, int &cell, float &off, f3 &v, int32_t pid,
                                               uint64_t counter)
{
    if constexpr (BC == BCK_PERIODIC) {
        if (cell < 0)
            cell += a.Nx;
        else if (cell >= a.Nx)
            cell -= a.Nx;
        return true;
    } else if constexpr (BC == BCK_REFLECTING) {
        bool const left = cell < 0, right = cell >= a.Nx;
        if (left || right) { // q1 -> 2 q1_boundary - q1 (Delegate.cc:199-228)
            if (left) {      // q1 - q1min = -1 + off -> 1 - off
                cell = off > 0.0f ? 0 : 1;
                off  = off > 0.0f ? 1.0f - off : 0.0f;
            } else { // q1 - q1min = Nx + off -> Nx - off
                cell = a.Nx - 1;
                off  = off > 0.0f ? 1.0f - off : 0.99999994f;
            }
            v.x = -v.x;
            if (a.randomize) {
                float s, c;
                sincosf(static_cast<float>(gyrophase(a.seed, counter, (uint64_t)a.species, (uint64_t)pid)), &s, &c);
                float const vy = v.y, vz = v.z;
                v.y = vy * c - vz * s;
                v.z = vy * s + vz * c;
            }
        }
        return true;
    } else {
        return cell >= 0 && cell < a.Nx;
    }
}

struct PipeStageMixed {
    int32_t cell[PIPE_CHUNK];
    float   off[PIPE_CHUNK], vx[PIPE_CHUNK], vy[PIPE_CHUNK], vz[PIPE_CHUNK], w[PIPE_CHUNK];
    int32_t celln[PIPE_CHUNK];
    float   offn[PIPE_CHUNK], wn[PIPE_CHUNK];
    int32_t pid[PIPE_CHUNK];
};
constexpr int    PIPE_STAGES_MIXED = 3;
constexpr int    PIPE_CTAS_PER_SM_MIXED = 3;
constexpr size_t PIPE_SMEM_MIXED   = sizeof(PipeStageMixed) * PIPE_STAGES_MIXED + 2 * PIPE_STAGES_MIXED * sizeof(uint64_t);

// the groups of one launch, as PushGroups in particles.cuh
template <int MAXG>
struct PushGroupsMixed {
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

template <int O, bool MIRROR, int BC, int MAXG>
__global__ void __launch_bounds__(PIPE_THREADS, PIPE_CTAS_PER_SM_MIXED)
    push_kernel_mixed(PushGroupsMixed<MAXG> const __grid_constant__ G)
{
    constexpr int   R      = 2;
    constexpr int   STAGES = PIPE_STAGES_MIXED;
    extern __shared__ __align__(128) unsigned char smraw[];
    __shared__ WarpOrder worder[PIPE_CONSUMER_WARPS];
    PipeStageMixed *stage = reinterpret_cast<PipeStageMixed *>(smraw);
    uint64_t       *full  = reinterpret_cast<uint64_t *>(smraw + sizeof(PipeStageMixed) * STAGES);
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
            for (int64_t i = 0; i < mine + STAGES; ++i) {
                int const s = static_cast<int>(i % STAGES);
                if (i >= STAGES && i - STAGES < mine) {
                    int64_t const        j = i - STAGES;
                    gr                     = group_of(G, c0 + j, gr);
                    PushArgsMixed const &a = G.g[gr];
                    if (!mbar_wait(&empty[s], static_cast<uint32_t>((j / STAGES) & 1))) {
                        atomicOr(a.status, ST_TIMEOUT);
                        break;
                    }
                    if (a.write_back) {
                        int64_t const  start = (c0 + j - G.chunk0[gr]) * PIPE_CHUNK;
                        uint32_t const cnt   = static_cast<uint32_t>(min(static_cast<int64_t>(PIPE_CHUNK), a.n - start));
                        uint32_t const b4    = round16(cnt * 4);
                        bulk_store(a.cell + start, stage[s].celln, b4);
                        bulk_store(a.off + start, stage[s].offn, b4);
                        bulk_store(a.vx + start, stage[s].vx, b4);
                        bulk_store(a.vy + start, stage[s].vy, b4);
                        bulk_store(a.vz + start, stage[s].vz, b4);
                        if (BC == BCK_ABSORBING)
                            bulk_store(a.w + start, stage[s].wn, b4);
                        bulk_commit();
                    }
                    bulk_wait_read_all();
                }
                if (i < mine) {
                    gl                     = group_of(G, c0 + i, gl);
                    PushArgsMixed const &a = G.g[gl];
                    bool const     lpid  = a.randomize != 0;
                    int64_t const  start = (c0 + i - G.chunk0[gl]) * PIPE_CHUNK;
                    uint32_t const cnt   = static_cast<uint32_t>(min(static_cast<int64_t>(PIPE_CHUNK), a.n - start));
                    uint32_t const b4    = round16(cnt * 4);
                    mbar_arrive_expect_tx(&full[s], (6 + (lpid ? 1 : 0)) * b4);
                    bulk_load(stage[s].cell, a.cell + start, b4, &full[s]);
                    bulk_load(stage[s].off, a.off + start, b4, &full[s]);
                    bulk_load(stage[s].vx, a.vx + start, b4, &full[s]);
                    bulk_load(stage[s].vy, a.vy + start, b4, &full[s]);
                    bulk_load(stage[s].vz, a.vz + start, b4, &full[s]);
                    bulk_load(stage[s].w, a.w + start, b4, &full[s]);
                    if (lpid)
                        bulk_load(stage[s].pid, a.pid + start, b4, &full[s]);
                }
            }
            bulk_wait_all();
        }
        return;
    }

    unsigned         bad = 0;
    int              gc  = -1;
    WindowF<O, R, 0> win0;
    WindowF<O, R, 1> win1;
    win0.init();
    win1.init();
    for (int64_t i = 0; i < mine; ++i) {
        int const s  = static_cast<int>(i % STAGES);
        int const gi = group_of(G, c0 + i, gc);
        if (gi != gc) {
            if (gc >= 0) {
                PushArgsMixed const &ap = G.g[gc];
                if (ap.deposit_mask & 1)
                    win0.finish(lane, ap);
                if (ap.deposit_mask & 2)
                    win1.finish(lane, ap);
                bad = __reduce_or_sync(0xffffffffu, bad);
                if (bad && lane == 0)
                    atomicOr(ap.status, bad);
                bad = 0;
                win0.init();
                win1.init();
            }
            gc = gi;
        }
        PushArgsMixed const &a        = G.g[gc];
        bool const           load_pid = a.randomize != 0;
        if (!mbar_wait(&full[s], static_cast<uint32_t>((i / STAGES) & 1))) {
            bad |= ST_TIMEOUT;
            break;
        }
        int64_t const   start = (c0 + i - G.chunk0[gc]) * PIPE_CHUNK;
        int const       cnt   = static_cast<int>(min(static_cast<int64_t>(PIPE_CHUNK), a.n - start));
        PipeStageMixed &P     = stage[s];
        int const       w0    = warp * 32 * PIPE_PPT;
        // pass A: push, move, boundary (FP32)
#pragma unroll 2
        for (int k = 0; k < PIPE_PPT; ++k) {
            int const idx   = w0 + k * 32 + lane;
            int       cell  = P.cell[idx];
            float     off   = P.off[idx];
            f3        v     = { P.vx[idx], P.vy[idx], P.vz[idx] };
            float     w     = P.w[idx];
            int32_t   pid   = load_pid ? P.pid[idx] : 0;
            bool      alive = true;
            if (a.move_steps == 2) {
                float dq = a.inv_D1 * v.x * (0.5f * a.dt);
                if constexpr (MIRROR) {
                    float s_, c_;
                    sincos_taylor_f(a.xiD1 * (static_cast<float>(cell) + a.full_min + off), s_, c_);
                    dq *= c_ * c_;
                }
                if (idx < cnt && !(fabsf(dq * a.travel_scale) < 1.0f))
                    bad |= ST_MOVED_TOO_FAR;
                move_cell(cell, off, dq);
                alive = boundary_mixed<BC>(a, cell, off, v, pid, a.counter);
                if (!alive)
                    w = 0.0f, cell = 0, off = 0.5f, v = { 0, 0, 0 };
                P.cell[idx] = cell, P.off[idx] = off;
            }
            ShapeF<O> const sh      = make_shape_f<O>(cell, off);
            bool const      in_grid = stencil_ok_f(sh, a.Nx);
            worder[warp].key[k * 32 + lane] = in_grid && idx < cnt ? sh.i0 : 0x7fffffff;
            if (in_grid) {
                if (alive && a.move_steps != 0) {
                    f3 E = { 0, 0, 0 }, dB = { 0, 0, 0 };
#pragma unroll
                    for (int j = 0; j <= O; ++j) {
                        float const *p  = a.EB + 6 * (sh.i0 + j);
                        float2 const x0 = __ldg(reinterpret_cast<float2 const *>(p));
                        float2 const x1 = __ldg(reinterpret_cast<float2 const *>(p + 2));
                        float2 const x2 = __ldg(reinterpret_cast<float2 const *>(p + 4));
                        float const  wj = sh.w[j];
                        E.x += x0.x * wj, E.y += x0.y * wj, E.z += x1.x * wj;
                        dB.x += x1.y * wj, dB.y += x2.x * wj, dB.z += x2.y * wj;
                    }
                    float c2 = 1.0f;
                    f3    B;
                    if constexpr (MIRROR) { // background field, as in background_B (particles.cuh)
                        float s_, c_;
                        sincos_taylor_f(a.xiD1 * (static_cast<float>(cell) + a.full_min + off), s_, c_);
                        c2              = c_ * c_;
                        float const ksc = a.xiO0_Oc * (s_ * c_);
                        B               = { a.O0 / c2, ksc * v.z, -ksc * v.y };
                    } else {
                        B = { a.O0, 0.0f, 0.0f };
                    }
                    B = (B + dB) * a.dtOc_2O0;
                    E = E * a.cDtOc_2O0;
                    v = v + E;
                    f3 const    u  = v + crossf(v, B);
                    float const sb = 2.0f * __frcp_rn(1.0f + (B.x * B.x + B.y * B.y + B.z * B.z));
                    v              = v + crossf(u, B * sb) + E;
                    float const dq = (a.inv_D1 * c2) * v.x * (a.move_steps == 2 ? 0.5f * a.dt : a.dt);
                    if (idx < cnt && !(fabsf(dq * a.travel_scale) < 1.0f))
                        bad |= ST_MOVED_TOO_FAR;
                    f3 const v_push = v;
                    move_cell(cell, off, dq);
                    alive = boundary_mixed<BC>(a, cell, off, v, pid, a.counter + (a.move_steps == 2 ? 1 : 0));
                    if (!alive)
                        w = 0.0f, cell = 0, off = 0.5f, v = { 0, 0, 0 };
                    if ((a.deposit_mask & 1) && (v.x != v_push.x || v.y != v_push.y || v.z != v_push.z)) {
                        if (idx < cnt) { // deposit at x^N with the pre-boundary velocity
                            float const wv    = P.w[idx];
                            float const vw[4] = { wv, v_push.x * wv, v_push.y * wv, v_push.z * wv };
#pragma unroll
                            for (int j = 0; j <= O; ++j)
#pragma unroll
                                for (int q = 0; q < 4; ++q)
                                    atomicAdd(a.dep[0][q] + sh.i0 + j, static_cast<double>(vw[q] * sh.w[j]));
                        }
                        P.cell[idx] = -0x40000000; // skipped by pass B
                    }
                }
            } else if (idx < cnt) {
                bad |= ST_OUT_OF_RANGE;
            }
            P.celln[idx] = cell;
            P.offn[idx]  = off;
            P.vx[idx]    = v.x;
            P.vy[idx]    = v.y;
            P.vz[idx]    = v.z;
            if (BC == BCK_ABSORBING)
                P.wn[idx] = w;
        }
        __syncwarp();
        warp_order(worder[warp], lane);
        if (a.deposit_mask & 1) {
#pragma unroll 1
            for (int k = 0; k < PIPE_PPT; ++k) {
                int const       idx   = w0 + worder[warp].order[k * 32 + lane];
                ShapeF<O> const sh    = make_shape_f<O>(P.cell[idx], P.off[idx]);
                bool const      valid = idx < cnt && stencil_ok_f(sh, a.Nx);
                win0.prepare(valid, sh.i0, lane, a);
                if (valid)
                    win0.add(sh, P.w[idx], f3{ P.vx[idx], P.vy[idx], P.vz[idx] }, a);
            }
        }
        if (a.deposit_mask & 2) {
#pragma unroll 1
            for (int k = 0; k < PIPE_PPT; ++k) {
                int const       idx   = w0 + worder[warp].order[k * 32 + lane];
                ShapeF<O> const sh    = make_shape_f<O>(P.celln[idx], P.offn[idx]);
                bool const      valid = idx < cnt && stencil_ok_f(sh, a.Nx);
                win1.prepare(valid, sh.i0, lane, a);
                if (valid)
                    win1.add(sh, BC == BCK_ABSORBING ? P.wn[idx] : P.w[idx], f3{ P.vx[idx], P.vy[idx], P.vz[idx] }, a);
            }
        }
        fence_proxy_async_smem();
        __syncwarp();
        if (lane == 0)
            mbar_arrive(&empty[s]);
    }
    if (gc >= 0) {
        PushArgsMixed const &a = G.g[gc];
        if (a.deposit_mask & 1)
            win0.finish(lane, a);
        if (a.deposit_mask & 2)
            win1.finish(lane, a);
        bad = __reduce_or_sync(0xffffffffu, bad);
        if (bad && lane == 0)
            atomicOr(a.status, bad);
    }
}


} // namespace h1d
