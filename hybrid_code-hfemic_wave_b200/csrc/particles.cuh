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
#include "tma.cuh"

namespace h1d {

enum { BCK_PERIODIC = 0, BCK_REFLECTING = 1, BCK_ABSORBING = 2 };

struct PushArgs {
    double        *q1, *vx, *vy, *vz;
    double        *w; // writable only for absorption (w = 0 marks a removed particle)
    int32_t const *pid;
    int64_t        n;
    int            ppt; // particles per lane per warp-chunk
    int            Nx;
    double const  *EB; // per cell {Ex, Ey, Ez, dBx, dBy, dBz}: E and B averaged onto the half grid
                       // (PartSpecies.cc:132-139), pointer at interior cell 0
    double        *dep[2][4]; // [deposit at x^N | x^{N+1}][n, nVx, nVy, nVz], at cell 0
    double         half_min, full_min, full_max, full_len;
    double         xi, xi2, xiD1, D1, inv_D1, O0, Oc, dt, travel_scale, xiO0_Oc;
    BorisK         boris;
    unsigned      *status;
    unsigned long long *fallbacks; // deposits that missed the register window (diagnostic)
    uint64_t       seed, counter;
    int            species, randomize, homogeneous_poly;
    int            move_steps; // 1: CAM-CL full step; 2: PC half step, push, half step; 0: deposit only
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
template <int O, int S, int R>
__device__ __forceinline__ void deposit_at(Acc<O, S> &acc, Shape<O> const &sh, double const (&vw)[4])
{
#pragma unroll
    for (int j = 0; j <= O; ++j)
#pragma unroll
        for (int q = 0; q < 4; ++q)
            acc.v[q][R + j] = fma(vw[q], sh.w[j], acc.v[q][R + j]);
}
template <int O, int S, int D>
__device__ __forceinline__ void deposit(Acc<O, S> &acc, int base, Shape<O> const &sh, double w, d3 v,
                                        PushArgs const &a)
{
    constexpr int RW     = S - O - 1; // window offsets 0..RW
    double const  vw[4] = { w, v.x * w, v.y * w, v.z * w };
    int const     r     = sh.i0 - base;
    static_assert(RW >= 1 && RW <= 3, "window offsets 0..RW with RW in {1, 2, 3}");
    if (r == 0)
        deposit_at<O, S, 0>(acc, sh, vw);
    else if (r == 1)
        deposit_at<O, S, 1>(acc, sh, vw);
    else if (RW >= 2 && r == 2)
        deposit_at<O, S, (RW >= 2 ? 2 : 0)>(acc, sh, vw);
    else if (RW >= 3 && r == 3)
        deposit_at<O, S, (RW >= 3 ? 3 : 0)>(acc, sh, vw);
    else {
        atomicAdd(a.fallbacks, 1ull);
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

// background mirror field at the particle with its gyro-radius offset (PartSpecies.cc:274-279;
// MFABasis.h:287-290; MirrorGeometry.cc:199-212).  With c = cos(xi D1 q1), s = sin(xi D1 q1):
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
// The particle pass.  Warp-specialised pipeline per CTA: one producer warp streams chunks of
// PIPE_CHUNK particles global -> shared with 1-D TMA bulk copies completing on mbarriers
// (PIPE_STAGES deep) and bulk-stores the updated particles back; PIPE_CONSUMER_WARPS warps
// compute.  A consumer warp owns 32 x PIPE_PPT consecutive (cell-sorted) particles of a chunk and
// makes two passes over them in shared memory: (1) push at x^N, deposit at x^N, move, boundary,
// results written in place; (2) deposit at the new position.  Splitting the two deposits halves
// the register windows.
//
// One pass of a species: CAM-CL (move_steps == 1): push at x^N, deposit, move, BC, deposit.
// Predictor-corrector (move_steps == 2, Domain_PC.cc:110-124, 169-181): half move, BC, push at
// the half-step position, half move, BC, deposit.  move_steps == 0: deposit only
// (Domain_PC.cc:36-44).
// ------------------------------------------------------------------------------------------------
constexpr int PIPE_CONSUMER_WARPS = 4;
constexpr int PIPE_THREADS        = 32 * (PIPE_CONSUMER_WARPS + 1);
constexpr int PIPE_PPT            = 4;
constexpr int PIPE_CHUNK          = 32 * PIPE_CONSUMER_WARPS * PIPE_PPT;
constexpr int PIPE_STAGES         = 3;
constexpr int PIPE_CTAS_PER_SM    = 2;

struct PipeStage {
    double  q1[PIPE_CHUNK], vx[PIPE_CHUNK], vy[PIPE_CHUNK], vz[PIPE_CHUNK], w[PIPE_CHUNK];
    double  q1n[PIPE_CHUNK], wn[PIPE_CHUNK]; // position and weight after the move
    int32_t pid[PIPE_CHUNK];
};
constexpr size_t PIPE_SMEM = sizeof(PipeStage) * PIPE_STAGES + 2 * PIPE_STAGES * sizeof(uint64_t);

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

// add a warp's register window to the global moments: one atomic per (cell, quantity) and warp
template <int O, int S, int D>
__device__ __forceinline__ void flush_rs(Acc<O, S> const &acc, int base, int lane, PushArgs const &a)
{
    constexpr int V  = 4 * S <= 16 ? 16 : 32;
    constexpr int SH = V == 16 ? 1 : 0;
    static_assert(4 * S <= 32, "window too wide for one reduce-scatter");
    double x[V];
#pragma unroll
    for (int q = 0; q < 4; ++q)
#pragma unroll
        for (int s = 0; s < S; ++s)
            x[q * S + s] = acc.v[q][s];
#pragma unroll
    for (int k = 4 * S; k < V; ++k)
        x[k] = 0;
    double const v  = reduce_scatter<V>(x, lane);
    int const    vi = lane >> SH;
    if ((lane & SH) == 0 && vi < 4 * S && v != 0.0) {
        int const q = vi / S, cell = base + vi % S;
        if (cell >= -PAD && cell < a.Nx + PAD)
            atomicAdd(a.dep[D][q] + cell, v);
        else
            atomicOr(a.status, ST_OUT_OF_RANGE);
    }
}

// A warp's deposit window: register accumulators over cells [base, base + S), S = O + 1 + R,
// kept across batches and chunks.  When a batch of 32 particles reaches outside the window the
// warp flushes it and re-bases it at the batch minimum; particles of a batch that spans more than
// R + 1 stencil bases deposit with direct atomics.
template <int O, int R, int D>
struct Window {
    static constexpr int S    = O + 1 + R;
    static constexpr int NONE = -0x40000000;
    Acc<O, S> acc;
    int       base;

    __device__ __forceinline__ void init()
    {
        acc_zero(acc);
        base = NONE;
    }
    // batch step: i0 is this lane's stencil base (valid lanes only)
    __device__ __forceinline__ void prepare(bool valid, int i0, int lane, PushArgs const &a)
    {
        bool const outside = valid && (i0 > base + R || i0 < base);
        if (__any_sync(0xffffffffu, outside)) {
            if (base != NONE)
                flush_rs<O, S, D>(acc, base, lane, a);
            acc_zero(acc);
            base = __reduce_min_sync(0xffffffffu, valid ? i0 : 0x7fffffff);
        }
    }
    __device__ __forceinline__ void add(Shape<O> const &sh, double w, d3 v, PushArgs const &a)
    {
        deposit<O, S, D>(acc, base, sh, w, v, a);
    }
    __device__ __forceinline__ void finish(int lane, PushArgs const &a)
    {
        if (base != NONE)
            flush_rs<O, S, D>(acc, base, lane, a);
    }
};

// In-warp counting sort of a warp's 32 x PIPE_PPT slots of a chunk by stencil base cell, so that
// each batch of 32 particles handed to a deposit window spans as few cells as possible even after
// the particles have drifted since the last global sort.  Slot s = k * 32 + lane holds key[s]
// (INT_MAX for a slot that deposits nothing); order[] receives the slots in key order, stable in
// (k, lane).  Keys that span more than 31 cells keep the slot order.  Ranks come from
// __match_any_sync groups whose leaders update a per-warp histogram, so the order is
// deterministic.
struct WarpOrder {
    int      key[32 * PIPE_PPT];
    uint16_t order[32 * PIPE_PPT];
    int      hist[32];
};

__device__ __forceinline__ void warp_order(WarpOrder &W, int lane)
{
    constexpr unsigned FULL = 0xffffffffu;
    constexpr int      NONE = 0x7fffffff;
    int                kk[PIPE_PPT];
    int                lo = NONE, hi = -NONE;
#pragma unroll
    for (int k = 0; k < PIPE_PPT; ++k) {
        kk[k] = W.key[k * 32 + lane];
        if (kk[k] != NONE)
            lo = min(lo, kk[k]), hi = max(hi, kk[k]);
    }
    lo = __reduce_min_sync(FULL, lo);
    hi = __reduce_max_sync(FULL, hi);
    if (lo == NONE || hi - lo > 30) {
#pragma unroll
        for (int k = 0; k < PIPE_PPT; ++k)
            W.order[k * 32 + lane] = static_cast<uint16_t>(k * 32 + lane);
        __syncwarp();
        return;
    }
    W.hist[lane] = 0;
    __syncwarp();
    unsigned const lt = (1u << lane) - 1u;
    int            rank[PIPE_PPT], bin[PIPE_PPT];
#pragma unroll
    for (int k = 0; k < PIPE_PPT; ++k) {
        int const      b      = kk[k] == NONE ? 31 : kk[k] - lo;
        unsigned const m      = __match_any_sync(FULL, b);
        int const      leader = __ffs(m) - 1;
        int            old    = 0;
        if (lane == leader) {
            old       = W.hist[b];
            W.hist[b] = old + __popc(m);
        }
        old     = __shfl_sync(FULL, old, leader);
        rank[k] = old + __popc(m & lt);
        bin[k]  = b;
        __syncwarp();
    }
    int const c   = W.hist[lane];
    int       inc = c;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        int const y = __shfl_up_sync(FULL, inc, o);
        if (lane >= o)
            inc += y;
    }
    __syncwarp();
    W.hist[lane] = inc - c; // exclusive start of each bin
    __syncwarp();
#pragma unroll
    for (int k = 0; k < PIPE_PPT; ++k)
        W.order[W.hist[bin[k]] + rank[k]] = static_cast<uint16_t>(k * 32 + lane);
    __syncwarp();
}

// ------------------------------------------------------------------------------------------------
// The particle pass.  Warp-specialised pipeline per CTA: one producer warp streams the CTA's
// contiguous run of chunks (PIPE_CHUNK particles each) global -> shared with 1-D TMA bulk copies
// completing on mbarriers (PIPE_STAGES deep) and bulk-stores the updated particles back;
// PIPE_CONSUMER_WARPS warps compute.  A consumer warp owns 32 x PIPE_PPT consecutive
// (cell-sorted) particles of each chunk and makes passes over them in shared memory: (A) push at
// x^N, move, boundary, results written beside the inputs; then, in the cell order of warp_order,
// (B) deposit at x^N and (C) deposit at the new position.  Its two deposit windows persist
// across the chunks of the run.
//
// CAM-CL (move_steps == 1): push at x^N, deposit, move, BC, deposit.
// Predictor-corrector (move_steps == 2, Domain_PC.cc:110-124, 169-181): half move, BC, push at
// the half-step position, half move, BC, deposit.  move_steps == 0: deposit only
// (Domain_PC.cc:36-44).
// ------------------------------------------------------------------------------------------------
// The groups of particles one launch of the pass covers: a run's species (one group per launch)
// or the species of many runs of an ensemble (up to MAXG per launch).  The launch's chunks are
// numbered consecutively over the groups; a CTA takes a contiguous range of them, and its warps
// flush their deposit windows and status bits whenever the range crosses into the next group.
// The table travels as the kernel's parameter block (at most 32 KB).
template <int MAXG>
struct PushGroups {
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

template <int O, bool MIRROR, int BC, int MAXG>
__global__ void __launch_bounds__(PIPE_THREADS, PIPE_CTAS_PER_SM) push_kernel(PushGroups<MAXG> const __grid_constant__ G)
{
    constexpr int R = 2;
    extern __shared__ __align__(128) unsigned char smraw[];
    __shared__ WarpOrder worder[PIPE_CONSUMER_WARPS];
    PipeStage    *stage = reinterpret_cast<PipeStage *>(smraw);
    uint64_t     *full  = reinterpret_cast<uint64_t *>(smraw + sizeof(PipeStage) * PIPE_STAGES);
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
            for (int64_t i = 0; i < mine + PIPE_STAGES; ++i) {
                int const s = static_cast<int>(i % PIPE_STAGES);
                if (i >= PIPE_STAGES && i - PIPE_STAGES < mine) { // retire the chunk held by stage s
                    int64_t const   j = i - PIPE_STAGES;
                    gr                = group_of(G, c0 + j, gr);
                    PushArgs const &a = G.g[gr];
                    if (!mbar_wait(&empty[s], static_cast<uint32_t>((j / PIPE_STAGES) & 1))) {
                        atomicOr(a.status, ST_TIMEOUT);
                        break;
                    }
                    if (a.write_back) {
                        int64_t const  start = (c0 + j - G.chunk0[gr]) * PIPE_CHUNK;
                        uint32_t const cnt   = static_cast<uint32_t>(min(static_cast<int64_t>(PIPE_CHUNK), a.n - start));
                        uint32_t const b8    = round16(cnt * 8);
                        bulk_store(a.q1 + start, stage[s].q1n, b8);
                        bulk_store(a.vx + start, stage[s].vx, b8);
                        bulk_store(a.vy + start, stage[s].vy, b8);
                        bulk_store(a.vz + start, stage[s].vz, b8);
                        if (BC == BCK_ABSORBING)
                            bulk_store(a.w + start, stage[s].wn, b8);
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
                    mbar_arrive_expect_tx(&full[s], 5 * b8 + (lpid ? b4 : 0));
                    bulk_load(stage[s].q1, a.q1 + start, b8, &full[s]);
                    bulk_load(stage[s].vx, a.vx + start, b8, &full[s]);
                    bulk_load(stage[s].vy, a.vy + start, b8, &full[s]);
                    bulk_load(stage[s].vz, a.vz + start, b8, &full[s]);
                    bulk_load(stage[s].w, a.w + start, b8, &full[s]);
                    if (lpid)
                        bulk_load(stage[s].pid, a.pid + start, b4, &full[s]);
                }
            }
            bulk_wait_all();
        }
        return;
    }

    // ---------------- consumers ----------------
    unsigned        bad = 0;
    int             gc  = -1; // current group
    Window<O, R, 0> win0;
    Window<O, R, 1> win1;
    win0.init();
    win1.init();
    for (int64_t i = 0; i < mine; ++i) {
        int const s  = static_cast<int>(i % PIPE_STAGES);
        int const gi = group_of(G, c0 + i, gc);
        if (gi != gc) { // entering the next group: settle the previous group's windows and status
            if (gc >= 0) {
                PushArgs const &ap = G.g[gc];
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
        PushArgs const &a        = G.g[gc];
        bool const      load_pid = a.randomize != 0;
        if (!mbar_wait(&full[s], static_cast<uint32_t>((i / PIPE_STAGES) & 1))) {
            bad |= ST_TIMEOUT;
            break;
        }
        int64_t const start = (c0 + i - G.chunk0[gc]) * PIPE_CHUNK;
        int const     cnt   = static_cast<int>(min(static_cast<int64_t>(PIPE_CHUNK), a.n - start));
        PipeStage    &P     = stage[s];
        int const     w0    = warp * 32 * PIPE_PPT;
        // pass A: push at x^N (half steps around it for PC), move, boundary; no warp collectives,
        // so the compiler interleaves the independent particles of a lane.  Slots past `cnt` hold
        // stale finite data and are processed but never deposited or stored.
#pragma unroll 2
        for (int k = 0; k < PIPE_PPT; ++k) {
            int const idx   = w0 + k * 32 + lane;
            double    q1    = P.q1[idx];
            d3        v     = { P.vx[idx], P.vy[idx], P.vz[idx] };
            double    w     = P.w[idx];
            int32_t   pid   = load_pid ? P.pid[idx] : 0;
            bool      alive = true;
            if (a.move_steps == 2) {
                double const moved = move<MIRROR>(a, q1, v.x, 0.5 * a.dt);
                if (idx < cnt && !(fabs(moved) < 1.0)) // long(moved * scale) != 0 (PartSpecies.cc:261)
                    bad |= ST_MOVED_TOO_FAR;
                alive = boundary<BC>(a, q1, v, pid, a.counter);
                if (!alive)
                    w = 0, q1 = a.full_min + 0.5, v = { 0, 0, 0 };
                P.q1[idx] = q1; // PC deposits nothing at the push position
            }
            Shape<O> const sh = make_shape<O>(q1 - a.half_min);
            bool const     in_grid = finite_pos(q1) && stencil_ok(sh, a.Nx);
            worder[warp].key[k * 32 + lane] = in_grid && idx < cnt ? sh.i0 : 0x7fffffff;
            if (in_grid) {
                if (alive && a.move_steps != 0) {
                    d3 E, dB;
                    interp_EB<O>(a.EB, sh, E, dB);
                    double   c2;
                    d3 const B = background_B<MIRROR>(a, q1, v, c2) + dB;
                    v          = boris_push(a.boris, v, B, E);
                    // contravariant q1-velocity v_x cos^2 / D1 at the position of the push (CurviBasis.h:65-69)
                    double moved = (a.inv_D1 * c2) * v.x * (a.move_steps == 2 ? 0.5 * a.dt : a.dt);
                    q1 += moved;
                    moved *= a.travel_scale;
                    if (idx < cnt && !(fabs(moved) < 1.0))
                        bad |= ST_MOVED_TOO_FAR;
                    d3 const v_push = v;
                    alive = boundary<BC>(a, q1, v, pid, a.counter + (a.move_steps == 2 ? 1 : 0));
                    if (!alive)
                        w = 0, q1 = a.full_min + 0.5, v = { 0, 0, 0 };
                    // the deposit at x^N uses the velocity before the boundary pass: a particle the
                    // boundary reflected or removed deposits it here and is skipped by pass B
                    if ((a.deposit_mask & 1) && (v.x != v_push.x || v.y != v_push.y || v.z != v_push.z)) {
                        if (idx < cnt) {
                            double const vw[4] = { P.w[idx], v_push.x * P.w[idx], v_push.y * P.w[idx], v_push.z * P.w[idx] };
#pragma unroll
                            for (int j = 0; j <= O; ++j)
#pragma unroll
                                for (int q = 0; q < 4; ++q)
                                    atomicAdd(a.dep[0][q] + sh.i0 + j, vw[q] * sh.w[j]);
                        }
                        P.q1[idx] = __longlong_as_double(0x7ff8000000000000LL);
                    }
                }
            } else if (idx < cnt) {
                bad |= ST_OUT_OF_RANGE;
            }
            P.q1n[idx] = q1;
            P.vx[idx]  = v.x;
            P.vy[idx]  = v.y;
            P.vz[idx]  = v.z;
            if (BC == BCK_ABSORBING)
                P.wn[idx] = w;
        }
        __syncwarp();
        warp_order(worder[warp], lane);
        // pass B: deposit at x^N with v^{N+1/2} (CAM-CL)
        if (a.deposit_mask & 1) {
#pragma unroll 1
            for (int k = 0; k < PIPE_PPT; ++k) {
                int const      idx   = w0 + worder[warp].order[k * 32 + lane];
                double const   q1    = P.q1[idx];
                Shape<O> const sh    = make_shape<O>(q1 - a.half_min);
                bool const     valid = idx < cnt && finite_pos(q1) && stencil_ok(sh, a.Nx);
                win0.prepare(valid, sh.i0, lane, a);
                if (valid)
                    win0.add(sh, P.w[idx], d3{ P.vx[idx], P.vy[idx], P.vz[idx] }, a);
            }
        }
        // pass C: deposit at the end position
        if (a.deposit_mask & 2) {
#pragma unroll 1
            for (int k = 0; k < PIPE_PPT; ++k) {
                int const      idx   = w0 + worder[warp].order[k * 32 + lane];
                double const   q1    = P.q1n[idx];
                Shape<O> const sh    = make_shape<O>(q1 - a.half_min);
                bool const     valid = idx < cnt && finite_pos(q1) && stencil_ok(sh, a.Nx);
                win1.prepare(valid, sh.i0, lane, a);
                if (valid)
                    win1.add(sh, BC == BCK_ABSORBING ? P.wn[idx] : P.w[idx], d3{ P.vx[idx], P.vy[idx], P.vz[idx] }, a);
            }
        }
        fence_proxy_async_smem();
        __syncwarp();
        if (lane == 0)
            mbar_arrive(&empty[s]);
    }
    if (gc >= 0) {
        PushArgs const &a = G.g[gc];
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
