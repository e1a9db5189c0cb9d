// Stable LSD radix sort of the particles of one species by cell, written for this library.
//
// The reference keeps particles in a std::deque in load order and never sorts them; here the
// particles are kept cell-sorted so that a warp's particles share a few cells (coalesced field
// reads, register-window deposits).  The key of a particle is its full-grid cell
// floor(q1 - q1min) in [0, Nx) (ParamSet.cc:22); under the absorbing boundary, absorbed particles
// (weight 0) get key Nx and move to the end, where the host trims them (under the other
// boundaries a weight of 0 is an ordinary particle: a test particle, or a delta-f one).  Sorting is stable, so the order is reproducible
// and equals std::stable_sort by key on the host.
//
// Keys lie in [0, Nx], so ceil(log2(Nx + 1)) bits are sorted, in one pass (up to 8 bits) or two
// passes of about half the bits each.  Between sorts particles drift by a fraction of a cell to a
// few cells, so the keys arrive nearly sorted and a tile holds a few distinct digits:
//   hist_kernel      per-tile digit histograms, stored digit-major [radix][tiles]; each warp adds
//                    one count per distinct digit of 32 keys (__match_any_sync), so equal digits
//                    do not serialise on a shared-memory atomic
//   scan (3 kernels) exclusive prefix over the histogram matrix
//   scatter_kernel   stable rank within each tile: each warp ranks its own 256 contiguous keys
//                    (match groups, a per-warp running count per digit), one block-wide prefix
//                    over the warps' counts, then every item goes to its place
// The first pass reads the keys straight from the particles and counts absorbed particles; the
// last pass moves the particle records themselves (no separate index array and gather).  Each
// thread issues all of its loads before it ranks, so a warp keeps 8 loads in flight.
//
// One launch of each kernel sorts a whole set of particle segments -- the species of one run, or
// of every member of an ensemble -- each in its own buffers.  Segment g owns the tiles
// [tile0[g], tile0[g+1]) and the histogram rows [(radix) * tile0[g], (radix) * tile0[g+1]), so a
// single exclusive scan over the whole histogram yields each item's place in the concatenation of
// the sorted segments; subtracting first[g] (the particles of the earlier segments) gives its
// place in its own segment.  Sorting by (segment, key) this way costs the same launches for 64
// members as for one.
#pragma once

#include "device_common.cuh"

namespace h1d {

constexpr int SORT_THREADS = 256;
constexpr int SORT_ITEMS   = 8;
constexpr int SORT_TILE    = SORT_THREADS * SORT_ITEMS;
constexpr int SCAN_THREADS = 256;
constexpr int SCAN_ITEMS   = 16;
constexpr int SCAN_SEG     = SCAN_THREADS * SCAN_ITEMS;

// digit widths of the passes: keys in [0, Nx] need ceil(log2(Nx + 1)) bits (Nx <= 65535)
struct SortPlan {
    int passes, bits[2];
};
inline SortPlan sort_plan(int Nx)
{
    int nbits = 1;
    while ((1 << nbits) <= Nx)
        ++nbits;
    if (nbits <= 8)
        return {1, {nbits, 0}};
    return {2, {(nbits + 1) / 2, nbits / 2}};
}

// where a pass reads its keys: the key array of the previous pass, or (first pass) the particles
struct SortKeys {
    uint32_t const     *keys;   // KEYS_ARRAY
    double const       *q1, *w; // KEYS_FP64
    int32_t const      *pos;    // KEYS_MIXED: fixed-point positions with fbits fraction bits
    int                 fbits;
    float const        *wf;
    double              full_min;
    int                 Nx;
    int                 absorbing; // weight 0 marks a removed particle only under the absorbing BC
    unsigned long long *dead;   // absorbed particles, counted once by the first histogram
    unsigned           *status;
};
enum { KEYS_ARRAY = 0, KEYS_FP64 = 1, KEYS_MIXED = 2 };

// the segments of one launch set (kernel parameter; MAXS == 1 makes them launch constants)
template <int MAXS>
struct SortSegs {
    static constexpr int MAX = MAXS;
    int                  n;                // segments, none of them empty
    int                  tile0[MAXS + 1];  // first tile of each segment; tile0[n] = all tiles
    uint32_t             first[MAXS];      // particles of the earlier segments (sum < 2^32)
    uint32_t             count[MAXS];      // particles of each segment
    SortKeys             key[MAXS];
    uint32_t const      *idx_in[MAXS];     // KEYS_ARRAY passes: the particle index of each key
};

// the segment that owns tile t: the last g with tile0[g] <= t
template <int MAXS>
__device__ __forceinline__ int seg_of(SortSegs<MAXS> const &S, int t)
{
    if constexpr (MAXS == 1) {
        return 0;
    } else {
        int lo = 0, hi = S.n - 1;
        while (lo < hi) {
            int const mid = (lo + hi + 1) >> 1;
            if (S.tile0[mid] <= t)
                lo = mid;
            else
                hi = mid - 1;
        }
        return lo;
    }
}

// where the scatter of each segment writes
template <class Move, int MAXS>
struct MoveSegs {
    Move mv[MAXS];
};

template <int KIND> struct KeyRaw;
template <> struct KeyRaw<KEYS_ARRAY> {
    uint32_t k;
};
template <> struct KeyRaw<KEYS_FP64> {
    double q, w;
};
template <> struct KeyRaw<KEYS_MIXED> {
    int32_t c;
    float   w;
};

template <int KIND>
__device__ __forceinline__ KeyRaw<KIND> key_load(SortKeys const &s, int64_t i)
{
    if constexpr (KIND == KEYS_ARRAY)
        return {s.keys[i]};
    else if constexpr (KIND == KEYS_FP64) // the weight only marks absorbed particles
        return {s.q1[i], s.absorbing ? s.w[i] : 1.0};
    else
        return {s.pos[i] >> s.fbits, s.absorbing ? s.wf[i] : 1.0f};
}

// the key of a loaded item; with `account`, absorbed particles are counted and lost ones flagged
template <int KIND>
__device__ __forceinline__ uint32_t key_of(SortKeys const &s, KeyRaw<KIND> const &r, bool account)
{
    if constexpr (KIND == KEYS_ARRAY) {
        return r.k;
    } else {
        bool     dead, lost;
        uint32_t k;
        if constexpr (KIND == KEYS_FP64) {
            // a kept particle lies in q1min <= q1 <= q1max: the boundary pass (Delegate.cc:33-50,
            // 101-145) leaves q1 < q1max, except that its wrap or reflection can round to q1max
            // itself, which the reference deposits into the ghost cell and wraps on the next pass.
            // Such a particle, and one an ulp below q1max where q1 - q1min rounds up to Nx, sorts
            // into the last cell.
            double const f = floor(r.q - s.full_min);
            dead           = s.absorbing && r.w == 0.0;
            lost           = !(r.q >= s.full_min && r.q <= s.full_min + static_cast<double>(s.Nx));
            k = lost || f >= static_cast<double>(s.Nx) ? (f >= 0.0 ? static_cast<uint32_t>(s.Nx - 1) : 0u)
                                                       : static_cast<uint32_t>(f);
        } else {
            dead = s.absorbing && r.w == 0.0f;
            lost = r.c < 0 || r.c >= s.Nx;
            k    = lost ? (r.c < 0 ? 0u : static_cast<uint32_t>(s.Nx - 1)) : static_cast<uint32_t>(r.c);
        }
        if (dead)
            k = static_cast<uint32_t>(s.Nx);
        if (account) {
            if (dead)
                atomicAdd(s.dead, 1ull);
            else if (lost) // a lost particle stays in range and is flagged
                atomicOr(s.status, ST_OUT_OF_RANGE);
        }
        return k;
    }
}

// warp w of a tile owns items [w0, w0 + 256); round r of lane l is item w0 + 32 r + l, so the
// rounds visit the warp's items in index order
__device__ __forceinline__ int64_t sort_warp_base(int tile)
{
    return static_cast<int64_t>(tile) * SORT_TILE + (threadIdx.x >> 5) * 32 * SORT_ITEMS;
}

// hist[(mask + 1) * tile0[g] + digit * ntiles(g) + tile]: each segment's rows digit-major
template <int KIND, int MAXS>
__global__ void __launch_bounds__(SORT_THREADS)
    hist_kernel(SortSegs<MAXS> const __grid_constant__ S, int shift, unsigned mask, uint32_t *hist)
{
    __shared__ uint32_t h[256];
    h[threadIdx.x]          = 0;
    int const       g       = seg_of(S, static_cast<int>(blockIdx.x));
    int const       tile    = static_cast<int>(blockIdx.x) - S.tile0[g];
    int const       ntiles  = S.tile0[g + 1] - S.tile0[g];
    int64_t const   n       = S.count[g];
    SortKeys const &s       = S.key[g];
    int const       lane    = threadIdx.x & 31;
    int64_t const   w0      = sort_warp_base(tile);
    KeyRaw<KIND>  raw[SORT_ITEMS];
#pragma unroll
    for (int r = 0; r < SORT_ITEMS; ++r) {
        int64_t const i = w0 + r * 32 + lane;
        if (i < n)
            raw[r] = key_load<KIND>(s, i);
    }
    __syncthreads();
#pragma unroll
    for (int r = 0; r < SORT_ITEMS; ++r) {
        bool const     valid = w0 + r * 32 + lane < n;
        unsigned const digit = valid ? (key_of<KIND>(s, raw[r], true) >> shift) & mask : 256u + lane;
        unsigned const m     = __match_any_sync(0xffffffffu, digit);
        if (valid && lane == __ffs(m) - 1)
            atomicAdd(&h[digit], static_cast<uint32_t>(__popc(m)));
    }
    __syncthreads();
    if (threadIdx.x <= mask)
        hist[static_cast<int64_t>(mask + 1) * S.tile0[g] + static_cast<int64_t>(threadIdx.x) * ntiles + tile] =
            h[threadIdx.x];
}

// block-wide exclusive scan of one value per thread; returns the block total
__device__ __forceinline__ uint32_t block_exclusive_scan(uint32_t v, uint32_t *warp_tot, uint32_t &total)
{
    int const lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = blockDim.x >> 5;
    uint32_t  x    = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        uint32_t const y = __shfl_up_sync(0xffffffffu, x, o);
        if (lane >= o)
            x += y;
    }
    if (lane == 31)
        warp_tot[wid] = x;
    __syncthreads();
    if (wid == 0) {
        uint32_t s = lane < nw ? warp_tot[lane] : 0;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            uint32_t const y = __shfl_up_sync(0xffffffffu, s, o);
            if (lane >= o)
                s += y;
        }
        if (lane < nw)
            warp_tot[lane] = s; // inclusive
    }
    __syncthreads();
    total            = warp_tot[nw - 1];
    uint32_t const p = wid ? warp_tot[wid - 1] : 0;
    __syncthreads();
    return p + x - v;
}

__global__ void __launch_bounds__(SCAN_THREADS) scan_reduce_kernel(uint32_t const *in, int64_t len, uint32_t *part)
{
    __shared__ uint32_t s[SCAN_THREADS / 32];
    int64_t const       b   = static_cast<int64_t>(blockIdx.x) * SCAN_SEG;
    uint32_t            sum = 0;
    for (int k = 0; k < SCAN_ITEMS; ++k) {
        int64_t const i = b + k * SCAN_THREADS + threadIdx.x;
        if (i < len)
            sum += in[i];
    }
    for (int o = 16; o > 0; o >>= 1)
        sum += __shfl_xor_sync(0xffffffffu, sum, o);
    if ((threadIdx.x & 31) == 0)
        s[threadIdx.x >> 5] = sum;
    __syncthreads();
    if (threadIdx.x == 0) {
        uint32_t t = 0;
        for (int k = 0; k < SCAN_THREADS / 32; ++k)
            t += s[k];
        part[blockIdx.x] = t;
    }
}

// single block: exclusive scan of the per-segment partial sums (in place)
__global__ void __launch_bounds__(1024) scan_partials_kernel(uint32_t *part, int nparts)
{
    __shared__ uint32_t wt[32];
    uint32_t            carry = 0;
    for (int b = 0; b < nparts; b += blockDim.x) {
        int const      i = b + threadIdx.x;
        uint32_t const v = i < nparts ? part[i] : 0;
        uint32_t       total;
        uint32_t const e = block_exclusive_scan(v, wt, total);
        if (i < nparts)
            part[i] = carry + e;
        carry += total;
    }
}

__global__ void __launch_bounds__(SCAN_THREADS) scan_down_kernel(uint32_t *data, int64_t len, uint32_t const *part)
{
    __shared__ uint32_t wt[32];
    int64_t const       b = static_cast<int64_t>(blockIdx.x) * SCAN_SEG;
    // each thread owns SCAN_ITEMS consecutive elements
    uint32_t v[SCAN_ITEMS];
    uint32_t sum = 0;
#pragma unroll
    for (int k = 0; k < SCAN_ITEMS; ++k) {
        int64_t const i = b + static_cast<int64_t>(threadIdx.x) * SCAN_ITEMS + k;
        v[k]            = i < len ? data[i] : 0;
        sum += v[k];
    }
    uint32_t total;
    uint32_t run = block_exclusive_scan(sum, wt, total) + part[blockIdx.x];
#pragma unroll
    for (int k = 0; k < SCAN_ITEMS; ++k) {
        int64_t const i = b + static_cast<int64_t>(threadIdx.x) * SCAN_ITEMS + k;
        if (i < len)
            data[i] = run;
        run += v[k];
    }
}

// what the scatter of a pass writes: (key, index) pairs for the next pass ...
// HOLD: how many of a thread's records are loaded before the block-wide barrier (registers)
struct MoveKeys {
    static constexpr int HOLD = SORT_ITEMS;
    uint32_t            *keys_out, *idx_out;
    struct Rec {
        uint32_t key, id;
    };
    __device__ __forceinline__ Rec  load(uint32_t key, uint32_t id) const { return {key, id}; }
    __device__ __forceinline__ void store(uint32_t pos, Rec const &r) const
    {
        keys_out[pos] = r.key;
        idx_out[pos]  = r.id;
    }
};
// ... or, in the last pass, the FP64 particle records (q1, vx, vy, vz, w, pid; with PSD also
// real_f and marker)
template <bool PSD>
struct MoveFP64T {
    static constexpr int NV   = PSD ? 7 : 5;
    static constexpr int HOLD = SORT_ITEMS / 2;
    double const        *src[NV];
    int32_t const       *pid_src;
    double              *dst[NV];
    int32_t             *pid_dst;
    struct Rec {
        double  v[NV];
        int32_t pid;
    };
    __device__ __forceinline__ Rec load(uint32_t, uint32_t j) const
    {
        Rec r;
#pragma unroll
        for (int k = 0; k < NV; ++k)
            r.v[k] = src[k][j];
        r.pid = pid_src[j];
        return r;
    }
    __device__ __forceinline__ void store(uint32_t pos, Rec const &r) const
    {
#pragma unroll
        for (int k = 0; k < NV; ++k)
            dst[k][pos] = r.v[k];
        pid_dst[pos] = r.pid;
    }
};
using MoveFP64 = MoveFP64T<false>;
// ... or the mixed-precision records (vx, vy, vz, w as FP32, with PSD also real_f and marker;
// the fixed-point position, pid)
template <bool PSD>
struct MoveMixedT {
    static constexpr int NV   = PSD ? 6 : 4;
    static constexpr int HOLD = SORT_ITEMS / 2;
    float const         *src[NV];
    int32_t const       *pos_src, *pid_src;
    float               *dst[NV];
    int32_t             *pos_dst, *pid_dst;
    struct Rec {
        float   v[NV];
        int32_t pos, pid;
    };
    __device__ __forceinline__ Rec load(uint32_t, uint32_t j) const
    {
        Rec r;
#pragma unroll
        for (int k = 0; k < NV; ++k)
            r.v[k] = src[k][j];
        r.pos = pos_src[j];
        r.pid = pid_src[j];
        return r;
    }
    __device__ __forceinline__ void store(uint32_t pos, Rec const &r) const
    {
#pragma unroll
        for (int k = 0; k < NV; ++k)
            dst[k][pos] = r.v[k];
        pos_dst[pos] = r.pos;
        pid_dst[pos] = r.pid;
    }
};
using MoveMixed = MoveMixedT<false>;

template <int KIND, class Move, int MAXS>
__global__ void __launch_bounds__(SORT_THREADS)
    scatter_kernel(SortSegs<MAXS> const __grid_constant__ S, MoveSegs<Move, MAXS> const __grid_constant__ M,
                   int shift, unsigned mask, uint32_t const *offsets)
{
    constexpr int       NW = SORT_THREADS / 32;
    __shared__ uint32_t cnt[NW][256]; // per-warp digit counts, then each warp's start per digit
    int const           g      = seg_of(S, static_cast<int>(blockIdx.x));
    int const           tile   = static_cast<int>(blockIdx.x) - S.tile0[g];
    int const           ntiles = S.tile0[g + 1] - S.tile0[g];
    int64_t const       n      = S.count[g];
    SortKeys const     &s      = S.key[g];
    uint32_t const     *idx_in = S.idx_in[g];
    Move const         &mv     = M.mv[g];
    int const           lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    int64_t const       w0   = sort_warp_base(tile);
    unsigned const      lt   = (1u << lane) - 1u;
    KeyRaw<KIND>        raw[SORT_ITEMS];
    uint32_t            key[SORT_ITEMS], id[SORT_ITEMS], dig[SORT_ITEMS], rank[SORT_ITEMS];
#pragma unroll
    for (int r = 0; r < SORT_ITEMS; ++r) {
        int64_t const i = w0 + r * 32 + lane;
        id[r]           = static_cast<uint32_t>(i);
        if (i < n) {
            raw[r] = key_load<KIND>(s, i);
            if constexpr (KIND == KEYS_ARRAY)
                id[r] = idx_in[i];
        }
    }
#pragma unroll
    for (int j = 0; j < 8; ++j)
        cnt[wid][j * 32 + lane] = 0;
    __syncwarp();
#pragma unroll
    for (int r = 0; r < SORT_ITEMS; ++r) { // rank among the warp's earlier items of equal digit
        bool const valid    = w0 + r * 32 + lane < n;
        key[r]              = valid ? key_of<KIND>(s, raw[r], false) : 0u;
        dig[r]              = valid ? (key[r] >> shift) & mask : 256u + lane;
        unsigned const m    = __match_any_sync(0xffffffffu, dig[r]);
        int const      lead = __ffs(m) - 1;
        uint32_t       old  = 0;
        if (valid && lane == lead) {
            old              = cnt[wid][dig[r]];
            cnt[wid][dig[r]] = old + static_cast<uint32_t>(__popc(m));
        }
        rank[r] = __shfl_sync(0xffffffffu, old, lead) + static_cast<uint32_t>(__popc(m & lt));
        __syncwarp();
    }
    constexpr int      H = Move::HOLD;
    typename Move::Rec rec[H]; // records in flight while the block agrees on places
#pragma unroll
    for (int r = 0; r < H; ++r)
        if (w0 + r * 32 + lane < n)
            rec[r] = mv.load(key[r], id[r]);
    __syncthreads();
    if (threadIdx.x <= mask) { // digit threadIdx.x: the tile's start in its segment plus the earlier warps
        uint32_t run = offsets[static_cast<int64_t>(mask + 1) * S.tile0[g] + static_cast<int64_t>(threadIdx.x) * ntiles +
                               tile] -
                       S.first[g];
#pragma unroll
        for (int w = 0; w < NW; ++w) {
            uint32_t const c    = cnt[w][threadIdx.x];
            cnt[w][threadIdx.x] = run;
            run += c;
        }
    }
    __syncthreads();
#pragma unroll
    for (int r = 0; r < H; ++r)
        if (w0 + r * 32 + lane < n)
            mv.store(cnt[wid][dig[r]] + rank[r], rec[r]);
    if constexpr (H < SORT_ITEMS) {
        typename Move::Rec more[SORT_ITEMS - H];
#pragma unroll
        for (int r = H; r < SORT_ITEMS; ++r)
            if (w0 + r * 32 + lane < n)
                more[r - H] = mv.load(key[r], id[r]);
#pragma unroll
        for (int r = H; r < SORT_ITEMS; ++r)
            if (w0 + r * 32 + lane < n)
                mv.store(cnt[wid][dig[r]] + rank[r], more[r - H]);
    }
}

} // namespace h1d
