// Stable LSD radix sort of the particles of one species by cell, written for this library.
//
// The reference keeps particles in a std::deque in load order and never sorts them; here the
// particles are kept cell-sorted so that a warp's particles share a few cells (coalesced field
// reads, register-window deposits).  The key of a particle is its full-grid cell
// floor(q1 - q1min) in [0, Nx) (ParamSet.cc:22); absorbed particles (weight 0) get key Nx and
// move to the end, where the host trims them.  Sorting is stable, so the order is reproducible
// and equals std::stable_sort by key on the host.
//
// Passes of 8 bits over (key, index) pairs:
//   keys_kernel      key per particle, identity index
//   hist_kernel      per-tile digit histograms, stored digit-major [256][tiles]
//   scan (3 kernels) exclusive prefix over the histogram matrix
//   scatter_kernel   stable rank within each tile (warp match + per-warp digit counts), scatter
// then gather_kernel permutes the particle arrays by the sorted index.
#pragma once

#include "device_common.cuh"

namespace h1d {

constexpr int SORT_THREADS = 256;
constexpr int SORT_ITEMS   = 8;
constexpr int SORT_TILE    = SORT_THREADS * SORT_ITEMS;
constexpr int SCAN_THREADS = 256;
constexpr int SCAN_ITEMS   = 16;
constexpr int SCAN_SEG     = SCAN_THREADS * SCAN_ITEMS;

__global__ void keys_kernel(double const *q1, double const *w, int64_t n, double full_min, int Nx, uint32_t *keys,
                            uint32_t *idx, unsigned long long *dead, unsigned *status)
{
    int64_t const i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i >= n)
        return;
    double const q = q1[i];
    double const f = floor(q - full_min);
    uint32_t     k;
    if (w[i] == 0.0) {
        k = static_cast<uint32_t>(Nx);
        atomicAdd(dead, 1ull);
    } else if (!(f >= 0.0 && f < static_cast<double>(Nx))) {
        k = f >= 0.0 ? static_cast<uint32_t>(Nx - 1) : 0u; // lost particle: keep it in range, flag it
        atomicOr(status, ST_OUT_OF_RANGE);
    } else {
        k = static_cast<uint32_t>(f);
    }
    keys[i] = k;
    idx[i]  = static_cast<uint32_t>(i);
}

__global__ void __launch_bounds__(SORT_THREADS) hist_kernel(uint32_t const *keys, int64_t n, int shift, int ntiles,
                                                            uint32_t *hist)
{
    __shared__ uint32_t h[256];
    h[threadIdx.x] = 0;
    __syncthreads();
    int64_t const t0 = static_cast<int64_t>(blockIdx.x) * SORT_TILE;
#pragma unroll
    for (int k = 0; k < SORT_ITEMS; ++k) {
        int64_t const i = t0 + k * SORT_THREADS + threadIdx.x;
        if (i < n)
            atomicAdd(&h[(keys[i] >> shift) & 255u], 1u);
    }
    __syncthreads();
    hist[static_cast<int64_t>(threadIdx.x) * ntiles + blockIdx.x] = h[threadIdx.x];
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

__global__ void __launch_bounds__(SORT_THREADS) scatter_kernel(uint32_t const *keys_in, uint32_t const *idx_in,
                                                               int identity_idx, int64_t n, int shift, int ntiles,
                                                               uint32_t const *offsets, uint32_t *keys_out,
                                                               uint32_t *idx_out)
{
    constexpr int       NW = SORT_THREADS / 32;
    __shared__ uint32_t base[256];      // global offset of each digit for this tile + running count
    __shared__ uint32_t wcnt[NW][256];  // per-warp digit counts of the current round -> exclusive prefix
    int const           lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    base[threadIdx.x]        = offsets[static_cast<int64_t>(threadIdx.x) * ntiles + blockIdx.x];
    int64_t const t0         = static_cast<int64_t>(blockIdx.x) * SORT_TILE;
    for (int r = 0; r < SORT_ITEMS; ++r) {
#pragma unroll
        for (int w = 0; w < NW; ++w)
            wcnt[w][threadIdx.x] = 0;
        __syncthreads();
        int64_t const i     = t0 + r * SORT_THREADS + threadIdx.x;
        bool const    valid = i < n;
        uint32_t      key = 0, id = 0, digit = 256 + lane; // invalid lanes get unique non-digits
        if (valid) {
            key   = keys_in[i];
            id    = identity_idx ? static_cast<uint32_t>(i) : idx_in[i];
            digit = (key >> shift) & 255u;
        }
        unsigned const peers = __match_any_sync(0xffffffffu, digit);
        unsigned const rank  = __popc(peers & ((1u << lane) - 1u));
        if (valid && rank == 0)
            wcnt[wid][digit] = __popc(peers);
        __syncthreads();
        { // exclusive prefix over warps for digit threadIdx.x, and advance the running base
            uint32_t run = 0;
#pragma unroll
            for (int w = 0; w < NW; ++w) {
                uint32_t const c = wcnt[w][threadIdx.x];
                wcnt[w][threadIdx.x] = run;
                run += c;
            }
            __syncthreads();
            if (valid) {
                uint32_t const pos = base[digit] + wcnt[wid][digit] + rank;
                keys_out[pos]      = key;
                idx_out[pos]       = id;
            }
            __syncthreads();
            base[threadIdx.x] += run;
        }
    }
}

struct GatherArgs {
    double const  *src[5];
    int32_t const *pid_src;
    double        *dst[5];
    int32_t       *pid_dst;
    uint32_t const *idx;
    int64_t        n;
};
__global__ void gather_kernel(GatherArgs a)
{
    int64_t const i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i >= a.n)
        return;
    uint32_t const j = a.idx[i];
#pragma unroll
    for (int k = 0; k < 5; ++k)
        a.dst[k][i] = a.src[k][j];
    a.pid_dst[i] = a.pid_src[j];
}

} // namespace h1d
