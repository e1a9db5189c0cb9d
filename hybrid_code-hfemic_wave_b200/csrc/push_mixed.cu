// Instantiations and launches of the mixed-precision particle pass (particles_mixed.cuh).
#include "push_launch.h"

#include <algorithm>
#include <memory>
#include <mutex>
#include <new>

namespace h1d {
namespace {

template <int O, bool M, int BC, int MAXG, bool PSD>
void pk(PushGroupsMixed<MAXG> const &G, dim3 g, cudaStream_t st)
{
    push_kernel_mixed<O, M, BC, MAXG, PSD><<<g, PIPE_THREADS, PSD ? PIPE_SMEM_MIXED_PSD : PIPE_SMEM_MIXED, st>>>(G);
}
template <int O, bool M, int BC, int MAXG, bool PSD>
cudaError_t pk_attr()
{
    return cudaFuncSetAttribute(push_kernel_mixed<O, M, BC, MAXG, PSD>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                static_cast<int>(PSD ? PIPE_SMEM_MIXED_PSD : PIPE_SMEM_MIXED));
}

// the CIC pass that also forms collect_all's second moments (NVV)
template <bool M, int BC>
void pk_nvv(PushGroupsMixed<1> const &G, dim3 g, cudaStream_t st)
{
    push_kernel_mixed<1, M, BC, 1, false, true><<<g, PIPE_THREADS, PIPE_SMEM_MIXED_NVV, st>>>(G);
}
template <bool M, int BC>
cudaError_t pk_nvv_attr()
{
    return cudaFuncSetAttribute(push_kernel_mixed<1, M, BC, 1, false, true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                static_cast<int>(PIPE_SMEM_MIXED_NVV));
}

template <int O, bool M, bool PSD, class GR>
void pk_bc(GR const &G, int bc, dim3 g, cudaStream_t st)
{
    if (bc == 0)
        pk<O, M, BCK_PERIODIC, GR::MAX, PSD>(G, g, st);
    else if (bc == 1)
        pk<O, M, BCK_REFLECTING, GR::MAX, PSD>(G, g, st);
    else
        pk<O, M, BCK_ABSORBING, GR::MAX, PSD>(G, g, st);
}
template <bool PSD = false, class GR>
void pk_dispatch(GR const &G, int order, bool mirror, int bc, dim3 g, cudaStream_t st)
{
    if (order == 1)
        mirror ? pk_bc<1, true, PSD>(G, bc, g, st) : pk_bc<1, false, PSD>(G, bc, g, st);
    else if (order == 2)
        mirror ? pk_bc<2, true, PSD>(G, bc, g, st) : pk_bc<2, false, PSD>(G, bc, g, st);
    else
        mirror ? pk_bc<3, true, PSD>(G, bc, g, st) : pk_bc<3, false, PSD>(G, bc, g, st);
}

template <int MAXG, bool PSD>
cudaError_t pk_attrs()
{
    cudaError_t e = cudaSuccess;
    auto        k = [&](cudaError_t x) {
        if (e == cudaSuccess)
            e = x;
    };
    k(pk_attr<1, false, 0, MAXG, PSD>()), k(pk_attr<1, false, 1, MAXG, PSD>()), k(pk_attr<1, false, 2, MAXG, PSD>());
    k(pk_attr<1, true, 0, MAXG, PSD>()), k(pk_attr<1, true, 1, MAXG, PSD>()), k(pk_attr<1, true, 2, MAXG, PSD>());
    k(pk_attr<2, false, 0, MAXG, PSD>()), k(pk_attr<2, false, 1, MAXG, PSD>()), k(pk_attr<2, false, 2, MAXG, PSD>());
    k(pk_attr<2, true, 0, MAXG, PSD>()), k(pk_attr<2, true, 1, MAXG, PSD>()), k(pk_attr<2, true, 2, MAXG, PSD>());
    k(pk_attr<3, false, 0, MAXG, PSD>()), k(pk_attr<3, false, 1, MAXG, PSD>()), k(pk_attr<3, false, 2, MAXG, PSD>());
    k(pk_attr<3, true, 0, MAXG, PSD>()), k(pk_attr<3, true, 1, MAXG, PSD>()), k(pk_attr<3, true, 2, MAXG, PSD>());
    return e;
}

cudaError_t set_smem_once()
{
    static std::mutex m;
    static bool       done[64] = {};
    int               dev      = 0;
    if (cudaGetDevice(&dev) != cudaSuccess)
        return cudaErrorNoDevice;
    std::lock_guard<std::mutex> lock(m);
    if (dev >= 0 && dev < 64 && done[dev])
        return cudaSuccess;
    cudaError_t e = pk_attrs<1, false>();
    if (e == cudaSuccess)
        e = pk_attrs<BATCH_GROUPS, false>();
    if (e == cudaSuccess)
        e = pk_attrs<1, true>();
    for (cudaError_t const x : { pk_nvv_attr<false, 0>(), pk_nvv_attr<false, 1>(), pk_nvv_attr<false, 2>(),
                                 pk_nvv_attr<true, 0>(), pk_nvv_attr<true, 1>(), pk_nvv_attr<true, 2>() })
        if (e == cudaSuccess)
            e = x;
    if (e == cudaSuccess && dev >= 0 && dev < 64)
        done[dev] = true;
    return e;
}

inline int64_t chunks_of(int64_t n) { return (n + MIX_CHUNK - 1) / MIX_CHUNK; }

template <class ArgsT, template <int> class GroupsT>
cudaError_t launch_groups(ArgsT const *args, int n, int order, bool mirror, int bc, int max_ctas, cudaStream_t st)
{
    int64_t total = 0;
    for (int i = 0; i < n; ++i)
        total += chunks_of(args[i].n);
    if (total == 0)
        return cudaSuccess;
    if (n == 1) { // the group's arguments become constants of the kernel
        GroupsT<1> G{};
        G.n = 1, G.chunk0[0] = 0, G.chunk0[1] = total, G.g[0] = args[0];
        pk_dispatch(G, order, mirror, bc, dim3(static_cast<unsigned>(std::min<int64_t>(total, max_ctas))), st);
        return cudaGetLastError();
    }
    std::unique_ptr<GroupsT<BATCH_GROUPS>> G(new (std::nothrow) GroupsT<BATCH_GROUPS>{});
    if (!G)
        return cudaErrorMemoryAllocation;
    for (int i0 = 0; i0 < n; i0 += BATCH_GROUPS) {
        int const m = std::min(BATCH_GROUPS, n - i0);
        int64_t   c = 0;
        G->n        = m;
        for (int i = 0; i < m; ++i)
            G->chunk0[i] = c, G->g[i] = args[i0 + i], c += chunks_of(args[i0 + i].n);
        G->chunk0[m] = c;
        if (c > 0)
            pk_dispatch(*G, order, mirror, bc, dim3(static_cast<unsigned>(std::min<int64_t>(c, max_ctas))), st);
        cudaError_t const e = cudaGetLastError();
        if (e != cudaSuccess)
            return e;
    }
    return cudaSuccess;
}

} // namespace
} // namespace h1d

namespace h1d {

cudaError_t set_push_smem_mixed() { return set_smem_once(); }

cudaError_t launch_push_groups(PushArgsMixed const *args, int n, int order, bool mirror, int bc, int max_ctas,
                               cudaStream_t st)
{
    return launch_groups<PushArgsMixed, PushGroupsMixed>(args, n, order, mirror, bc, max_ctas, st);
}

cudaError_t launch_push_psd(PushArgsMixed const &a, int order, bool mirror, int bc, int max_ctas, cudaStream_t st)
{
    int64_t const total = chunks_of(a.n);
    if (total == 0)
        return cudaSuccess;
    PushGroupsMixed<1> G{};
    G.n = 1, G.chunk0[0] = 0, G.chunk0[1] = total, G.g[0] = a;
    pk_dispatch<true>(G, order, mirror, bc, dim3(static_cast<unsigned>(std::min<int64_t>(total, max_ctas))), st);
    return cudaGetLastError();
}

cudaError_t launch_push_nvv(PushArgsMixed const &a, bool mirror, int bc, int max_ctas, cudaStream_t st)
{
    int64_t const total = chunks_of(a.n);
    if (total == 0)
        return cudaSuccess;
    PushGroupsMixed<1> G{};
    G.n = 1, G.chunk0[0] = 0, G.chunk0[1] = total, G.g[0] = a;
    dim3 const g(static_cast<unsigned>(std::min<int64_t>(total, max_ctas)));
    if (bc == 0)
        mirror ? pk_nvv<true, BCK_PERIODIC>(G, g, st) : pk_nvv<false, BCK_PERIODIC>(G, g, st);
    else if (bc == 1)
        mirror ? pk_nvv<true, BCK_REFLECTING>(G, g, st) : pk_nvv<false, BCK_REFLECTING>(G, g, st);
    else
        mirror ? pk_nvv<true, BCK_ABSORBING>(G, g, st) : pk_nvv<false, BCK_ABSORBING>(G, g, st);
    return cudaGetLastError();
}

} // namespace h1d
