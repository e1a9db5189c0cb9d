// Launches of the particle pass, compiled in their own translation units (push_fp64.cu,
// push_mixed.cu): one launch covers one group of particles (a species of a run) or up to
// BATCH_GROUPS groups of an ensemble that share shape order, geometry, boundary and precision.
#pragma once

#include "particles_mixed.cuh"

#include <cuda_runtime.h>

namespace h1d {

constexpr int BATCH_GROUPS = 64;

// opt every instantiation into its dynamic shared memory, once per process and device
cudaError_t set_push_smem_fp64();
cudaError_t set_push_smem_mixed();

// one pass over `n` groups; grid = min(chunks, max_ctas) persistent CTAs
cudaError_t launch_push_groups(PushArgs const *args, int n, int order, bool mirror, int bc, int max_ctas,
                               cudaStream_t st);
cudaError_t launch_push_groups(PushArgsMixed const *args, int n, int order, bool mirror, int bc, int max_ctas,
                               cudaStream_t st);
// one pass over a species whose weights evolve (push_kernel<..., PSD = true>, push_kernel_mixed<..., PSD = true>)
cudaError_t launch_push_psd(PushArgs const &a, int order, bool mirror, int bc, int max_ctas, cudaStream_t st);
cudaError_t launch_push_psd(PushArgsMixed const &a, int order, bool mirror, int bc, int max_ctas, cudaStream_t st);
// a CIC pass (order 1, fixed weights) that also deposits collect_all's second moments into a.nvv
cudaError_t launch_push_nvv(PushArgs const &a, bool mirror, int bc, int max_ctas, cudaStream_t st);
cudaError_t launch_push_nvv(PushArgsMixed const &a, bool mirror, int bc, int max_ctas, cudaStream_t st);
// CTAs per SM of a second-moment launch (its windows take more shared memory)
constexpr int PIPE_CTAS_PER_SM_NVV_FP64  = 2;
constexpr int PIPE_CTAS_PER_SM_NVV_MIXED = 3;

} // namespace h1d
