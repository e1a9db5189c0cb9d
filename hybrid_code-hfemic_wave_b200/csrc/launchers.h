// Host-side launchers of the grid kernels, which live in their own translation unit
// (fields_kernels.cu) because that unit is compiled without FMA contraction.
#pragma once

#include "fields.cuh"
#include "h1d_gpu.h"

#include <cuda_runtime.h>

namespace h1d {

struct EnergyArgs {
    double const *B, *E; // cell 0
    int           Nx, ns;
    double const *n[MAXK + MAXC], *nV[MAXK + MAXC], *nvv[MAXK + MAXC];
    double        factor[MAXK + MAXC];
    double       *out; // 6 + 6 * ns
};

cudaError_t set_field_smem(size_t bytes);
cudaError_t launch_camcl_fields(FieldArgs const &a, int blocks, int threads, size_t smem, cudaStream_t st);
cudaError_t launch_pc_fields(FieldArgs const &a, int blocks, int threads, size_t smem, cudaStream_t st);
// an ensemble in one launch: block b runs segment map[b].seg of run map[b].run (device arrays)
cudaError_t set_field_batch_smem(size_t bytes);
cudaError_t launch_camcl_fields_batch(FieldArgs const *table, FieldBlock const *map, int blocks, int threads,
                                      size_t smem, cudaStream_t st);
cudaError_t launch_pc_fields_batch(FieldArgs const *table, FieldBlock const *map, int blocks, int threads,
                                   size_t smem, cudaStream_t st);
cudaError_t launch_prep_fields(double *B, double *E, double *EB, float *EBf, int Nx, cudaStream_t st);
cudaError_t launch_ghost_fill(double *dst, double const *src, int nc, int Nx, cudaStream_t st);
cudaError_t launch_finalize_kinetic(double const *raw, double const *eq, double *out, int Nx, double s1,
                                    int reflecting, cudaStream_t st);
cudaError_t launch_finalize_cold(double const *n_full, double const *nV_full, double *out, int Nx, double w,
                                 cudaStream_t st);
cudaError_t launch_energy(EnergyArgs const &a, cudaStream_t st);
cudaError_t launch_iota(int32_t *pid, int64_t n, cudaStream_t st);
cudaError_t launch_fill(double *a, int64_t n, double v, cudaStream_t st);
cudaError_t launch_fill_f(float *a, int64_t n, float v, cudaStream_t st);
// the external sources of a run at time t (source_kernel, post.cuh)
struct SourceArgs {
    h1d_source_desc d[MAXE];
    int             ne;
    double          t, half_min, half_len, weighting;
    double         *J[MAXE][3]; // cell 0 of each component array (Nx + 2 PAD cells)
    int             M;
};
cudaError_t launch_sources(SourceArgs const &a, cudaStream_t st);

} // namespace h1d
