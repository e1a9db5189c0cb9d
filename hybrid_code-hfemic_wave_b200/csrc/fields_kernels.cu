// Grid kernels of the hybrid_1d hot path.  This translation unit is compiled with
// --fmad=false: the field cycle is latency-bound, and without contraction it evaluates the
// reference's expressions operation for operation.
#define H1D_FIELD_TU
#include "launchers.h"
#include "post.cuh"

namespace h1d {

cudaError_t set_field_smem(size_t bytes)
{
    cudaError_t e = cudaFuncSetAttribute(camcl_field_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(bytes));
    if (e != cudaSuccess)
        return e;
    return cudaFuncSetAttribute(pc_field_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(bytes));
}
cudaError_t launch_pc_fields(FieldArgs const &a, int blocks, int threads, size_t smem, cudaStream_t st)
{
    pc_field_kernel<<<blocks, threads, smem, st>>>(a);
    return cudaGetLastError();
}
cudaError_t launch_camcl_fields(FieldArgs const &a, int blocks, int threads, size_t smem, cudaStream_t st)
{
    camcl_field_kernel<<<blocks, threads, smem, st>>>(a);
    return cudaGetLastError();
}
cudaError_t set_field_batch_smem(size_t bytes)
{
    cudaError_t e = cudaFuncSetAttribute(camcl_field_batch_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         static_cast<int>(bytes));
    if (e != cudaSuccess)
        return e;
    return cudaFuncSetAttribute(pc_field_batch_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(bytes));
}
cudaError_t launch_camcl_fields_batch(FieldArgs const *table, FieldBlock const *map, int blocks, int threads,
                                      size_t smem, cudaStream_t st)
{
    camcl_field_batch_kernel<<<blocks, threads, smem, st>>>(table, map);
    return cudaGetLastError();
}
cudaError_t launch_pc_fields_batch(FieldArgs const *table, FieldBlock const *map, int blocks, int threads,
                                   size_t smem, cudaStream_t st)
{
    pc_field_batch_kernel<<<blocks, threads, smem, st>>>(table, map);
    return cudaGetLastError();
}
cudaError_t launch_prep_fields(double *B, double *E, double *EB, float *EBf, int Nx, cudaStream_t st)
{
    prep_fields_kernel<<<(Nx + 2 * PAD + 255) / 256, 256, 0, st>>>(B, E, EB, EBf, Nx);
    return cudaGetLastError();
}
cudaError_t launch_ghost_fill(double *dst, double const *src, int nc, int Nx, cudaStream_t st)
{
    ghost_fill_kernel<<<1, 32, 0, st>>>(dst, src, nc, Nx);
    return cudaGetLastError();
}
cudaError_t launch_finalize_kinetic(double const *raw, double const *eq, double *out, int Nx, double s1,
                                    int reflecting, cudaStream_t st)
{
    finalize_kinetic_kernel<<<(Nx + 2 * PAD + 127) / 128, 128, 0, st>>>(raw, eq, out, Nx, s1);
    fold_moments_kernel<<<1, 32, 0, st>>>(out, Nx, reflecting);
    return cudaGetLastError();
}
cudaError_t launch_finalize_cold(double const *n_full, double const *nV_full, double *out, int Nx, double w,
                                 cudaStream_t st)
{
    finalize_cold_kernel<<<1, 256, 0, st>>>(n_full, nV_full, out, Nx, w);
    return cudaGetLastError();
}
cudaError_t launch_energy(EnergyArgs const &a, cudaStream_t st)
{
    energy_kernel<<<1, 256, 0, st>>>(a);
    return cudaGetLastError();
}
cudaError_t launch_sources(SourceArgs const &a, cudaStream_t st)
{
    source_kernel<<<1, 256, 0, st>>>(a);
    return cudaGetLastError();
}
cudaError_t launch_fill(double *a, int64_t n, double v, cudaStream_t st)
{
    fill_kernel<<<static_cast<unsigned>((n + 255) / 256), 256, 0, st>>>(a, n, v);
    return cudaGetLastError();
}
cudaError_t launch_fill_f(float *a, int64_t n, float v, cudaStream_t st)
{
    fill_f_kernel<<<static_cast<unsigned>((n + 255) / 256), 256, 0, st>>>(a, n, v);
    return cudaGetLastError();
}
cudaError_t launch_iota(int32_t *pid, int64_t n, cudaStream_t st)
{
    iota_kernel<<<static_cast<unsigned>((n + 255) / 256), 256, 0, st>>>(pid, n);
    return cudaGetLastError();
}

} // namespace h1d
