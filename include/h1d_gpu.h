/*
 * h1d_gpu.h -- C-ABI of the B200 (sm_100a) implementation of the hybrid_1d per-step hot path.
 *
 * The hot path is one step of the kinetic-ion / fluid-electron cycle of the 1-D hybrid code
 * for HFEMIC wave simulations (kyungguk1/hybrid_code-hfemic_wave):
 *   Boris push of kinetic ions in the mirror field B0(1 + xi^2 x^2) with its curvilinear
 *   transforms, Shape<1..3> interpolation of E and dB to the particles, deposit of the n and
 *   nV moments (nvv on demand), particle boundary conditions, and the CAM-CL or
 *   predictor-corrector B/E/current cycle that consumes the moments.
 *
 * Every entry point replaces one piece of the reference's `Domain` interface, so that a
 * `Domain` subclass can forward `advance_by` here:
 *
 *   h1d_create            <- Domain_CAMCL / Domain_PC constructors
 *                            (src/hybrid_1d/Core/Domain_CAMCL.cc:11, Core/Domain_PC.cc:11,
 *                             Core/Domain.cc:42-55) with the compile-time `Input` of
 *                            src/hybrid_1d/Include/Inputs.h:13-241 passed as a runtime struct
 *   h1d_upload_particles  <- PartSpecies::bucket after populate/load_ptls
 *                            (Core/PartSpecies.h:33-34, Core/PartSpecies.cc:75-101)
 *   h1d_upload_fields     <- Domain::bfield / Domain::efield contents (Core/Domain.h:30-31)
 *   h1d_upload_cold       <- ColdSpecies::mom0_full / mom1_full (Core/ColdSpecies.h:21-22)
 *   h1d_advance           <- Domain::advance_by(unsigned) (Core/Domain.h:46,
 *                            Core/Domain_CAMCL.cc:21-56, Core/Domain_PC.cc:21-78)
 *   h1d_download_*        <- what the recorders read after advance_by: bfield, efield,
 *                            charge, current, Species::moment<0..2>() (Core/Species.h:61-75),
 *                            the particle bucket (Driver.cc:211-220)
 *   h1d_energy            <- EnergyRecorder::dump (src/hybrid_1d/Recorder/EnergyRecorder.cc:98-140)
 *
 * Conventions
 *   - Every function returns an int status (H1D_OK = 0).  Nonzero codes map to the
 *     reference's exceptions: H1D_ERR_MOVED_TOO_FAR is the std::domain_error
 *     "particle(s) moved too far" of PartSpecies::update_pos (Core/PartSpecies.cc:113);
 *     H1D_ERR_INVALID_ARG is std::invalid_argument of the descriptors/ParamSet checks.
 *     h1d_status_string() gives the detail of the last error of a run.
 *   - Grid buffers use the reference GridArray layout (LibPIC/PIC/GridArray.h:36-38):
 *     (Nx + 2*H1D_PAD) elements from dead_begin() to dead_end(), ghost cells included;
 *     CartVector elements are interleaved {x,y,z} (24 B), CartTensor elements are
 *     {xx,yy,zz,xy,yz,zx} (48 B, LibPIC/PIC/VT/TensorTemplate.h:25-38).
 *   - Particle buffers are structure-of-arrays in caller memory.  The library keeps no
 *     pointer to caller memory after a call returns.  The library owns all device memory.
 *   - One run is driven by one host thread at a time (the reference Domain is
 *     single-threaded).  Each run owns one CUDA stream; all work of a run is ordered on it.
 */
#ifndef H1D_GPU_H
#define H1D_GPU_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define H1D_ABI_VERSION 4

/* number of ghost cells on each side; Input::number_of_ghost_cells (Include/Inputs.h:22) */
#define H1D_PAD 3
#define H1D_MAX_KINETIC 8
#define H1D_MAX_COLD 4
#define H1D_MAX_SOURCES 2
#define H1D_MAX_SOURCE_POINTS 16

/* status codes */
enum {
    H1D_OK                = 0,
    H1D_ERR_INVALID_ARG   = 1, /* std::invalid_argument in the reference */
    H1D_ERR_MOVED_TOO_FAR = 2, /* std::domain_error, PartSpecies.cc:113 */
    H1D_ERR_OOM           = 3,
    H1D_ERR_CUDA          = 4,
    H1D_ERR_TIMEOUT       = 5,
    H1D_ERR_NAN           = 6,
    H1D_ERR_STATE         = 7, /* call out of order, e.g. advance before upload */
    H1D_ERR_NO_DEVICE     = 8
};

/* Algorithm (LibPIC/PIC/Predefined.h:35-38): same numeric values */
enum { H1D_ALGO_PC = 0, H1D_ALGO_CAMCL = 1 };
/* BC (Predefined.h:49-52): same numeric values; ABSORBING is an extension without a
 * reference counterpart (particles leaving the domain are dropped) */
enum { H1D_BC_PERIODIC = 0, H1D_BC_REFLECTING = 1, H1D_BC_ABSORBING = 2 };
/* arithmetic of the particle push/deposit; the field cycle is FP64 in both */
enum { H1D_PREC_FP64 = 0, H1D_PREC_MIXED = 1 };

/* particle schemes (ParticleScheme, LibPIC/PIC/Predefined.h:28-31) */
#define H1D_FULL_F  0
#define H1D_DELTA_F 1

/* the equilibrium distribution of a kinetic species (the alternatives of VDFVariant,
 * LibPIC/PIC/VDFVariant.h): its f0 and its moments n0, nV0 = 0, nvv0 enter the step only when the
 * species' weights evolve (delta-f or PSD refresh) */
#define H1D_VDF_BIMAXWELLIAN  0 /* MaxwellianVDF (VDF/MaxwellianVDF.cc), BiMaxPlasmaDesc */
#define H1D_VDF_LOSSCONE      1 /* LossconeVDF (VDF/LossconeVDF.cc), LossconePlasmaDesc */
#define H1D_VDF_PARTIAL_SHELL 2 /* PartialShellVDF (VDF/PartialShellVDF.cc), PartialShellPlasmaDesc */
#define H1D_VDF_COUNTER_BEAM  3 /* CounterBeamVDF (VDF/CounterBeamVDF.cc), CounterBeamPlasmaDesc */

/* KineticPlasmaDesc (LibPIC/PIC/PlasmaDesc.h:118-177) with the parameters of its equilibrium
 * distribution (BiMaxPlasmaDesc, LossconePlasmaDesc, PartialShellPlasmaDesc, CounterBeamPlasmaDesc:
 * PlasmaDesc.h:207-345) */
typedef struct h1d_kinetic_desc {
    double  Oc;          /* PlasmaDesc::Oc, signed cyclotron frequency */
    double  op;          /* PlasmaDesc::op, plasma frequency */
    int64_t n_smooth;    /* PlasmaDesc::number_of_source_smoothings */
    int64_t Nc;          /* KineticPlasmaDesc::Nc, particles per cell: h1d_create reserves device
                            buffers for Nx * Nc particles (more are allocated on upload if needed) */
    int64_t shape_order; /* 1 (CIC), 2 (TSC) or 3 */
    double  moment_norm; /* PartSpecies::Nc (PartSpecies.cc:45-49): Nx*Nc*Nrefcell_div_Ntotal,
                            the particle count of the reference cell used to normalise moments */
    /* Phase-space density weighting.  With scheme H1D_DELTA_F, or a nonzero psd_refresh_frequency,
     * every particle carries its physical density real_f and marker density marker
     * (Particle::PSD, LibPIC/PIC/Particle.h:26-34; h1d_upload_psd) and its weight is recomputed
     * every step from the equilibrium f0 of the species' distribution `vdf` at its new velocity
     * (PartSpecies::impl_update_weight, Core/PartSpecies.cc:178-208); delta-f moments add the
     * equilibrium moments n0, nV0 = 0, nvv0 (PartSpecies.cc:115-143).  The fields below the
     * scheme are read only for such species. */
    int32_t scheme;                /* H1D_FULL_F or H1D_DELTA_F (KineticPlasmaDesc::scheme) */
    int32_t vdf;                   /* H1D_VDF_*; 0 (bi-Maxwellian) in a zero-initialised desc */
    double  psd_refresh_frequency; /* KineticPlasmaDesc::psd_refresh_frequency (>= 0) */
    double  vth1;                  /* thermal speed sqrt(beta) c |Oc| / op of the distribution: beta1
                                      (bi-Maxwellian, loss-cone: MaxwellianVDF.cc:24, LossconeVDF.cc:33)
                                      or the thermal spread beta (partial shell, counter-beam:
                                      PartialShellVDF.cc:27, CounterBeamVDF.cc:40) */
    double  T2_T1;                 /* bi-Maxwellian, loss-cone: BiMaxPlasmaDesc::T2_T1 at the
                                      equator (for a LossconePlasmaDesc built from a vth_ratio,
                                      (1 + beta) vth_ratio, PlasmaDesc.h:271-272); others: unused */
    double  vdf_param[3];          /* loss-cone: {losscone.beta, -, -};
                                      partial shell: {zeta (a non-negative integer), vs, -};
                                      counter-beam: {nu, vs, -}; bi-Maxwellian: unused */
} h1d_kinetic_desc;

/* ColdPlasmaDesc (PlasmaDesc.h:92-114) */
typedef struct h1d_cold_desc {
    double  Oc;
    double  op;
    int64_t n_smooth;
} h1d_cold_desc;

/* eFluidDesc (PlasmaDesc.h:66-88); gamma = closure/10 / (closure%10) */
typedef struct h1d_efluid_desc {
    double Oc;
    double op;
    double beta;
    double gamma;
} h1d_efluid_desc;

/* ExternalSourceDesc<N> (LibPIC/PIC/PlasmaDesc.h:363-437): an antenna current of angular frequency
 * omega applied over [start, start + duration] with cosine ease-in/-out ramps, at n_points source
 * positions q1 with complex field-aligned amplitudes J0 = J0re + i J0im
 * (Core/ExternalSource.cc:12-66) */
typedef struct h1d_source_desc {
    double  omega;
    double  start, duration; /* ExternalSourceBase::extent {loc, len} */
    double  ease_in, ease_out;
    int64_t n_smooth;        /* PlasmaDesc::number_of_source_smoothings */
    int64_t n_points;        /* <= H1D_MAX_SOURCE_POINTS */
    double  pos[H1D_MAX_SOURCE_POINTS];
    double  J0re[H1D_MAX_SOURCE_POINTS][3];
    double  J0im[H1D_MAX_SOURCE_POINTS][3];
} h1d_source_desc;

/* The runtime form of `struct Input` (Include/Inputs.h:13-241) for one run */
typedef struct h1d_params {
    int64_t Nx;          /* Input::Nx, whole domain (one GPU holds the whole field line) */
    double  Dx;          /* Input::Dx */
    double  xi;          /* Input::xi */
    double  O0;          /* Input::O0 */
    double  c;           /* Input::c */
    double  dt;          /* Input::dt */
    int64_t n_subcycles; /* Input::n_subcycles (CAM-CL only), >= 2 */
    int32_t algorithm;   /* H1D_ALGO_* */
    int32_t particle_bc; /* H1D_BC_* */
    int32_t randomize_gyrophase; /* Input::should_randomize_gyrophase_of_reflecting_particles;
                                    the reference seeds from std::random_device (Delegate.cc:146-156);
                                    here a counter-based hash of (seed, step, particle) */
    int32_t precision;   /* H1D_PREC_* */
    uint64_t gyrophase_seed;
    int64_t phase_retardation_inset;  /* Input::phase_retardation (MaskingFunction.h:14-39) */
    double  phase_retardation_factor;
    int64_t amplitude_damping_inset;  /* Input::amplitude_damping */
    double  amplitude_damping_factor;
    double  moment_weighting; /* Species::m_moment_weighting_factor = 1/clones (Species.cc:10-17); 1 */
    int32_t sort_interval;    /* steps between particle cell sorts; 0 = library default */
    int32_t n_kinetic;
    int32_t n_cold;
    int32_t n_sources;        /* external current sources (Input::source_descs) */
    h1d_efluid_desc  efluid;
    h1d_kinetic_desc kinetic[H1D_MAX_KINETIC];
    h1d_cold_desc    cold[H1D_MAX_COLD];
    h1d_source_desc  sources[H1D_MAX_SOURCES];
} h1d_params;

typedef struct h1d_run h1d_run;

/* ABI introspection: H1D_ABI_VERSION and sizeof(h1d_params) the library was built with */
int  h1d_abi_version(void);
size_t h1d_params_size(void);

/* Validate params (same checks as InputWrapper.h:132-155, ParamSet.cc:25-29 and the
 * descriptor constructors) and allocate the run on the current CUDA device. */
int h1d_create(const h1d_params *params, h1d_run **out);
int h1d_destroy(h1d_run *run);

/* Device memory.  The library allocates its device buffers (runs, batches, served requests) from
 * a memory pool of its own per device, which keeps the blocks a destroyed run releases for the
 * next run instead of returning them to the driver (the reference holds its grids and particles
 * in host containers and has no counterpart).  h1d_trim_device_memory returns the pool's unused
 * blocks on the current device to the driver, keeping at most `keep_bytes` of them;
 * *pool_bytes, when not null, receives the device memory the pool still holds afterwards (blocks
 * in use included). */
int h1d_trim_device_memory(size_t keep_bytes, size_t *pool_bytes);

/* Particles of kinetic species `s` as SoA, positions q1 in [-Nx/2, Nx/2) (ParamSet.cc:22).
 * Replaces any previous particles of that species. */
int h1d_upload_particles(h1d_run *run, int s, int64_t n, const double *q1, const double *vx,
                         const double *vy, const double *vz, const double *w);
/* Phase-space densities of the particles of species `s` (Particle::PSD::real_f, ::marker), in the
 * order of the last h1d_upload_particles and before the first step, for a species whose weights
 * evolve (scheme H1D_DELTA_F or psd_refresh_frequency != 0); INVALID_ARG for other species, when
 * n differs from the uploaded count or after the particles were reordered.  Until it is called,
 * real_f = w and marker = 1.  Mixed-precision runs keep them in FP32. */
int h1d_upload_psd(h1d_run *run, int s, int64_t n, const double *real_f, const double *marker);
/* ... and back, in the order of h1d_download_particles; either pointer may be NULL. */
int h1d_download_psd(h1d_run *run, int s, double *real_f, double *marker);
/* PartSpecies::populate with a bi-Maxwellian MaxwellianVDF (VDF/MaxwellianVDF.cc:88-134),
 * on the device: n particles of kinetic species `s` with parallel beta `beta1` and T_perp/T_par
 * `T2_T1`, positions from the base-2 radical inverse through q1_of_N, velocities from base-3/5
 * radical inverses and two counter-based uniforms of (seed, s, particle), full-f weight 1.
 * Replaces any previous particles of that species.  The reference seeds its generators with fixed
 * constants; here `seed` selects the sequences, and loader.py computes the same particles on the
 * host.  Refuses species whose weights evolve or whose `vdf` is not H1D_VDF_BIMAXWELLIAN
 * (H1D_ERR_INVALID_ARG): those are loaded on the host and uploaded. */
int h1d_populate(h1d_run *run, int s, int64_t n, uint64_t seed, double beta1, double T2_T1);
/* B (full grid) and E (half grid), each (Nx+2*H1D_PAD)*3 doubles, GridArray layout */
int h1d_upload_fields(h1d_run *run, const double *B, const double *E);
/* cold species `i`: mom0_full (Nx+2*H1D_PAD doubles), mom1_full ((Nx+2*H1D_PAD)*3) */
int h1d_upload_cold(h1d_run *run, int i, const double *n_full, const double *nV_full);

/* Domain::advance_by(n_steps), then wait and check the device status word. */
int h1d_advance(h1d_run *run, uint32_t n_steps);
/* Enqueue advance_by(n_steps) on the run's stream without waiting. */
int h1d_advance_async(h1d_run *run, uint32_t n_steps);
/* Wait for the run's stream; report a device-side error (moved too far, NaN) if any. */
int h1d_synchronize(h1d_run *run);
/* The run's cudaStream_t, for callers that time or order work around the run. */
int h1d_get_stream(h1d_run *run, void **stream);

int h1d_particle_count(h1d_run *run, int s, int64_t *n);
/* Any output pointer may be NULL.  pid[k] is the upload index of the k-th particle (the
 * library keeps particles cell-sorted, so the order is its own). */
int h1d_download_particles(h1d_run *run, int s, double *q1, double *vx, double *vy, double *vz,
                           double *w, int64_t *pid);
int h1d_download_fields(h1d_run *run, double *B, double *E);
/* Domain::charge and Domain::current after the last step ((Nx+2*H1D_PAD) and *3 doubles) */
int h1d_download_sources(h1d_run *run, double *charge, double *current);
/* Species::moment<0..2>() of kinetic species `s` after the post-process collect_all
 * (PartSpecies.cc:129-143, 225-244, always CIC) and boundary_gather; any pointer may be NULL.
 * On a CAM-CL run whose species are all CIC with fixed weights, the last step of h1d_advance
 * forms these sums in its particle pass; otherwise they are computed here, after a sort of the
 * particles that moved since their last one. */
int h1d_download_moments(h1d_run *run, int s, double *n, double *nV, double *nvv);
/* cold species moments after collect_all (ColdSpecies.cc:48-77) and mom0_full/mom1_full */
int h1d_download_cold(h1d_run *run, int i, double *n, double *nV, double *nvv, double *n_full,
                      double *nV_full);
/* EnergyRecorder::dump (EnergyRecorder.cc:98-140): dB2O2[3], dE2O2[3], and for every kinetic
 * species then every cold species KE_lab[3], KE_pla[3]; computed on the device */
int h1d_energy(h1d_run *run, double *dB2O2, double *dE2O2, double *KE_lab, double *KE_pla);

/* VHistogramRecorder (Recorder/VHistogramRecorder.cc:222-306) on the device: gyro-averaged velocity
 * histogram of kinetic species `s` over the particles with q1 in [ext_loc, ext_loc + ext_len),
 * relative to the bulk velocity of the recorded moments, v1 (parallel) in v1dim bins over
 * [v1min, v1min + v1len) and v2 (perpendicular speed) in v2dim bins over [v2min, v2min + v2len).
 * out[3 * (i1 * v2dim + i2) + {0, 1, 2}] = {marker count, weight sum, real_f/marker sum} / total
 * (real_f/marker = w for species whose weights do not evolve),
 * total = the particles in the extent (the recorder's normalisation).  Zero-based bins; the
 * recorder writes them one-based. */
int h1d_vhistogram(h1d_run *run, int s, double ext_loc, double ext_len, double v1min, double v1len, int64_t v1dim,
                   double v2min, double v2len, int64_t v2dim, double *out, int64_t *total);

/* Phase timing with CUDA events recorded on the run's stream around each kernel group while
 * profiling is enabled; read() waits for the stream and returns the accumulated figures. */
typedef struct h1d_profile {
    double  push_ms;          /* fused push/deposit kernels */
    double  sort_ms;          /* cell sort (keys, histograms, scans, scatters, gather) */
    double  field_ms;         /* grid-phase kernel */
    int64_t push_launches;
    int64_t sort_calls;
    int64_t field_launches;
    int64_t kernel_launches;  /* every kernel this library launched while profiling */
    int64_t particles_pushed; /* sum over push launches of the particles each processed */
    int64_t window_misses;    /* particle deposits that missed the register window of their warp */
} h1d_profile;
int h1d_profile_enable(h1d_run *run, int on); /* on != 0 also resets the counters */
int h1d_profile_read(h1d_run *run, h1d_profile *out);

/* Evaluate the device arithmetic primitives of the particle kernels on the current device, for
 * self-checks against the host C library: for each x[k] (|x| < 2^30) writes
 * out[5k .. 5k+4] = floor(x), round(x) (halves away from zero), ceil(x), and for |x| <= pi/2
 * sin(x), cos(x) as computed by the kernels. */
int h1d_math_check(const double *x, int64_t n, double *out);

/* Allocation-free moment collection.  No counterpart in the reference: it is an addition for
 * callers that cannot call cudaMalloc -- for example code running inside an application whose
 * own pool allocator has reserved the device memory (an allocation outside the pool fails or
 * defeats its accounting), or a latency-critical loop where an allocation, which may
 * synchronise the device, is not acceptable.
 *
 * Computes the weighted sums of h1d_download_moments -- n, nV, nvv with the CIC shape, scaled by
 * 1/moment_norm and ghost-folded for the given particle boundary (PartSpecies::collect_all +
 * boundary_gather) -- from particles the caller holds in device memory, into device buffers the
 * caller provides (GridArray layout: n[Nx+6], nV[(Nx+6)*3], nvv[(Nx+6)*6]).  These are the moments
 * of a full-f species; for a delta-f species h1d_download_moments also adds the equilibrium
 * moments n0 and nvv0 on the interior (PartSpecies.cc:134-142), which a caller of this entry point
 * adds itself.  Work is enqueued on `stream` (a cudaStream_t; NULL for the legacy default stream)
 * and the call returns after that stream has finished it.  A particle outside the padded grid
 * (or with a non-finite position) gives H1D_ERR_NAN; a failed call has finished its queued work
 * before it returns.
 *
 * Scratch space is a fixed array compiled into this library (a static __device__ array of
 * 20 * (H1D_NOALLOC_MAX_NX + 6) doubles plus a status word, about 0.65 MB, held on every GPU that
 * loads the library until the process exits).  Nx above H1D_NOALLOC_MAX_NX is rejected with
 * H1D_ERR_INVALID_ARG.  The first call on a device looks up that array's device address (once per
 * device, with the device current).  All calls share the one array: calls that overlap on the GPU (concurrent streams or threads) race and
 * must be serialised by the caller.  The looked-up address is kept for the life of the process:
 * do not call this entry point again on a device after cudaDeviceReset. */
#define H1D_NOALLOC_MAX_NX 4096
int h1d_collect_moments_noalloc(int64_t Nx, double moment_norm, int particle_bc, const double *q1, const double *vx,
                                const double *vy, const double *vz, const double *w, int64_t n, double *n_out,
                                double *nV_out, double *nvv_out, void *stream);

/* Checkpoint / resume, the content of the reference's snapshot (Recorder/Snapshot.cc:148-185,
 * 330-375; HDF5 there, a flat little-endian byte image here): step count, a signature of the
 * parameters that a load verifies (Snapshot.cc:340-342: "signature verification failed" ->
 * H1D_ERR_INVALID_ARG), B, E, every kinetic species' particles with their ids in the run's own
 * precision, every cold species' mom0_full / mom1_full.  After a load the next advance starts as
 * the reference's does after loading a snapshot (sources recomputed from the particles). */
int h1d_checkpoint_size(h1d_run *run, size_t *bytes);
int h1d_checkpoint_save(h1d_run *run, void *buffer, size_t capacity, size_t *written);
int h1d_checkpoint_load(h1d_run *run, const void *buffer, size_t size);
/* the step count (the reference's Driver step count after advance_by calls) */
int h1d_step_count(h1d_run *run, int64_t *step);

/* Tuning of a run: steps between cell sorts (0 keeps the current value) and CTAs per SM of the
 * particle pass (0 = the kernel's default, at most 3 for FP64 and 4 for mixed precision).  No
 * counterpart in the reference, which never sorts. */
int h1d_configure(h1d_run *run, int sort_interval, int push_ctas_per_sm);
/* Autotuner (no counterpart in the reference): advances the run by real CAM-CL steps while timing
 * two sort blocks for each candidate sort interval (8, 12, 16, 24, 32) and then for each CTA count of the
 * particle pass, and keeps the fastest.  *steps_taken receives the number of steps it advanced. */
int h1d_autotune(h1d_run *run, uint32_t *steps_taken, int *sort_interval, int *push_ctas_per_sm);

/* ---- Ensembles (no counterpart in the reference) ---------------------------------------------
 * A batch advances many runs of one algorithm together on one stream of the current device: all
 * CAM-CL, or all predictor-corrector.  A CAM-CL step is one launch of the particle pass per kind
 * of particle group (shape order, geometry, boundary, precision) covering every species of every
 * member (a species with evolving weights, delta-f or PSD refresh, takes a launch of its own), and
 * one launch of the field cycle covering every member's grid; a predictor-corrector step is three
 * such field launches (Domain_PC.cc:79-205) around the predictor and the corrector particle passes.  Steps come in blocks of sort_interval steps, all groups cell-sorted at the
 * start of a block.  When no member uses absorbing particles or gyrophase randomization, a pair of
 * blocks is captured once as a CUDA graph and replayed while the members are unchanged (an upload
 * to a member invalidates it).  Members stay owned by the caller, must outlive the batch and
 * belong to one batch at a time; while a member, a run's work is ordered on the batch's stream,
 * and h1d_download_* / h1d_energy on it are allowed between batch calls. */
typedef struct h1d_batch h1d_batch;
typedef struct h1d_batch_stats {
    int64_t steps;           /* batch steps taken */
    int64_t kernel_launches; /* kernels of this library launched, graph replays included */
    int64_t graph_launches;  /* CUDA graph replays */
    int64_t graphs_built;
} h1d_batch_stats;
int h1d_batch_create(h1d_run *const *runs, int n_runs, h1d_batch **out);
int h1d_batch_destroy(h1d_batch *batch);
int h1d_batch_advance(h1d_batch *batch, uint32_t n_steps);
int h1d_batch_advance_async(h1d_batch *batch, uint32_t n_steps);
/* Member i (in the order given to h1d_batch_create) advances by n_steps[i]: all members step
 * together until the smallest count is reached, then that member leaves the particle passes, the
 * sorts and the field launch, and the rest go on, so each member ends as its own
 * advance_by(n_steps[i]) would leave it (a count of 0 leaves a member as it was).  Steps are eager
 * when the counts differ; equal counts are h1d_batch_advance_async. */
int h1d_batch_advance_members_async(h1d_batch *batch, const uint32_t *n_steps);
int h1d_batch_synchronize(h1d_batch *batch);
int h1d_batch_get_stream(h1d_batch *batch, void **stream);
/* sort_interval > 0 sets the block length (0 keeps it); push_ctas_per_sm as in h1d_configure;
 * use_graphs = 0 keeps every step eager */
int h1d_batch_configure(h1d_batch *batch, int sort_interval, int push_ctas_per_sm, int use_graphs);
/* the autotuner of h1d_autotune over the whole batch; the choice also becomes every member's */
int h1d_batch_autotune(h1d_batch *batch, uint32_t *steps_taken, int *sort_interval, int *push_ctas_per_sm);
int h1d_batch_stats_read(h1d_batch *batch, h1d_batch_stats *out);
const char *h1d_batch_status_string(h1d_batch *batch);

/* ---- Serving loop (no counterpart in the reference) --------------------------------------------
 * Requests wait in a queue until the device memory they need fits the server's budget; admitted
 * runs are built on the device (h1d_populate, cold fluid at rest, zero fields), advance together
 * as one batch by up to `steps_per_tick` steps per h1d_server_tick, and are read back (fields,
 * energies, moments) and freed when their steps are done, which admits the next requests.  The
 * caller drives the loop by calling h1d_server_tick from one thread; submit, poll, result and
 * release may come from other threads and do not wait for a tick in progress (the server's lock is
 * not held while the GPU works).  Requests admitted during a tick are built while the batches
 * advance and join them at the next tick; a request whose run fails (e.g. moved too far) fails
 * alone.  Times are seconds since h1d_server_create on a monotonic clock. */
typedef struct h1d_server h1d_server;
typedef struct h1d_request {
    h1d_params params;                    /* a CAM-CL or predictor-corrector run */
    double     beta1[H1D_MAX_KINETIC];    /* loader of each kinetic species: parallel beta */
    double     T2_T1[H1D_MAX_KINETIC];    /* and T_perp / T_par */
    int64_t    n_particles[H1D_MAX_KINETIC];
    uint64_t   seed;                      /* loader seed */
    uint32_t   n_steps;
    uint32_t   reserved0;
} h1d_request;
enum { H1D_REQ_QUEUED = 0, H1D_REQ_ACTIVE = 1, H1D_REQ_DONE = 2, H1D_REQ_FAILED = 3 };
typedef struct h1d_server_stats {
    int64_t submitted, admitted, completed, failed;
    int64_t steps, kernel_launches, graph_launches, batches_built;
    int64_t bytes_in_use, peak_bytes; /* device memory of admitted runs, by the admission estimate */
} h1d_server_stats;
int h1d_server_create(size_t hbm_budget_bytes, int steps_per_tick, h1d_server **out);
int h1d_server_configure(h1d_server *server, int sort_interval);
int h1d_server_submit(h1d_server *server, const h1d_request *request, uint64_t *id);
/* admit what fits, advance the active runs by one quantum, retire the finished ones */
int h1d_server_tick(h1d_server *server, int *n_active, int *n_queued);
/* state is H1D_REQ_*; returns the run's error status for a failed request */
int h1d_server_poll(h1d_server *server, uint64_t id, int *state, double *t_submit, double *t_admit, double *t_done);
/* results of a finished request: B and E ((Nx+2*H1D_PAD)*3 each), energy (6 + 6*(n_kinetic+n_cold):
 * dB2O2[3], dE2O2[3], then per species KE_lab[3], KE_pla[3]), and per kinetic species n, nV, nvv
 * as h1d_download_moments, species after species; any pointer may be NULL */
int h1d_server_result(h1d_server *server, uint64_t id, double *B, double *E, double *energy, double *n,
                      double *nV, double *nvv);
int h1d_server_release(h1d_server *server, uint64_t id);
int h1d_server_stats_read(h1d_server *server, h1d_server_stats *out);
int h1d_server_destroy(h1d_server *server);

const char *h1d_status_string(h1d_run *run);
const char *h1d_error_name(int status);

#ifdef __cplusplus
}
#endif
#endif /* H1D_GPU_H */
