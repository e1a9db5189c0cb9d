/*
 * Domain_GPU.h -- drop-in GPU Domain for the hybrid_1d code of kyungguk1/hybrid_code-hfemic_wave.
 *
 * Domain_CAMCL_GPU and Domain_PC_GPU are Domain subclasses (src/hybrid_1d/Core/Domain.h:26-63)
 * whose advance_by(n) (Domain.h:46) runs the step cycle of Domain_CAMCL (Core/Domain_CAMCL.cc:21-56)
 * or Domain_PC (Core/Domain_PC.cc:21-78) on one GPU through the C ABI of libh1d_gpu.so
 * (include/h1d_gpu.h).  They are compiled inside the reference's own source tree: the reference's
 * Inputs.h, ParamSet, PartSpecies / ColdSpecies, BField, EField, Charge, Current and the recorders
 * keep their types, and Driver::make_domain (src/hybrid_1d/Driver.cc:137-147) constructs one of
 * these instead of Domain_CAMCL / Domain_PC.
 *
 * Data movement follows what the reference's callers read:
 *   - particles, fields and cold-fluid moments are uploaded on the first advance_by, after the
 *     Driver populated (Driver.cc:101-112) or a snapshot loaded them; invalidate() makes the next
 *     advance_by upload them again after the host changed them;
 *   - after every advance_by, the post-process arrays of Domain_CAMCL::advance_by
 *     (Domain_CAMCL.cc:45-55) come back into the reference's own GridArrays: bfield, efield,
 *     charge, current, every species' moment<0..2>() and every cold species' mom0_full / mom1_full;
 *   - particles come back into PartSpecies::bucket only on sync_particles(), which the Driver calls
 *     before the particle recorders and snapshots read them (Driver.cc:211-220).
 *
 * Library status codes become the reference's exceptions: H1D_ERR_MOVED_TOO_FAR is the
 * std::domain_error of PartSpecies::update_pos (Core/PartSpecies.cc:113), H1D_ERR_INVALID_ARG a
 * std::invalid_argument, anything else a std::runtime_error with the library's message.
 *
 * One GPU holds the whole field line, so the Inputs must have one subdomain and one particle
 * clone (the MPI domain split is replaced, not distributed).
 */
#pragma once

#include "Core/Domain.h"
#include "h1d_gpu.h"

#include <cstdint>
#include <vector>

HYBRID1D_BEGIN_NAMESPACE
class Domain_GPU : public Domain {
public:
    ~Domain_GPU() override;
    Domain_GPU(Domain_GPU const &)            = delete;
    Domain_GPU &operator=(Domain_GPU const &) = delete;

    void advance_by(unsigned n_steps) override;

    /// Copy the particles on the GPU back into every PartSpecies::bucket (order: the library's cell
    /// order; ids, velocities, positions and phase-space densities as the reference keeps them).
    void sync_particles();
    /// The host changed particles, fields or cold moments (e.g. a snapshot load): the next
    /// advance_by uploads them again.
    void invalidate() noexcept { m_on_device = false; }

    [[nodiscard]] h1d_run *handle() const noexcept { return m_run; }
    [[nodiscard]] int      precision() const noexcept { return m_precision; }

protected:
    Domain_GPU(ParamSet const &params, Delegate *delegate, int algorithm, int precision);

private:
    // the ids and phase-space densities of the uploaded particles, by upload index, so that a
    // download restores what the GPU does not evolve (ids always; real_f / marker of species whose
    // weights are fixed)
    struct Uploaded {
        std::vector<long long> id;
        std::vector<double>    real_f, marker;
    };
    h1d_run              *m_run{};
    int                   m_precision{};
    bool                  m_on_device{ false };
    std::vector<Uploaded> m_uploaded;

    void upload();
    void download_recorded();
    void check(int status, char const *what) const;
};

/// Domain_CAMCL (Core/Domain_CAMCL.cc) with advance_by on the GPU.
class Domain_CAMCL_GPU final : public Domain_GPU {
public:
    Domain_CAMCL_GPU(ParamSet const &params, Delegate *delegate, int precision = H1D_PREC_FP64);
};

/// Domain_PC (Core/Domain_PC.cc) with advance_by on the GPU.
class Domain_PC_GPU final : public Domain_GPU {
public:
    Domain_PC_GPU(ParamSet const &params, Delegate *delegate, int precision = H1D_PREC_FP64);
};

/// The runtime form of the compile-time Input (Include/Inputs.h) that h1d_create takes.
[[nodiscard]] h1d_params h1d_params_of(ParamSet const &params, int algorithm, int precision);
HYBRID1D_END_NAMESPACE
