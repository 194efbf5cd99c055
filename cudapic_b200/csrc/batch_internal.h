// batch_internal.h -- the per-discharge descriptor of a batch and the
// launchers of the batched kernels (kernels_batch.cu, kernels_poisson.cu).
//
// A batch steps many independent discharges (cudapic_state objects) in
// lockstep: one launch per kernel of the step covers every discharge.  The
// descriptors hold each discharge's buffers as they were oriented when the
// batch was (re)built; the launches select the side and density roles of
// the current step by index, the same for every discharge.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>

#include "../../include/cudapic.h"

namespace cudapic {

// Largest number of discharges one batch takes (the per-CTA plan is a
// shared-memory prefix over the discharges' counts).
constexpr uint32_t BATCH_MAX_DISCHARGES = 1024;

struct BatchDisc {
    cudapic_grid g;                                        // dev_err, work: the discharge's own words
    float *x[2][2], *vx[2][2], *vy[2][2], *vz[2][2];       // [species][side]
    uint32_t *rng[2][4];                                   // [species][plane]
    float *e_dens[2], *i_dens[2];                          // [role]
    uint32_t *counters;                                    // n_e, n_i, alive, step, dev_err, alive_i, ticket
    float *efield, *pot;
    const float *pot0_table;
    const float *cs, *sigma_tot_e, *sigma_tot_i;
    float sigma_max_e;
    cudapic_wall_counters *wall;                           // [2]: electrons, ions (measurement)
    unsigned long long *mcount;                            // [3]: e / i collisions, EEPF samples
    double *cumul_e, *cumul_i, *esum;
    uint32_t *eepf;
};

// Roles of a particle step: sides and density buffers by index.
struct StepRoles {
    int src, dst;      // the species' source and destination side
    int ion_side;      // electrons: side of the ions receiving ionization spawns
    int dens;          // density buffer receiving the survivors
    int dens_i;        // electrons: ion density buffer receiving spawned ions
    int measure;       // count absorbed particles and collisions
};

// Solves every discharge's field (one CTA each) and writes the clamped
// particle counts: counts[d] electrons, counts[D + d] ions.  e_read / i_read:
// density buffers read; the other electron buffer is cleared, and the other
// ion buffer too when ion_step.  measure: adds the read densities to the
// time-averaged ones (ions only on an ion step).
int launch_batch_poisson(const BatchDisc *desc, uint32_t *counts, uint32_t D, uint32_t max_n_g, uint32_t flags,
                         int e_read, int i_read, int ion_step, int measure, cudaStream_t stream);
// The fused electron step (mcc) or the ion push with deposit (!mcc) of every
// discharge; counts: that species' counts written by launch_batch_poisson.
int launch_batch_step(bool mcc, const BatchDisc *desc, const uint32_t *counts, uint32_t D, uint64_t cap_sum,
                      uint32_t max_n_g, const StepRoles &r, cudaStream_t stream);
// Ion collisions of every discharge (ions on `side`, counts read from the
// discharges' counters).
int launch_batch_collisions_i(const BatchDisc *desc, uint32_t D, uint64_t cap_sum, int side, int measure,
                              cudaStream_t stream);
// EEPF and centre-energy samples of every discharge (electrons on `side`).
int launch_batch_eepf(const BatchDisc *desc, uint32_t D, uint64_t cap_sum, int side, cudaStream_t stream);

}  // namespace cudapic
