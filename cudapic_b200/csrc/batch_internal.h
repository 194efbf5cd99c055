// batch_internal.h -- the per-discharge descriptor of a batch and the
// launchers of the batched kernels (kernels_batch.cu, kernels_poisson.cu).
//
// A batch steps many independent discharges (cudapic_state objects) in
// lockstep: one launch per kernel of the step covers every discharge.  The
// particle planes of all discharges live in one pool, so the kernels take
// the plane bases as launch parameters and each discharge's offset from its
// descriptor; the descriptors hold the other per-discharge buffers, with
// the density roles as they were oriented when the batch was (re)built.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>

#include "../../include/cudapic.h"

namespace cudapic {

// Largest number of discharges one batch takes (the per-CTA plan is a
// shared-memory prefix over the discharges' counts).
constexpr uint32_t BATCH_MAX_DISCHARGES = 1024;

// Pooled particle planes of a batch: one allocation of PLANES x len
// elements; discharge d owns [off_d, off_d + capacity_d) of every plane
// (off_d a multiple of 64, so every discharge starts 256-byte aligned).
// Plane (species, side, component) is (species * 2 + side) * 4 + component
// with components x, vx, vy, vz; RNG plane (species, k) is 16 + species * 4 + k.
constexpr int POOL_PLANES = 24;
constexpr int pool_plane(int species, int side, int comp) { return (species * 2 + side) * 4 + comp; }
constexpr int pool_rng_plane(int species, int k) { return 16 + species * 4 + k; }

// Particle planes of a step, read as kernel parameters.  Indices into them
// are `off` + a discharge-local index: off = 0 for a one-discharge launch,
// the discharge's offset in a batch's pooled planes otherwise, so the bases
// stay launch constants and only the offset is per discharge.
struct StepPlanes {
    const float *sx, *svx, *svy, *svz;        // source side
    float *dx, *dvx, *dvy, *dvz;              // destination side
    uint32_t *rng0, *rng1, *rng2, *rng3;      // electrons: RNG planes (by source slot)
    float *ix, *ivx, *ivy, *ivz;              // electrons: ion side receiving ionization spawns
};

// The electron planes of the live side of an in-place step (inplace.cuh),
// read and written in place, and the ion side receiving ionization spawns.
struct InplacePlanes {
    float *x, *vx, *vy, *vz;
    uint32_t *rng0, *rng1, *rng2, *rng3;
    float *ix, *ivx, *ivy, *ivz;
};

// The collider list of an in-place step: one record (slot, vx, vy, vz and
// the RNG state past the test draw) per collider in eight planes of
// capacity entries: the other side's x, vx, vy, vz planes of the electrons
// and of the ions, which an in-place electron step does not otherwise use.
struct CollList {
    uint32_t *slot;
    float *vx, *vy, *vz;
    uint32_t *r0, *r1, *r2, *r3;
};

// Counters-block words of the in-place step (after the fused step's words:
// n_e, n_i, alive, step, dev_err, alive_i, ticket, pad, work).
constexpr int CTR_COLL_COUNT = 12;   // colliders listed by the stream pass
constexpr int CTR_COLL_TICKET = 13;  // CTA completion ticket of the scatter pass
constexpr int CTR_SPAWN_FROM = 14;   // slot count when the stream pass ran (first spawn slot)

struct BatchDisc {
    cudapic_grid g;                                        // dev_err, work: the discharge's own words
    uint32_t off;                                          // element offset in the pooled planes
    float *e_dens[2], *i_dens[2];                          // [role]
    uint32_t *counters;                                    // n_e, n_i, alive, step, dev_err, alive_i, ticket
    float *efield, *pot;
    const float *pot0_table;
    const float *cs, *sigma_tot_e, *sigma_tot_i;
    float sigma_max_e;
    float ion_k;                                           // the ion test's certain-rejection bound
    cudapic_wall_counters *wall;                           // [2]: electrons, ions (measurement)
    unsigned long long *mcount;                            // [3]: e / i collisions, EEPF samples
    double *cumul_e, *cumul_i, *esum;
    uint32_t *eepf;
    double *xt;                                            // XT accumulators (may be null), n_xt columns
    uint32_t n_xt;
};

// Density roles of a particle step (the same for every discharge).
struct StepRoles {
    int dens;          // density buffer receiving the survivors
    int dens_i;        // electrons: ion density buffer receiving spawned ions
    int measure;       // count absorbed particles and collisions
};

// Planes of one species on one side (ion collisions, EEPF).
struct SidePlanes {
    float *x, *vx, *vy, *vz;
    uint32_t *rng0, *rng1, *rng2, *rng3;
};

// Solves every discharge's field (one CTA each) and writes the clamped
// particle counts: counts[d] electrons, counts[D + d] ions.  e_read / i_read:
// density buffers read; the other electron buffer is cleared, and the other
// ion buffer too when ion_step.  measure: adds the read densities to the
// time-averaged ones (ions only on an ion step).
int launch_batch_poisson(const BatchDisc *desc, uint32_t *counts, uint32_t D, uint32_t max_n_g, uint32_t flags,
                         int e_read, int i_read, int ion_step, int measure, cudaStream_t stream);
// The fused electron step (mcc) or the ion push with deposit (!mcc) of every
// discharge over the pooled planes `pl` (the source, destination and spawn
// sides chosen by the caller); counts: that species' counts written by
// launch_batch_poisson.
int launch_batch_step(bool mcc, const StepPlanes &pl, const BatchDisc *desc, const uint32_t *counts, uint32_t D,
                      uint64_t cap_sum, uint32_t max_n_g, const StepRoles &r, cudaStream_t stream);
// The in-place electron step of every discharge (inplace.cuh): the stream
// pass over the live side `pl` (counts: the electron counts written by
// launch_batch_poisson; colliders recorded in `list`, the pooled planes of
// the other side, at each discharge's offset), then the scatter pass
// (spawned ions to pl.ix..ivz; ticket: a word of the batch, zero between
// launches).
int launch_batch_inplace(const InplacePlanes &pl, const CollList &list, const BatchDisc *desc, const uint32_t *counts,
                         uint32_t D, uint64_t cap_sum, uint32_t max_n_g, const StepRoles &r, cudaStream_t stream);
int launch_batch_scatter(const InplacePlanes &pl, const CollList &list, const BatchDisc *desc, uint32_t D,
                         uint64_t cap_sum, const StepRoles &r, uint32_t *ticket, cudaStream_t stream);
// Ion collisions of every discharge (ions on the pooled side `ions`, counts
// read from the discharges' counters).
int launch_batch_collisions_i(const SidePlanes &ions, const BatchDisc *desc, uint32_t D, uint64_t cap_sum,
                              int measure, cudaStream_t stream);
// EEPF and centre-energy samples of every discharge (electrons on the pooled
// side `electrons`).
int launch_batch_eepf(const SidePlanes &electrons, const BatchDisc *desc, uint32_t D, uint64_t cap_sum,
                      cudaStream_t stream);
// XT accumulation of one species of every discharge (before its push).
int launch_batch_xt_particles(bool ions, const SidePlanes &sp, const BatchDisc *desc, uint32_t D, uint32_t max_n_g,
                              uint64_t cap_sum, cudaStream_t stream);

}  // namespace cudapic
