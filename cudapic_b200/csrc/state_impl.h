// state_impl.h -- the simulation state object of libcudapic (state.cpp),
// shared with the batch driver (batch.cpp).
#pragma once

#include <cuda_runtime.h>

#include <cstdint>
#include <vector>

#include "internal.h"

struct cudapic_state {
    int device = 0;
    cudapic_params params{};
    cudapic_grid grid{};
    cudaStream_t stream = nullptr;
    bool own_stream = false;

    // [species][side]
    float *x[2][2] = {}, *vx[2][2] = {}, *vy[2][2] = {}, *vz[2][2] = {};
    int side[2] = {0, 0};
    uint32_t *rng[2][4] = {};
    // counters block: n_e, n_i, alive, step, dev_err, alive_i, ticket, pad, work (u64 at +32),
    // [12] in-place step's collider count, [13] its scatter ticket, [14] its first spawn slot
    uint32_t *counters = nullptr;
    float *efield = nullptr, *pot = nullptr, *pot0_table = nullptr;
    // Charge densities, double-buffered for the fused step: [cur] feeds the
    // Poisson solve, [cur ^ 1] accumulates the next step's (electrons) or
    // the next ion step's (ions) deposits.
    float *e_dens[2] = {}, *i_dens[2] = {};
    int e_cur = 0, i_cur = 0;
    bool fused = true;        // deposit inside push / collisions (default)
    bool overlap = true;      // programmatic dependent launch between the step's kernels (default)
    bool inplace = true;      // fused mode: in-place electron steps between compacting ones (default)
    bool spawn_collide = false;  // in-place steps: new electrons also collide in their birth step (eduPIC)
    // in-place steps: the scatter pass's last CTA solves the next step's
    // field (default); poisson_ahead: the step being enqueued finds its
    // solve already enqueued by the step before it
    bool solve_ahead = true;
    bool poisson_ahead = false;
    bool dens_valid = false;  // e_dens[e_cur] and both ion buffers describe the particles
    int graph_key[2][4] = {{-1, -1, -1, -1}, {-1, -1, -1, -1}};  // sides and buffer roles at capture
    float *cs = nullptr, *sigma_tot_e = nullptr, *sigma_tot_i = nullptr;
    float sigma_max_e = 0.0f;  // largest entry of sigma_tot_e (the fused step's certain-rejection bound)
    float ion_k = INFINITY;    // the fused driver's ion-test bound (ion_reject_k of sigma_tot_i)
    double *cumul_e = nullptr, *cumul_i = nullptr;
    cudapic_wall_counters *wall = nullptr;  // [0] electrons, [1] ions (measurement window)
    // measurement window: [0] electron and [1] ion collision events, [2] EEPF
    // electrons sampled; esum: their energies [eV]; measure_steps on the host
    unsigned long long *mcount = nullptr;
    double *esum = nullptr;
    uint64_t measure_steps = 0;
    double max_e_coll_freq = 0.0, max_i_coll_freq = 0.0;  // of the tables [1/s]
    uint32_t *eepf = nullptr;
    double *xt = nullptr;   // XT accumulators [XT_RAW][n_g][n_xt] (allocated when measuring starts)
    uint32_t n_xt = 0;      // XT columns (0: N_T is not a multiple of XT_BIN)

    bool measure = false;
    uint64_t steps_done = 0;
    cudaGraphExec_t graph[2] = {nullptr, nullptr};  // [measure]
    uint64_t graph_gen[2] = {0, 0};                  // tuning generation at capture
    bool graphs_enabled = true;
    std::vector<void *> allocations;
    void *batch = nullptr;  // the batch whose pool holds the particle planes (batch.cpp)

    uint32_t *n_e() const { return counters + 0; }
    uint32_t *n_i() const { return counters + 1; }
    uint32_t *alive() const { return counters + 2; }
    uint32_t *step_counter() const { return counters + 3; }
    uint32_t *dev_err() const { return counters + 4; }
    uint32_t *alive_i() const { return counters + 5; }  // fused mode: ion push slot counter
    uint32_t *ticket() const { return counters + 6; }   // fused mode: CTA completion ticket (StepLink)
    unsigned long long *work() const { return reinterpret_cast<unsigned long long *>(counters + 8); }
    float *e_density() const { return e_dens[e_cur]; }
    float *i_density() const { return i_dens[i_cur]; }
};

namespace cudapic {

struct DeviceGuard {
    int prev = 0;
    bool ok = false;
    explicit DeviceGuard(int dev) {
        if (cudaGetDevice(&prev) == cudaSuccess && cudaSetDevice(dev) == cudaSuccess) ok = true;
    }
    ~DeviceGuard() {
        if (ok) cudaSetDevice(prev);
    }
};

// Fused mode, first step after an upload: deposits the present particles into
// the current electron density and both ion densities and clears the slot
// counters, on `stream`; sets dens_valid.
int state_prime_fused(cudapic_state *s, cudaStream_t stream);
// True when step `step` moves the ions (every N_SUB-th step of an RF period).
bool state_is_ion_step(const cudapic_state *s, uint64_t step);
// Device memory owned by the state (freed with it).
int state_alloc(cudapic_state *s, void **p, size_t bytes);
// Frees a buffer allocated by the state (no-op for memory it does not own).
void state_release(cudapic_state *s, void *p);
// Drops the captured CUDA graphs (after the state's buffers moved).
void state_drop_graphs(cudapic_state *s);
// Space- and time-averaged <j E> power of the electrons and ions from the
// XT diagnostics [W m^-3] (NaN without them), xt.cpp.
int xt_power(cudapic_state *s, double *power_e, double *power_i);

}  // namespace cudapic
