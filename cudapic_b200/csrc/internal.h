// internal.h -- host-side helpers shared by the entry points of libcudapic.
#pragma once

#include <cuda_runtime.h>

#include <cmath>
#include <cstdint>
#include <string>
#include <utility>
#include <vector>

#include "../../include/cudapic.h"

namespace cudapic {

// Records a message for cudapic_last_error() and returns `status`.
int fail(int status, const std::string &msg);
// Maps a CUDA error to CUDAPIC_ERR_CUDA with a message (OK stays OK).
int check_cuda(cudaError_t e, const char *what);
// Launch-error check after a <<<>>> launch.
int check_launch(const char *kernel);

// Number of SMs of the current device (cached per device).
int sm_count();
// Dynamic shared memory ceiling per block of the current device.
int max_smem_optin();

inline bool aligned16(const void *p) { return (reinterpret_cast<uintptr_t>(p) & 15u) == 0; }

// Validation shared by the entry points.
int validate_grid(const cudapic_grid *g);

// Current launch shapes (defaults filled in for zero fields).
cudapic_tuning tuning();
// Advanced by every cudapic_set_tuning: captured graphs baked the shapes of
// the generation they were captured in.
uint64_t tuning_generation();

// Programmatic dependent launch (PDL).  Inside a PdlScope the kernel
// launches of the calling thread carry cudaLaunchAttributeProgrammatic-
// StreamSerialization, so a kernel may be scheduled while the previous one
// drains.  Every kernel of this library executes grid_dep_wait()
// (common.cuh) before it reads or writes global data another kernel may
// touch, so only its prologue (shared-memory set-up, static tables) overlaps.
// The driver opens a scope around its own steps; the drop-in entry points
// never do, because a caller's preceding kernel may write what a prologue reads.
bool pdl_enabled();
struct PdlScope {
    bool prev;
    explicit PdlScope(bool on);
    ~PdlScope();
};

// Launches `kern` on `stream` (with the PDL attribute inside a PdlScope).
template <typename... KArgs, typename... Args>
int launch_kernel(const char *name, void (*kern)(KArgs...), dim3 grid, dim3 block, size_t smem, cudaStream_t stream,
                  Args &&...args) {
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = grid;
    cfg.blockDim = block;
    cfg.dynamicSmemBytes = smem;
    cfg.stream = stream;
    cudaLaunchAttribute attr[1];
    if (pdl_enabled()) {
        attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
        attr[0].val.programmaticStreamSerializationAllowed = 1;
        cfg.attrs = attr;
        cfg.numAttrs = 1;
    }
    const cudaError_t e = cudaLaunchKernelEx(&cfg, kern, std::forward<Args>(args)...);
    if (e != cudaSuccess) return check_cuda(e, name);
    return check_launch(name);
}

// Grid of a persistent kernel: min(SMs x per_sm, work units), at least 1.
unsigned persistent_grid(int per_sm, uint64_t units);

// Publishes a particle count at the end of a kernel without a separate copy
// node: the last CTA to finish (a ticket counter, zero between launches)
// stores min(*src, capacity) into *dst and, with clear_src, zeroes *src.
// ticket == nullptr: nothing published.
struct StepLink {
    uint32_t *ticket = nullptr;
    uint32_t *dst = nullptr;
    uint32_t *src = nullptr;
    int clear_src = 0;
};

// Launchers used by both the drop-in entry points and the driver.
// zero_a / zero_b (may be null): n_g-float buffers the kernel clears after
// reading the densities (the driver's next-step density accumulators).
int launch_poisson(const float *e_density, const float *i_density, float *pot, float *efield, float pot0,
                   const float *pot0_table, uint32_t *step_counter, const cudapic_grid &g, cudaStream_t stream,
                   float *zero_a = nullptr, float *zero_b = nullptr);
// Adjoint of launch_poisson's solve and field in FP64 (kernels_poisson.cu):
// eb (field adjoint, cleared) -> neb, nib_acc (density adjoints, the ion one
// accumulated unless reset_acc) and vbar += cosv * (pot0 adjoint).
int launch_poisson_adjoint(double *eb, double *neb, double *nib_acc, int reset_acc, double cosv, double *vbar,
                           const cudapic_grid &g, cudaStream_t stream);
// FP64 solve and field from FP64 node sums (kernels_poisson.cu, the all-FP64
// twin): pot0 from pot0_table[*step % n_t], *step advanced; measurement sums
// may be null.
int launch_poisson_f64(const double *dens_e, const double *dens_i, double *pot, double *efield,
                       const double *pot0_table, uint32_t *step, int ion_step, double *cumul_e, double *cumul_i,
                       double *pot_sum, const cudapic_grid &g, cudaStream_t stream);
// dens_out (may be null): also deposit the survivors' new positions there;
// wall (may be null): count the absorbed particles (with IFEDs for ions).
int launch_move_and_compact(const float *efield, const float *sx, const float *svx, const float *svy,
                            const float *svz, float *dx_, float *dvx, float *dvy, float *dvz, uint32_t *alive,
                            const uint32_t *n_active, float factor, float dt, const cudapic_grid &g,
                            cudaStream_t stream, float *dens_out = nullptr, const StepLink &link = StepLink(),
                            cudapic_wall_counters *wall = nullptr, bool wall_ions = false);
// True when `count` planes are 16-byte aligned and the capacity is a multiple
// of 4 (the bulk-copy tiles of the fused electron step).
bool electron_step_eligible(const void *const *planes, int count, uint32_t capacity);
// Fused electron step of the driver: push, compaction, collisions with the
// RNG stream of each particle's source slot, next-step deposit (kernels_step.cu).
// Returns CUDAPIC_ERR_NOT_SUPPORTED, recording nothing, when the buffers do not
// meet its alignment rules (the caller then runs push and collisions apart).
int launch_electron_step(const float *efield, const float *sx, const float *svx, const float *svy, const float *svz,
                         float *dx_, float *dvx, float *dvy, float *dvz, uint32_t *rng0, uint32_t *rng1,
                         uint32_t *rng2, uint32_t *rng3, const float *sigma_tot_e, const float *cs, float sigma_max_e,
                         float *ix, float *ivx, float *ivy, float *ivz, uint32_t *alive, const uint32_t *n_active,
                         uint32_t *n_i, float *dens_e, float *dens_i, const cudapic_grid &g, cudaStream_t stream,
                         const StepLink &link, cudapic_wall_counters *wall = nullptr,
                         unsigned long long *coll = nullptr);
// dep_e / dep_i (may be null): next-step densities receiving the spawns;
// coll (may be null): += collision events.
int launch_collisions_e(const float *total_cs_e, const float *cs, const uint32_t *active_e, float *x, float *vx,
                        float *vy, float *vz, uint32_t *rng0, uint32_t *rng1, uint32_t *rng2, uint32_t *rng3,
                        float *i_x, float *i_vx, float *i_vy, float *i_vz, uint32_t *alive_e, uint32_t *alive_i,
                        uint8_t *events, const cudapic_grid &g, cudaStream_t stream, float *dep_e = nullptr,
                        float *dep_i = nullptr, unsigned long long *coll = nullptr);
// ion_k: max(sigma_tot_i) dt_i rounded up (the ion test's certain-rejection
// bound, mcc.cuh ion_collides); +inf: every ion takes the full test.
int launch_collisions_i(const float *total_cs_i, const float *cs, const uint32_t *active_i, float *vx, float *vy,
                        float *vz, uint32_t *rng0, uint32_t *rng1, uint32_t *rng2, uint32_t *rng3, uint8_t *events,
                        const cudapic_grid &g, cudaStream_t stream, unsigned long long *coll = nullptr,
                        float ion_k = INFINITY);
// The bound ion_k for a table whose largest entry is sigma_max_i.
float ion_reject_k(float sigma_max_i, const cudapic_grid &g);
int launch_eepf(const float *x, const float *vx, const float *vy, const float *vz, const float *efield,
                const uint32_t *active_e, uint32_t *eepf, const cudapic_grid &g, cudaStream_t stream,
                double *esum = nullptr, unsigned long long *ecount = nullptr);

// XT diagnostics (kernels_xt.cu): steps per column (eduPIC's N_BIN) and the
// raw accumulators, each [n_g][n_xt] doubles, n_xt = N_T / XT_BIN.
constexpr uint32_t XT_BIN = 20;
enum XtRaw : int {
    XT_COUNT_E = 0, XT_UE, XT_MEANEE, XT_IONIZ,  // electron weights and weighted sums
    XT_COUNT_I, XT_UI, XT_MEANEI,                // ion weights and weighted sums
    XT_POT, XT_EFIELD, XT_NE, XT_NI,             // grid quantities
    XT_RAW
};
// Adds one species' particles (before the push) to the XT column of the step
// the Poisson kernel just solved.
int launch_xt_particles(bool ions, const float *x, const float *vx, const float *vy, const float *vz,
                        const uint32_t *n_active, const float *efield, const float *cs, const uint32_t *step_counter,
                        const cudapic_grid &g, uint32_t n_xt, double *xt, cudaStream_t stream);
// Adds the potential, field and densities of that step.
int launch_xt_grid(const float *pot, const float *efield, const float *e_density, const float *i_density,
                   const uint32_t *step_counter, const cudapic_grid &g, uint32_t n_xt, double *xt,
                   cudaStream_t stream);

// Largest electron / ion collision frequencies of the total tables [1/s]
// (C/eduPIC.cc:252-276) and the CFL energy limit [eV] (report.cpp).
void table_coll_freqs(const float *sigma_tot_e, const float *sigma_tot_i, double *max_e, double *max_i);
double cfl_max_energy(const cudapic_params &p);

// RNG sidecar of a checkpoint (<path>.rng, checkpoint.cpp): both species'
// four planes over `capacity` slots.  read: CUDAPIC_ERR_NOT_SUPPORTED,
// nothing recorded, when the file does not exist.
int rng_sidecar_write(const char *path, uint32_t capacity, const std::vector<uint32_t> planes[2][4]);
int rng_sidecar_read(const char *path, uint32_t capacity, std::vector<uint32_t> planes[2][4]);

// The in-place electron step (kernels_inplace.cu): the stream pass over
// [0, *n_active) -- electrons stay in their slots, absorbed ones are marked,
// colliders are recorded in `list` / *count -- and the scatter pass over the
// records (spawns appended at *n_e and *n_i; its last CTA adds the
// collision count to *coll and clears *count and *ticket).  spawn_from (may
// be null): receives the slot count the stream pass saw.
struct InplacePlanes;
struct CollList;
int launch_electron_inplace(const InplacePlanes &pl, const float *efield, const float *sigma_tot_e, const float *cs,
                            float sigma_max, const uint32_t *n_active, const CollList &list, uint32_t *count,
                            float *dens_e,
                            const cudapic_grid &g, cudaStream_t stream, cudapic_wall_counters *wall,
                            uint32_t *spawn_from);
// The next step's Poisson solve (launch_poisson's arguments), run by the
// last CTA of the scatter pass once every CTA has added its spawns.
struct PoissonAhead {
    const float *e_density, *i_density;
    float *pot, *efield;
    const float *pot0_table;
    uint32_t *step_counter;
    float *zero_a, *zero_b;
};
// Largest grid the scatter pass can solve (one node per thread of its
// 1024-thread CTAs, the separate solve kernel's shape up to this size).
constexpr uint32_t POISSON_AHEAD_MAX_NG = 1024;
int launch_electron_scatter(const InplacePlanes &pl, const CollList &list, const float *cs, uint32_t *count,
                            uint32_t *ticket, uint32_t *n_e, uint32_t *n_i, const cudapic_grid &g,
                            cudaStream_t stream, float *dens_e, float *dens_i, unsigned long long *coll,
                            const PoissonAhead *ahead = nullptr);
// eduPIC's same-step collisions of new electrons: one CTA tests and scatters
// the electrons appended since *spawn_from (written by the stream pass).
int launch_spawn_collide(const InplacePlanes &pl, const float *sigma_tot_e, const float *cs,
                         const uint32_t *spawn_from, uint32_t *n_e, uint32_t *n_i, const cudapic_grid &g,
                         cudaStream_t stream, float *dens_e, float *dens_i, unsigned long long *coll);

// One CTA whose bounded mbarrier wait runs out after `limit` SM clocks and
// sets CUDAPIC_DEVERR_TIMEOUT in dev_err (kernels_misc.cu).
int launch_wait_timeout_probe(uint32_t *dev_err, long long limit, cudaStream_t stream);

}  // namespace cudapic

#define CUDAPIC_CHECK(expr)                                   \
    do {                                                      \
        int _rc = (expr);                                     \
        if (_rc != CUDAPIC_OK) return _rc;                    \
    } while (0)

#define CUDAPIC_REQUIRE(cond, msg)                                   \
    do {                                                             \
        if (!(cond)) return ::cudapic::fail(CUDAPIC_ERR_ARG, (msg)); \
    } while (0)
