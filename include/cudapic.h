/*
 * cudapic.h -- C ABI of libcudapic.so, the B200 (sm_100a) implementation of
 * cudaPIC's per-timestep PIC/MCC cycle (1d3v argon CCP, eduPIC physics).
 *
 * Two layers:
 *
 *  1. Drop-in kernel entry points.  One function per reference kernel of the
 *     cuda-oxide module `kernels` (Rust-CUDA/src/main.rs:352-1358), with the
 *     reference's argument order.  The reference bakes the discharge
 *     constants in at compile time (Rust-CUDA/src/main.rs:29-110); here they
 *     travel in a `cudapic_grid` built once by cudapic_grid_from_params().
 *     All pointers are device pointers owned by the caller; no entry point
 *     allocates device memory or synchronises; every launch goes to the
 *     caller's stream.  Counters (n_active, alive_counter, ...) stay in
 *     device memory exactly as in the reference, so a sequence of calls
 *     never needs the host to read a count.
 *
 *  2. A simulation state (`cudapic_state`) that owns the SoA buffers, the
 *     cross-section tables and the RNG planes (the reference's GpuSimState,
 *     Rust-CUDA/src/main.rs:131-350) and runs the reference's per-step loop
 *     (Rust-CUDA/src/main.rs:1725-1808) from CUDA graphs.
 *
 * Every function returns a cudapic_status.  Kernels never trap: device-side
 * problems (spawn beyond capacity, a particle outside [0, L]) set bits of a
 * device error word (cudapic_grid.dev_err) and the offending write is
 * skipped.  cudapic_last_error() returns a message for the last failure of
 * the calling thread.
 */
#ifndef CUDAPIC_H
#define CUDAPIC_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define CUDAPIC_VERSION 100

/* Same object as cudaStream_t (the CUDA runtime's stream handle). */
typedef struct CUstream_st *cudapic_stream_t;

typedef enum cudapic_status {
    CUDAPIC_OK = 0,
    CUDAPIC_ERR_CUDA = 1,          /* a CUDA runtime call failed                  */
    CUDAPIC_ERR_CAPACITY = 2,      /* a device error word reports a capacity hit  */
    CUDAPIC_ERR_ARG = 3,           /* invalid argument (null, size, alignment)    */
    CUDAPIC_ERR_TIMEOUT = 4,       /* a bounded device wait gave up               */
    CUDAPIC_ERR_NOT_SUPPORTED = 5, /* device is not sm_100 / feature unavailable  */
    CUDAPIC_ERR_STATE = 6          /* call out of order on a cudapic_state        */
} cudapic_status;

/* Bits of the device error word. */
#define CUDAPIC_DEVERR_SPAWN_E  0x1u  /* electron spawn dropped: capacity reached   */
#define CUDAPIC_DEVERR_SPAWN_I  0x2u  /* ion spawn dropped: capacity reached        */
#define CUDAPIC_DEVERR_POSITION 0x4u  /* gather/deposit met x outside [0,L] or NaN  */
#define CUDAPIC_DEVERR_ACTIVE   0x8u  /* a count exceeded capacity and was clamped  */
#define CUDAPIC_DEVERR_TIMEOUT  0x10u /* a bounded wait on an async copy gave up    */
#define CUDAPIC_DEVERR_RECORDS  0x20u /* sensitivity tape: collision records full    */

/* Discharge and run parameters: the reference's compile-time constants
 * (Rust-CUDA/src/main.rs:40-50, :79) as runtime values. */
typedef struct cudapic_params {
    uint32_t n_g;            /* grid points, 3..16384                        */
    uint32_t n_t;            /* time steps per RF period                     */
    uint32_t n_sub;          /* ion subcycling factor                        */
    uint32_t capacity;       /* preallocated particles per species           */
    double frequency;        /* RF frequency [Hz]                            */
    double voltage;          /* RF amplitude [V]                             */
    double gap;              /* electrode gap L [m]                          */
    double pressure;         /* gas pressure [Pa]                            */
    double temperature;      /* gas temperature [K]                          */
    double weight;           /* superparticle weight                         */
    double electrode_area;   /* electrode area [m^2]                         */
    uint32_t flags;          /* CUDAPIC_FLAG_*                               */
} cudapic_params;

/* Poisson prefix sums in f32 as the reference does (default: FP64 sums,
 * f32 inputs/outputs). */
#define CUDAPIC_FLAG_POISSON_F32_SCAN 0x1u
/* Deposit arithmetic.  Default: CIC weights in 2^-20 fixed point summed
 * with 32-bit integer shared atomics (exact, order-independent sums inside a
 * thread-block cluster; a weight carries a quantum of 2^-21, below the f32
 * rounding of x * inv_dx; the fastest shared atomic on B200).
 * FIXED_POINT: 32.32 fixed-point weights summed with 64-bit shared atomics.
 * F32: the reference's f32 weights summed with shared f32 atomics.  Where
 * both are set, FIXED_POINT wins.  The fused deposits of the driver step
 * (cudapic_move_and_compact_deposit, cudapic_step_electrons) always use the
 * default arithmetic. */
#define CUDAPIC_FLAG_DEPOSIT_FIXED_POINT 0x2u
#define CUDAPIC_FLAG_DEPOSIT_F32 0x4u

/* Derived per-discharge constants handed to every drop-in kernel (by value
 * on the kernel side).  Built by cudapic_grid_from_params(); the fields are
 * the reference's `X as Real` constants (Rust-CUDA/src/main.rs:53-109). */
typedef struct cudapic_grid {
    uint32_t n_g;
    uint32_t capacity;
    uint32_t n_t;
    uint32_t n_sub;
    uint32_t flags;
    float inv_dx;
    float weight_factor;
    float gap;
    float dt_e, dt_i;
    float factor_e, factor_i;
    float e_charge;
    float alpha;
    float half_dx_over_eps;
    float half_inv_dx;
    float normal_range;
    float f1, f2;
    float half_me_over_e;
    float half_mu_over_e;
    float min_x, max_x;
    float eepf_half_kick;
    double dx;
    double weight_factor_d;
    double gas_density;
    double voltage;
    uint32_t *dev_err;             /* device error word (may be NULL)          */
    unsigned long long *work;      /* device particle-step counter (may be NULL) */
} cudapic_grid;

void cudapic_params_default(cudapic_params *p);
int cudapic_grid_from_params(const cudapic_params *p, cudapic_grid *out);

/* Launch shapes of the kernels (process-wide; set it before launching, not
 * concurrently with launches).  Zero fields keep the built-in choice.
 * The reference has no counterpart: its shapes are compile-time constants
 * (Rust-CUDA/src/main.rs:84-88).  cudapic_b200.autotune sweeps these. */
typedef struct cudapic_tuning {
    int density_threads;      /* get_density CTA size: 256, 512 or 1024                 */
    int density_ctas_per_sm;  /* resident CTAs per SM used (<= occupancy)               */
    int density_copies;       /* warp-private shared histogram copies per CTA (1..32)    */
    int density_cluster;      /* CTAs per thread-block cluster for the reduction: 1,2,4,8 */
    int push_stages;          /* move_and_compact bulk-copy pipeline depth: 2..6         */
    int push_ctas_per_sm;
    int mcc_stages;           /* check_collisions_e/i pipeline depth: 2..4               */
    int mcc_ctas_per_sm;
    int mcc_variant;          /* 1: shared-memory resident sigma table (any alignment),
                                 2: bulk-copy staged tiles (16-byte aligned pointers)    */
    int step_stages;          /* fused electron step bulk-copy pipeline depth: 2..6      */
    int step_ctas_per_sm;
    int step_rows;            /* fused electron step particles per thread and tile: 1, 2, 4 */
    int inplace_ctas_per_sm;  /* in-place electron step: resident CTAs per SM used          */
    int inplace_copies;       /* in-place electron step: fixed-point deposit histogram copies
                                 (1..8), -1: one f32 shared histogram                     */
    int inplace_prefetch;     /* in-place electron step: rounds of a CTA's slots prefetched
                                 into L2 ahead of their loads (1..4), -1: none             */
    int scatter_ctas_per_sm;  /* in-place electron step, scatter pass: CTAs per SM (1..8)   */
} cudapic_tuning;

int cudapic_get_tuning(cudapic_tuning *out);
int cudapic_set_tuning(const cudapic_tuning *t);
const char *cudapic_status_string(int status);
const char *cudapic_last_error(void);
int cudapic_version(void);

/* ------------------------------------------------------------------ */
/* 1. drop-in kernels                                                  */
/* ------------------------------------------------------------------ */

/* get_density (Rust-CUDA/src/main.rs:356-406): CIC deposit of x[0..*n_active)
 * ADDED to density[n_g] (pre-zero it, as the reference's loop does at :1729).
 * Boundary nodes receive double weight. */
int cudapic_get_density(const float *x, float *density, const uint32_t *n_active,
                        const cudapic_grid *grid, cudapic_stream_t stream);

/* solve_poisson_scan_f32 (Rust-CUDA/src/main.rs:408-494): potential with
 * pot[0] = pot0, pot[n_g-1] = 0 and the field, from the two densities.
 * One CTA; FP64 prefix sums unless CUDAPIC_FLAG_POISSON_F32_SCAN. */
int cudapic_solve_poisson_scan_f32(const float *e_density, const float *i_density, float *pot,
                                   float *efield, float pot0, const cudapic_grid *grid,
                                   cudapic_stream_t stream);

/* solve_poisson_dps_flexible (Rust-CUDA/src/main.rs:496-564): psi'' = source
 * on n nodes spaced dx with psi[0] = psi_left, psi[n-1] = psi_right. */
int cudapic_solve_poisson_dps_flexible(const float *source, float *pot, uint32_t n, float psi_left,
                                       float psi_right, float dx, cudapic_stream_t stream);

/* move_and_compact (Rust-CUDA/src/main.rs:566-678): leapfrog push of
 * src[0..*n_active), survivors (0 <= x' <= L) appended to dst at
 * atomicAdd(alive_counter).  Survivor order is unspecified across blocks, as
 * in the reference.  src and dst must not overlap; all particle pointers
 * 16-byte aligned. */
int cudapic_move_and_compact(const float *efield, const float *src_x, const float *src_vx,
                             const float *src_vy, const float *src_vz, float *dst_x, float *dst_vx,
                             float *dst_vy, float *dst_vz, uint32_t *alive_counter,
                             const uint32_t *n_active, float factor, float dt,
                             const cudapic_grid *grid, cudapic_stream_t stream);

/* move_and_compact fused with the next step's deposit: as
 * cudapic_move_and_compact, and the CIC weights of every survivor's new
 * position are ADDED to next_density[n_g] (boundary nodes doubled), i.e.
 * get_density(dst) without re-reading the particles.  No reference
 * counterpart: the reference recomputes the density from the particles at
 * the start of every step (Rust-CUDA/src/main.rs:1729-1739), which gives
 * the same values because collisions do not move particles. */
int cudapic_move_and_compact_deposit(const float *efield, const float *src_x, const float *src_vx,
                                     const float *src_vy, const float *src_vz, float *dst_x, float *dst_vx,
                                     float *dst_vy, float *dst_vz, uint32_t *alive_counter,
                                     const uint32_t *n_active, float factor, float dt, float *next_density,
                                     const cudapic_grid *grid, cudapic_stream_t stream);

/* check_collisions_e (Rust-CUDA/src/main.rs:971-1165): MCC of electrons
 * [0, *active_e) against the gas; ionization appends an electron at
 * atomicAdd(alive_e) and an ion at atomicAdd(alive_i) (bounded by capacity).
 * total_cs_e[1e6], cs[5*1e6] are the tables of cudapic_cross_sections(). */
int cudapic_check_collisions_e(const float *total_cs_e, const float *cs, const uint32_t *active_e,
                               float *x, float *vx, float *vy, float *vz, uint32_t *rng0,
                               uint32_t *rng1, uint32_t *rng2, uint32_t *rng3, float *i_x,
                               float *i_vx, float *i_vy, float *i_vz, uint32_t *alive_e,
                               uint32_t *alive_i, const cudapic_grid *grid,
                               cudapic_stream_t stream);

/* check_collisions_e whose spawned electrons / ions are also deposited
 * into e_next_density / i_next_density (either may be NULL), completing the
 * next-step densities of cudapic_move_and_compact_deposit.  No reference
 * counterpart (see there). */
int cudapic_check_collisions_e_deposit(const float *total_cs_e, const float *cs, const uint32_t *active_e,
                                       float *x, float *vx, float *vy, float *vz, uint32_t *rng0,
                                       uint32_t *rng1, uint32_t *rng2, uint32_t *rng3, float *i_x, float *i_vx,
                                       float *i_vy, float *i_vz, uint32_t *alive_e, uint32_t *alive_i,
                                       float *e_next_density, float *i_next_density, const cudapic_grid *grid,
                                       cudapic_stream_t stream);

/* Fused electron step: one launch doing the work of move_and_compact
 * (Rust-CUDA/src/main.rs:566-678), check_collisions_e (:971-1165) and the
 * next step's get_density (:356-406); no single reference counterpart.
 * Electron k of src[0, *n_e) is pushed in `efield` (factor_e, dt_e of the
 * grid); a survivor is tested for a collision with the RNG stream of slot k
 * (the planes are updated in place), scattered, and written with any
 * spawned electron to dst[0, *alive_counter) (*alive_counter must be 0 on
 * entry; order unspecified); spawned ions are appended at *n_i (bounded by
 * capacity).  Survivors and spawned electrons are added to e_next_density,
 * spawned ions to i_next_density (both accumulate).  sigma_max_e must be
 * the largest entry of total_cs_e: it bounds the collision probability so
 * that most electrons skip the table (decisions are bit-identical).  The
 * eight planes must be 16-byte aligned and the capacity a multiple of 4. */
int cudapic_step_electrons(const float *efield, const float *src_x, const float *src_vx, const float *src_vy,
                           const float *src_vz, float *dst_x, float *dst_vx, float *dst_vy, float *dst_vz,
                           uint32_t *rng0, uint32_t *rng1, uint32_t *rng2, uint32_t *rng3, const float *total_cs_e,
                           const float *cs, float sigma_max_e, float *i_x, float *i_vx, float *i_vy, float *i_vz,
                           uint32_t *alive_counter, const uint32_t *n_e, uint32_t *n_i, float *e_next_density,
                           float *i_next_density, const cudapic_grid *grid, cudapic_stream_t stream);

/* The electron step in place (no reference counterpart: the electron half
 * of the reference's step, move_and_compact + check_collisions_e + the next
 * get_density, Rust-CUDA/src/main.rs:566-678, 971-1165, 356-406, with every
 * electron kept in its slot).  Two launches:
 *  - cudapic_step_electrons_inplace pushes electrons [0, *n_e), tests them
 *    for collision (one draw of each slot's stream) and deposits the
 *    survivors' new positions ADDED to e_next_density; x, vx and the RNG
 *    state are written back to the same slots (vy, vz unchanged).  An
 *    electron that leaves through an electrode is marked in its slot with
 *    x = -1 (CUDAPIC_DEAD_X): later in-place steps skip such slots, and
 *    cudapic_step_electrons drops them while compacting.  Each collider is
 *    recorded in the eight planes coll[0..7] (capacity entries each: slot,
 *    with bit 31 set for an ionization, vx, vy, vz, then the four words of
 *    its RNG state past the test draw; capacity at most 2^31) and counted
 *    in *n_colliders (zero on entry); the RNG state written to
 *    a collider's slot is already the one past all of its scattering's
 *    draws (the event draw, made here from cs, tells how many).  *n_e is
 *    unchanged.
 *  - cudapic_scatter_colliders_e scatters the recorded colliders in place,
 *    continuing each recorded stream (collision_e) and writing the velocity
 *    back to the slots (not the RNG state: the stream pass wrote it);
 *    spawned electrons take slots *n_e, *n_e + 1, ... (updating *n_e),
 *    spawned ions slots *n_i, ... of i_*; both are deposited into the next
 *    densities.  Its last CTA resets *n_colliders and *ticket (zero on
 *    entry) to zero.
 * Same plane alignment and capacity rules as cudapic_step_electrons. */
#define CUDAPIC_DEAD_X (-1.0f)
int cudapic_step_electrons_inplace(const float *efield, float *x, float *vx, const float *vy, const float *vz,
                                   uint32_t *rng0, uint32_t *rng1, uint32_t *rng2, uint32_t *rng3,
                                   const float *total_cs_e, const float *cs, float sigma_max_e, const uint32_t *n_e,
                                   uint32_t *const coll[8], uint32_t *n_colliders, float *e_next_density,
                                   const cudapic_grid *grid, cudapic_stream_t stream);
int cudapic_scatter_colliders_e(float *x, float *vx, float *vy, float *vz, uint32_t *rng0, uint32_t *rng1,
                                uint32_t *rng2, uint32_t *rng3, const float *cs, uint32_t *const coll[8],
                                uint32_t *n_colliders, uint32_t *ticket, float *i_x, float *i_vx, float *i_vy,
                                float *i_vz, uint32_t *n_e, uint32_t *n_i, float *e_next_density,
                                float *i_next_density, const cudapic_grid *grid, cudapic_stream_t stream);

/* cudapic_step_electrons for callers that cannot allocate device memory
 * (a host whose device memory belongs to its own pool or framework and that
 * hands this library only its particle buffers, or code that must not call
 * cudaMalloc because it synchronises the device).  It has no counterpart in
 * the reference.  Same arguments and results as cudapic_step_electrons
 * except that no alive_counter is passed: the kernel's slot counter and
 * completion ticket live in a library-owned static device array of
 * CUDAPIC_NOALLOC_SCRATCH_BYTES (held by every GPU that loads the library
 * until exit), and the new electron count is written into *n_e in place.
 * The call allocates nothing; it clears the two counters on `stream` before
 * the launch.  Every call looks up the array's address in the calling
 * thread's current context (so a non-primary context, or the module that a
 * cudaDeviceReset reloads, gets its own array); the first call on a device
 * may load the library's module, so make it before any stream capture.
 * Every call shares
 * the array: calls whose kernels overlap on one GPU race.  Rejects (with
 * CUDAPIC_ERR_ARG) a capacity above CUDAPIC_NOALLOC_MAX_CAPACITY, where the
 * shared 32-bit slot counter could wrap, besides the checks of
 * cudapic_step_electrons. */
#define CUDAPIC_NOALLOC_SCRATCH_BYTES 256u
#define CUDAPIC_NOALLOC_MAX_CAPACITY 0x80000000u
int cudapic_step_electrons_noalloc(const float *efield, const float *src_x, const float *src_vx,
                                   const float *src_vy, const float *src_vz, float *dst_x, float *dst_vx,
                                   float *dst_vy, float *dst_vz, uint32_t *rng0, uint32_t *rng1, uint32_t *rng2,
                                   uint32_t *rng3, const float *total_cs_e, const float *cs, float sigma_max_e,
                                   float *i_x, float *i_vx, float *i_vy, float *i_vz, uint32_t *n_e, uint32_t *n_i,
                                   float *e_next_density, float *i_next_density, const cudapic_grid *grid,
                                   cudapic_stream_t stream);

/* check_collisions_i (Rust-CUDA/src/main.rs:1167-1292): MCC of ions
 * [0, *active_i) against Maxwellian target atoms. */
int cudapic_check_collisions_i(const float *total_cs_i, const float *cs, const uint32_t *active_i,
                               float *vx, float *vy, float *vz, uint32_t *rng0, uint32_t *rng1,
                               uint32_t *rng2, uint32_t *rng3, const cudapic_grid *grid,
                               cudapic_stream_t stream);

/* Same as the two above, also writing the collision event of every particle
 * to events[0..*active) (0 none, 1 elastic, 2 excitation, 3 ionization;
 * 4 isotropic, 5 backscatter for ions).  No reference counterpart: a
 * diagnostic used by the parity tests. */
int cudapic_check_collisions_e_events(const float *total_cs_e, const float *cs,
                                      const uint32_t *active_e, float *x, float *vx, float *vy,
                                      float *vz, uint32_t *rng0, uint32_t *rng1, uint32_t *rng2,
                                      uint32_t *rng3, float *i_x, float *i_vx, float *i_vy,
                                      float *i_vz, uint32_t *alive_e, uint32_t *alive_i,
                                      uint8_t *events, const cudapic_grid *grid,
                                      cudapic_stream_t stream);
int cudapic_check_collisions_i_events(const float *total_cs_i, const float *cs,
                                      const uint32_t *active_i, float *vx, float *vy, float *vz,
                                      uint32_t *rng0, uint32_t *rng1, uint32_t *rng2,
                                      uint32_t *rng3, uint8_t *events, const cudapic_grid *grid,
                                      cudapic_stream_t stream);

/* cudapic_check_collisions_i with the largest entry of total_cs_i given
 * (sigma_max_i), as cudapic_step_electrons takes sigma_max_e: an ion whose
 * test draw lies above a bound on its collision probability over every
 * target atom the draws can give skips the target's Box-Muller
 * transcendentals (its RNG state advances past the same five draws), so
 * results are identical to cudapic_check_collisions_i's and most ions cost
 * a few integer operations.  events may be NULL.  No reference counterpart;
 * the state drivers use it. */
int cudapic_check_collisions_i_bounded(const float *total_cs_i, const float *cs, const uint32_t *active_i,
                                       float *vx, float *vy, float *vz, uint32_t *rng0, uint32_t *rng1,
                                       uint32_t *rng2, uint32_t *rng3, float sigma_max_i, uint8_t *events,
                                       const cudapic_grid *grid, cudapic_stream_t stream);

/* accumulate_density (Rust-CUDA/src/main.rs:1294-1299): cumul[k] += density[k]. */
int cudapic_accumulate_density(const float *density, double *cumul, const cudapic_grid *grid,
                               cudapic_stream_t stream);

/* accumulate_eepf (Rust-CUDA/src/main.rs:1301-1339): EEPF histogram
 * (2000 bins of 0.05 eV) of electrons in (0.45 L, 0.55 L). */
int cudapic_accumulate_eepf(const float *x, const float *vx, const float *vy, const float *vz,
                            const float *efield, const uint32_t *active_e, uint32_t *eepf,
                            const cudapic_grid *grid, cudapic_stream_t stream);

/* xoshiro128p_test_wrapper (Rust-CUDA/src/main.rs:1341-1357): one step from
 * (s0..s3); dest[0] = output, dest[1..4] = next state. */
int cudapic_xoshiro128p_test_wrapper(uint32_t s0, uint32_t s1, uint32_t s2, uint32_t s3,
                                     uint32_t *dest, cudapic_stream_t stream);

/* xoshiro128_seed_streams (Rust-CUDA/src/main.rs:1446-1496), on the GPU:
 * stream k = master after k jumps of 2^64, written to the four planes.
 * n <= 2^28. */
int cudapic_xoshiro128_seed_streams(const uint32_t master[4], uint32_t n, uint32_t *rng0,
                                    uint32_t *rng1, uint32_t *rng2, uint32_t *rng3,
                                    cudapic_stream_t stream);

/* init_cross_sections (Rust-CUDA/src/main.rs:1378-1444), on the host:
 * cs[5*1e6] (elastic, excitation, ionization, ion isotropic, ion backward)
 * and the total macroscopic tables for the given gas density.  Host
 * pointers.  Uses all host threads. */
#define CUDAPIC_CS_RANGES 1000000u
int cudapic_cross_sections(double gas_density, float *cs, float *sigma_tot_e, float *sigma_tot_i);

/* Particles absorbed at the electrodes (C/eduPIC.cc:623-667; the GPU
 * reference keeps none, Rust-CUDA has no counterpart): a particle whose
 * pushed position is x < 0 counts at the powered electrode, x > L at the
 * grounded one.  Ions also add their energy 1/2 M v^2 / e (f32, v after the
 * push) to the ion flux-energy distribution of that electrode: 1 eV bins,
 * energies of 200 eV and above not binned (C/eduPIC.cc:118-119, 645-657).
 * A device-memory block; the counters only grow (zero it to restart). */
#define CUDAPIC_N_IFED 200
typedef struct cudapic_wall_counters {
    unsigned long long abs_pow;          /* absorbed at x < 0 (powered electrode)  */
    unsigned long long abs_gnd;          /* absorbed at x > L (grounded electrode) */
    uint32_t ifed_pow[CUDAPIC_N_IFED];   /* ions: counts per 1 eV energy bin       */
    uint32_t ifed_gnd[CUDAPIC_N_IFED];
} cudapic_wall_counters;

/* move_and_compact that also counts the absorbed particles into `wall`
 * (device pointer); ions != 0 also fills its IFEDs.  No single reference
 * counterpart: the boundary check of C/eduPIC.cc:623-667 fused into the push. */
int cudapic_move_and_compact_wall(const float *efield, const float *src_x, const float *src_vx,
                                  const float *src_vy, const float *src_vz, float *dst_x, float *dst_vx,
                                  float *dst_vy, float *dst_vz, uint32_t *alive_counter, const uint32_t *n_active,
                                  float factor, float dt, cudapic_wall_counters *wall, int ions,
                                  const cudapic_grid *grid, cudapic_stream_t stream);

/* Evaluates the kernels' f32 transcendental functions on device arrays
 * (fn: 0 exp, 1 log, 2 sin, 3 cos, 4 tan, 5 atan, 6 acos, 7 atan2(in, in2)).
 * No reference counterpart: a diagnostic for the bit-exactness tests. */
int cudapic_math_eval(int fn, const float *in, const float *in2, float *out, uint32_t n,
                      cudapic_stream_t stream);

/* eduPIC's particle checkpoint file picdata.bin (save_particle_data /
 * load_particle_data, C/eduPIC.cc:726-781): doubles [Time, cycles_done, N_e,
 * x_e[N_e], vx_e, vy_e, vz_e, N_i, x_i[N_i], vx_i, vy_i, vz_i].  Host
 * pointers; e[4] / i[4] are the x, vx, vy, vz planes.  Writing widens the
 * f32 values exactly; reading rounds to the nearest f32; read rejects
 * (CUDAPIC_ERR_CAPACITY) more particles than max_e / max_i. */
int cudapic_picdata_write(const char *path, double time, uint32_t cycles_done, const float *const e[4],
                          uint32_t n_e, const float *const i[4], uint32_t n_i);
int cudapic_picdata_read_header(const char *path, double *time, uint32_t *cycles_done, uint32_t *n_e,
                                uint32_t *n_i);
int cudapic_picdata_read(const char *path, float *const e[4], uint32_t max_e, float *const i[4],
                         uint32_t max_i);

/* The accuracy conditions that follow from the parameters alone
 * (check_and_save_info, C/eduPIC.cc:925-1030): the largest collision
 * frequency of the cross-section tables times the time step, for electrons
 * and ions (each OK below 0.05; max_electron_coll_freq / max_ion_coll_freq,
 * :252-276), and the largest electron energy [eV] for which the CFL
 * condition holds.  Host only; lets a parameter sweep flag a discharge
 * before it runs.  conditions_ok: both frequencies within their bound. */
typedef struct cudapic_precheck {
    double max_e_coll_dt_e;
    double max_i_coll_dt_i;
    double cfl_max_energy;
    int conditions_ok;
} cudapic_precheck;
int cudapic_stability_precheck(const cudapic_params *p, cudapic_precheck *out);

/* ------------------------------------------------------------------ */
/* 2. simulation state and driver                                      */
/* ------------------------------------------------------------------ */

typedef struct cudapic_state cudapic_state;

/* Device pointers of a state (current ping-pong side). */
typedef struct cudapic_buffers {
    float *x[2], *vx[2], *vy[2], *vz[2];     /* [0] electrons, [1] ions            */
    float *tmp_x[2], *tmp_vx[2], *tmp_vy[2], *tmp_vz[2];
    uint32_t *rng[2][4];
    uint32_t *n_electrons, *n_ions, *alive_counter;
    float *efield, *pot, *e_density, *i_density;
    float *cs, *sigma_tot_e, *sigma_tot_i;
    double *cumul_e_density, *cumul_i_density;
    uint32_t *eepf;
    uint32_t *dev_err;
    unsigned long long *work;
    float sigma_max_e;                       /* largest entry of sigma_tot_e        */
} cudapic_buffers;

#define CUDAPIC_ELECTRONS 0
#define CUDAPIC_IONS 1

/* Allocates every buffer on `device`, builds the cross-section tables,
 * zeroes counters.  The state launches on its own non-blocking stream
 * unless cudapic_state_set_stream() is called. */
int cudapic_state_create(const cudapic_params *p, int device, cudapic_state **out);
int cudapic_state_destroy(cudapic_state *s);
int cudapic_state_set_stream(cudapic_state *s, cudapic_stream_t stream);
cudapic_stream_t cudapic_state_stream(const cudapic_state *s);
int cudapic_state_grid(const cudapic_state *s, cudapic_grid *out);
int cudapic_state_buffers(const cudapic_state *s, cudapic_buffers *out);

/* Host <-> device particle transfer (host pointers; pinned memory gives
 * asynchronous copies).  upload sets the species count to n. */
int cudapic_state_upload(cudapic_state *s, int species, const float *x, const float *vx,
                         const float *vy, const float *vz, uint32_t n);
/* Copies min(count, max_n) particles; *n_out = device count (synchronises). */
int cudapic_state_download(cudapic_state *s, int species, float *x, float *vx, float *vy,
                           float *vz, uint32_t max_n, uint32_t *n_out);
/* Seeds both species' RNG planes from master states (all capacity slots). */
int cudapic_state_seed(cudapic_state *s, const uint32_t e_master[4], const uint32_t i_master[4]);
/* Zeroes the measurement accumulators and turns per-step measurement on/off
 * (accumulate_density + accumulate_eepf, Rust-CUDA/src/main.rs:1746-1756, 1802-1807). */
int cudapic_state_set_measure(cudapic_state *s, int on);
/* Enqueues n_steps reference-order time steps (Rust-CUDA/src/main.rs:1728-1807)
 * on the state's stream.  Asynchronous. */
int cudapic_state_run_steps(cudapic_state *s, uint64_t n_steps);
/* on (default): each step runs the fused electron kernel
 * (cudapic_step_electrons: push, collisions and the next step's deposit in
 * one launch, electrons drawing from their source slot's RNG stream) and the
 * ion push deposits the ions' next density (cudapic_move_and_compact_deposit);
 * the kernels publish the particle counts themselves.  The first step after
 * an upload runs the separate deposit.  Planes that are not 16-byte aligned
 * (or a capacity that is not a multiple of 4) fall back to push + deposit and
 * cudapic_check_collisions_e_deposit.  off: the reference's launch sequence. */
int cudapic_state_set_fused(cudapic_state *s, int on);
/* Fused mode, on (default): between compacting steps the electrons are
 * stepped in place (cudapic_step_electrons_inplace + cudapic_scatter_
 * colliders_e: no compaction, absorbed electrons marked in their slots,
 * spawns appended).  The step before every N_SUB-th step and the last step
 * of every cudapic_state_run_steps call run the compacting fused kernel,
 * which drops the marked slots, so the planes are compact between calls.
 * off: every step compacts.  The captured graphs are rebuilt. */
int cudapic_state_set_inplace(cudapic_state *s, int on);
/* off (default): electrons spawned by an ionization are first tested for
 * collision in the next step, as in the reference's GPU path
 * (Rust-CUDA/src/main.rs:992).  on: eduPIC's semantics -- they are tested
 * (and may collide and ionize again) in the step of their birth
 * (C/eduPIC.cc:669-703).  Applies to the in-place steps (all but one step in
 * N_SUB); the compacting steps keep the reference's semantics. */
int cudapic_state_set_spawn_collide(cudapic_state *s, int on);
/* on (default): an in-place step whose successor is in the same run (not
 * the last step of a cudapic_state_run_steps call or graph) solves the
 * successor's Poisson problem in the last CTA of its scatter pass, after the
 * step's last deposit, instead of in a kernel of its own at the start of the
 * successor; the same solve on the same densities (N_G <= 1024; not while
 * measuring or with spawn collisions, whose kernels read this step's field
 * or add to the densities after the scatter pass).  off: one solve kernel
 * per step.  The captured graphs are rebuilt. */
int cudapic_state_set_solve_ahead(cudapic_state *s, int on);
/* on (default): the driver launches its kernels with programmatic dependent
 * launch, so a kernel's launch and prologue overlap the previous kernel's
 * tail (every kernel waits for its predecessor before touching global data).
 * off: plain stream order.  The captured graphs are rebuilt. */
int cudapic_state_set_overlap(cudapic_state *s, int on);
/* on (default when N_T is a multiple of N_SUB): run_steps replays captured
 * CUDA graphs of 2 N_SUB steps.  off: every step is launched from the host,
 * as the reference's driver does (Rust-CUDA/src/main.rs:1725-1808). */
int cudapic_state_set_graphs(cudapic_state *s, int on);
/* Reads the counters (synchronises the state's stream). */
int cudapic_state_counts(cudapic_state *s, uint32_t *n_e, uint32_t *n_i);
/* Reads and returns the device error word (synchronises). */
int cudapic_state_device_error(cudapic_state *s, uint32_t *bits);
/* Clears the state's device error word (on its stream), e.g. after a
 * capacity overflow was handled by re-uploading the particles. */
int cudapic_state_clear_device_error(cudapic_state *s);
/* Self-test of the bounded device waits (no reference counterpart; the
 * reference has no device-side error reporting): enqueues on the state's
 * stream one CTA that arms an mbarrier for a transfer no copy delivers and
 * waits on it for at most limit_cycles SM clocks (1 .. 2^31), so the wait
 * runs out and CUDAPIC_DEVERR_TIMEOUT is set in the state's device error
 * word; cudapic_state_device_error then returns CUDAPIC_ERR_TIMEOUT.  The
 * context stays usable; the state's error word keeps the bit. */
int cudapic_state_debug_wait_timeout(cudapic_state *s, long long limit_cycles);
/* Particle-steps processed so far (electrons each step, ions each N_SUB). */
int cudapic_state_work(cudapic_state *s, unsigned long long *particle_steps);
int cudapic_state_steps_done(const cudapic_state *s, uint64_t *steps);
int cudapic_state_synchronize(cudapic_state *s);
int cudapic_state_download_measurements(cudapic_state *s, double *cumul_e, double *cumul_i,
                                        uint32_t *eepf);
/* The electrode counters of the measurement window (zeroed by
 * cudapic_state_set_measure(s, 1)): out[0] electrons, out[1] ions, host
 * memory (synchronises). */
int cudapic_state_wall_counters(cudapic_state *s, cudapic_wall_counters out[2]);
/* eduPIC's simulation report (check_and_save_info, C/eduPIC.cc:925-1030)
 * for the measurement window (since cudapic_state_set_measure(s, 1)):
 * plasma characteristics at the centre, the stability and accuracy
 * conditions, and the particle fluxes at the electrodes.  The centre
 * density is the window's average of the electron density at node N_G/2;
 * the mean energy is that of the electrons the EEPF samples; collision
 * frequencies are events per second per particle present; fluxes are
 * absorbed particles x weight / electrode area / window time; mean ion
 * energies are those of the IFEDs (NaN without absorbed ions). */
typedef struct cudapic_report {
    uint64_t steps_measured;
    double density_center;        /* m^-3                                     */
    double plasma_freq;           /* rad/s                                    */
    double mean_energy_center;    /* eV                                       */
    double debye_length;          /* m                                        */
    double e_coll_freq;           /* 1/s                                      */
    double i_coll_freq;
    double wp_dt_e;               /* plasma frequency x DT_E     (OK < 0.20)  */
    double dx_over_debye;         /* DX / Debye length           (OK < 1.00)  */
    double max_e_coll_dt_e;       /* max e coll. frequency x DT_E (OK < 0.05) */
    double max_i_coll_dt_i;       /* max ion coll. frequency x DT_I (< 0.05)  */
    int conditions_ok;
    double cfl_max_energy;        /* eV                                       */
    double ion_flux_pow, ion_flux_gnd;   /* m^-2 s^-1                         */
    double mean_ion_energy_pow, mean_ion_energy_gnd;   /* eV                  */
    double e_flux_pow, e_flux_gnd;       /* m^-2 s^-1                         */
    double power_e, power_i;      /* <j E> of the XT diagnostics, W m^-3 (NaN
                                     without them), C/eduPIC.cc:1011-1026   */
} cudapic_report;
int cudapic_state_report(cudapic_state *s, cudapic_report *out);
/* Writes the report as eduPIC's info.txt (same lines and number formats). */
int cudapic_state_write_info(cudapic_state *s, const char *path);
/* Spatio-temporal (XT) diagnostics of the measurement window (eduPIC's
 * measurement mode, C/eduPIC.cc:557-614 and :705-715, normalised as
 * norm_all_xt, :864-903): [N_G][N_XT] doubles, N_XT = N_T / CUDAPIC_XT_BIN
 * columns of CUDAPIC_XT_BIN steps of the RF period each.  Collected while
 * measuring when N_T is a multiple of CUDAPIC_XT_BIN (else n_xt = 0).
 * Quantities in the order of eduPIC's save_all_xt files. */
#define CUDAPIC_XT_BIN 20
enum {
    CUDAPIC_XT_POT = 0,     /* potential [V]                       pot_xt.dat     */
    CUDAPIC_XT_EFIELD,      /* electric field [V/m]                efield_xt.dat  */
    CUDAPIC_XT_NE,          /* electron density [m^-3]             ne_xt.dat      */
    CUDAPIC_XT_NI,          /* ion density [m^-3]                  ni_xt.dat      */
    CUDAPIC_XT_JE,          /* electron current density [A m^-2]   je_xt.dat      */
    CUDAPIC_XT_JI,          /* ion current density [A m^-2]        ji_xt.dat      */
    CUDAPIC_XT_POWERE,      /* electron power absorption [W m^-3]  powere_xt.dat  */
    CUDAPIC_XT_POWERI,      /* ion power absorption [W m^-3]       poweri_xt.dat  */
    CUDAPIC_XT_MEANEE,      /* mean electron energy [eV]           meanee_xt.dat  */
    CUDAPIC_XT_MEANEI,      /* mean ion energy [eV]                meanei_xt.dat  */
    CUDAPIC_XT_IONIZ,       /* ionization rate [m^-3 s^-1]         ioniz_xt.dat   */
    CUDAPIC_XT_QUANTITIES
};
int cudapic_state_xt_shape(const cudapic_state *s, uint32_t *n_g, uint32_t *n_xt);
/* One normalised quantity, out[node * n_xt + column].  Synchronises. */
int cudapic_state_download_xt(cudapic_state *s, int quantity, double *out);
/* eduPIC's eleven *_xt.dat files (one row per node, "%e  " per column) in
 * `directory`.  Synchronises. */
int cudapic_state_write_xt(cudapic_state *s, const char *directory);

/* Checkpoint: the particles of both species in eduPIC's picdata.bin format
 * at `path` (Time = steps done x DT_E, cycles_done = whole RF periods), and
 * the RNG planes of every slot in `path`.rng.  Synchronises. */
int cudapic_state_save(cudapic_state *s, const char *path);
/* Resume from a picdata.bin (this library's or eduPIC's own): uploads both
 * species, sets the steps done (and the RF phase) from its Time, and
 * restores the RNG planes from `path`.rng, or seeds the reference's master
 * streams when there is none (a file written by eduPIC).  Synchronises. */
int cudapic_state_load(cudapic_state *s, const char *path);

/* ---------------------------------------------------------------- batches
 * Many independent discharges stepped in lockstep: every kernel of a step
 * is ONE launch over all discharges of the batch (persistent grids over the
 * discharges' concatenated particles, per-discharge descriptors, counters
 * and tickets), 2 N_SUB steps per captured CUDA graph.  The reference runs
 * one discharge per process and has no counterpart; this serves parameter
 * sweeps of many small discharges, which alone leave most SMs idle.
 *
 * The discharges are existing states (fused mode, one device, equal N_T and
 * N_SUB and Poisson arithmetic flag, all at the same step, all measuring or
 * none, none in another batch).  While the batch exists their particle and
 * RNG planes live in one pool it owns (pointers from cudapic_state_buffers
 * taken before cudapic_batch_create are stale); every state call keeps
 * working between batch runs, and cudapic_batch_destroy gives each state its
 * own planes back.  A batch does not own its states: destroy it before them.
 * At most 1024 discharges, capacities summing to at most 2^31. */
typedef struct cudapic_batch cudapic_batch;
int cudapic_batch_create(cudapic_state *const *states, uint32_t count, cudapic_batch **out);
int cudapic_batch_destroy(cudapic_batch *b);
/* Enqueues n_steps of every discharge on the batch's stream, after the
 * work pending on each state's stream; each state's stream then waits for
 * the batch.  Asynchronous. */
int cudapic_batch_run_steps(cudapic_batch *b, uint64_t n_steps);
int cudapic_batch_synchronize(cudapic_batch *b);
/* Per-kernel device time of the batched step (no reference counterpart: a
 * measurement aid).  Runs n_steps (<= 4096) like cudapic_batch_run_steps but
 * uncaptured, with CUDA events around every kernel launch of a step, waits,
 * and returns per kernel kind the summed milliseconds and launch counts.
 * Programmatic dependent launch is off between the kernels of these steps. */
#define CUDAPIC_BATCH_K_POISSON 0           /* batched Poisson (+ XT grid columns)     */
#define CUDAPIC_BATCH_K_ION_PUSH 1          /* ion push + compaction + deposit         */
#define CUDAPIC_BATCH_K_ELECTRON_STEP 2     /* compacting fused electron step          */
#define CUDAPIC_BATCH_K_ION_COLLISIONS 3    /* ion MCC                                 */
#define CUDAPIC_BATCH_K_ELECTRON_INPLACE 4  /* in-place electron step, stream pass     */
#define CUDAPIC_BATCH_K_ELECTRON_SCATTER 5  /* in-place electron step, scatter pass    */
#define CUDAPIC_BATCH_KERNELS 6
int cudapic_batch_profile_steps(cudapic_batch *b, uint64_t n_steps, double ms[CUDAPIC_BATCH_KERNELS],
                                uint64_t launches[CUDAPIC_BATCH_KERNELS]);
cudapic_stream_t cudapic_batch_stream(const cudapic_batch *b);

/* ------------------------------------------------------- sensitivities
 * d(observable)/d(voltage) of one discharge by a pathwise adjoint with
 * collision events and random draws frozen.  The reference has no
 * differentiation; this differentiates its step loop
 * (Rust-CUDA/src/main.rs:1725-1808) in slot form: the same kernels in the
 * same order, but absorbed particles are marked dead (x = -1) instead of
 * compacted and the spawns of a step take the next free slots in the order
 * of their parents, so every particle keeps its RNG stream and a run is a
 * deterministic function of (initial state, voltage).  Deposits are exact
 * integer sums, the Poisson sums FP64 (a state with
 * CUDAPIC_FLAG_POISSON_F32_SCAN is refused), scattering uses algebraic sines
 * and cosines.
 *
 * Observables, averaged over a window of K steps from RF phase zero:
 *   obs[0] = J_P  <j E> electron power averaged over the gap [W m^-3]
 *                 (C/eduPIC.cc:593-614, 1011-1026, summed per particle);
 *   obs[1] = J_G  ion flux to the grounded electrode [m^-2 s^-1], the CIC
 *                 flux density n v at node N_G-1 (C/eduPIC.cc:651-658 counts
 *                 the same flux).
 * The forward run saves a checkpoint every `checkpoint_every` steps; the
 * backward pass recomputes each interval from its checkpoint with a tape
 * and sweeps it in reverse.  horizon (a multiple of checkpoint_every, 0 =
 * the whole window): the adjoint restarts from zero at every multiple of
 * `horizon` steps (the sensitivity with the influence of the voltage
 * truncated to that horizon; chaotic particle dynamics make the full-window
 * pathwise derivative grow without bound over long windows). */
typedef struct cudapic_sens cudapic_sens;
#define CUDAPIC_SENS_POWER_E     0
#define CUDAPIC_SENS_ION_FLUX_GND 1
/* Snapshot of the state's particles and RNG planes (its current contents;
 * the state is not changed and may be stepped further); window_steps and
 * checkpoint_every are whole ion cycles (N_SUB), window_steps a multiple of
 * checkpoint_every; n_g <= 4096.  The object runs on the state's stream
 * and reads the state's cross-section tables: destroy it before the state. */
int cudapic_sens_create(cudapic_state *st, uint32_t window_steps, uint32_t checkpoint_every, uint32_t horizon,
                        cudapic_sens **out);
/* Runs the window from the snapshot at RF amplitude `voltage` (the same
 * snapshot and RNG streams every call: common random numbers). */
int cudapic_sens_forward(cudapic_sens *s, double voltage, double obs[2]);
/* d obs / d voltage at the voltage of the last forward run. */
int cudapic_sens_backward(cudapic_sens *s, double grad[2]);
/* Slot counts and device error word after the last run; device memory held. */
int cudapic_sens_info(cudapic_sens *s, uint32_t counts[2], uint32_t *dev_err, uint64_t *device_bytes);
/* Particles of one species after the last run (all `capacity` >= the
 * state's capacity slots; dead slots have x = -1); rng (may be NULL): the
 * four planes one after another. */
int cudapic_sens_download(cudapic_sens *s, int species, float *x, float *vx, float *vy, float *vz, uint32_t *rng,
                          uint32_t capacity);
int cudapic_sens_destroy(cudapic_sens *s);

/* ------------------------------------------------------------ all-FP64
 * An all-FP64 twin of a discharge for the precision study: the reference's
 * launch sequence (Rust-CUDA/src/main.rs:1725-1808) with particles, fields,
 * densities, collision tests and scattering in double (CUDA's double
 * transcendentals; the reference's RNG draws and f32 cross-section tables
 * widened to double).  The reference computes in f32 and has no
 * counterpart.  Created from a state at the start of an ion cycle (its
 * particles widened, its RNG planes copied, its RF phase continued); the
 * state is not changed.  n_g <= 4096.  The twin runs on the state's stream
 * and reads the state's cross-section tables: destroy it before the state. */
typedef struct cudapic_fp64 cudapic_fp64;
int cudapic_fp64_create(cudapic_state *st, cudapic_fp64 **out);
/* Starts (on) or stops a measurement window; both clear the window sums. */
int cudapic_fp64_set_measure(cudapic_fp64 *d, int on);
int cudapic_fp64_run_steps(cudapic_fp64 *d, uint64_t n_steps);
/* Window sums (each may be NULL): node densities summed every step
 * (electrons) or every ion step (ions), boundary nodes doubled [m^-3 x
 * steps]; potential summed every step [V x steps]; EEPF counts (2000 bins of
 * 0.05 eV, central 10 % of the gap, after each step); power_sum: the sum
 * over steps and electrons of (v + f E/2) E at the push [V s^-1], so that
 * -e (W/A) / L x power_sum / steps is the <j E> power [W m^-3]; steps[0]
 * measured steps, steps[1] measured ion steps; counts: n_e, n_i now;
 * dev_err: CUDAPIC_DEVERR_* bits. */
int cudapic_fp64_measurements(cudapic_fp64 *d, double *cumul_e, double *cumul_i, double *pot_sum, uint32_t *eepf,
                              double *power_sum, uint64_t steps[2], uint32_t counts[2], uint32_t *dev_err);
int cudapic_fp64_destroy(cudapic_fp64 *d);

#ifdef __cplusplus
}
#endif
#endif /* CUDAPIC_H */
