// kernels_mcc.cu -- Monte-Carlo collisions of electrons and ions.
//
// Reference: check_collisions_e / collision_e, Rust-CUDA/src/main.rs:971-1165,
// check_collisions_i / collision_i, :1167-1292.  Per electron: energy index
// min(int(E/1 meV + 0.5), 1e6-1), nu = sigma_tot(E) |v|, collide iff
// u < 1 - exp(-nu dt); the type (elastic / excitation / ionization) from
// the cumulative cross-section ratios; Euler-angle rotation of the relative
// velocity; ionization spawns an electron and an ion.  Per ion: a Maxwellian
// target atom (Box-Muller), relative energy, isotropic or backward
// scattering.  The RNG draw order of the reference is kept exactly.
//
// B200 design: HBM-bound streaming (28 B read + 16 B RNG written per
// particle; velocities written only by colliders, ~0.5 % of electrons per
// step at the reference conditions).  Two kernels share the physics:
//  * resident-table kernel (default, cudapic_tuning.mcc_variant = 1): one
//    1024-thread CTA per SM keeps the first 32768 entries of sigma_tot in
//    shared memory, every thread issues the loads of two particles before
//    computing, and colliders go to warp-private queues drained 32 at a
//    time -- no block barrier in the main loop;
//  * bulk-copy kernel (mcc_variant = 2): tiles of the seven SoA arrays staged
//    by cp.async.bulk on mbarriers, a CTA-wide collider queue.
// Common to both:
//  * the collision test of every particle is uniform work; the provably
//    exact fast reject skips exp() for almost all of them; non-colliders
//    store their advanced RNG state (coalesced);
//  * a collider keeps its slot and its RNG state before the test; the drain
//    re-runs the deterministic test and scatters it on a full warp (one
//    collider per lane) instead of one lane in 32;
//  * ionization spawns claim slots with one warp-aggregated atomicAdd per
//    counter, bounded by capacity: a spawn that does not fit is dropped and
//    flagged, never written out of bounds (the reference writes unbounded,
//    :1132-1149);
//  * transcendentals from detmath.cuh (bit-reproducible, see there).
#include "common.cuh"
#include "internal.h"
#include "mcc.cuh"
#include "tma.cuh"

namespace cudapic {

constexpr int MCC_THREADS = 256;

// ------------------------------------------------------------------ bulk-copy kernels

constexpr int MT_U = 2;                       // particles per thread and tile
constexpr int MT_TILE = MCC_THREADS * MT_U;   // 512
constexpr int MT_MAX_STAGES = 4;              // pipeline depth: cudapic_tuning.mcc_stages
constexpr int MT_ARRAYS = 7;                  // vx, vy, vz, rng0..3
constexpr int MT_QFLUSH = 256;                // drain the queue when it holds more
constexpr int MT_QCAP = MT_QFLUSH + MT_TILE;  // never overflows: one tile adds <= 512
constexpr int MT_QWORDS = 5;                  // slot index + the RNG state before the test

size_t mcc_tma_smem_bytes(int stages) {
    return (size_t)stages * MT_ARRAYS * MT_TILE * 4 + (size_t)MT_QCAP * MT_QWORDS * 4 +
           (size_t)stages * sizeof(uint64_t);
}

// ION = false: check_collisions_e; ION = true: check_collisions_i.
// A queued collider keeps only its slot and its RNG state before the test;
// the drain re-runs the (deterministic) test from that state, reading the
// velocity again, and continues into the scattering.
template <bool ION, bool EVENTS>
__global__ void __launch_bounds__(MCC_THREADS, 4)
    check_collisions_tma_kernel(const float *__restrict__ sigma_tot, const float *__restrict__ cs,
                                const uint32_t *__restrict__ active, float *x, float *vx, float *vy, float *vz,
                                uint32_t *rng0, uint32_t *rng1, uint32_t *rng2, uint32_t *rng3, float *ix,
                                float *ivx, float *ivy, float *ivz, uint32_t *alive_e, uint32_t *alive_i,
                                uint8_t *events, const __grid_constant__ cudapic_grid g, int stages,
                                float *dep_e, float *dep_i, unsigned long long *coll, float ion_k) {
    extern __shared__ __align__(128) unsigned char smem[];
    uint32_t *in = reinterpret_cast<uint32_t *>(smem);             // [stages][7][TILE]
    uint32_t *queue = in + stages * MT_ARRAYS * MT_TILE;           // [5][QCAP]
    uint64_t *bar = reinterpret_cast<uint64_t *>(queue + MT_QWORDS * MT_QCAP);
    __shared__ uint32_t s_q;
    __shared__ int s_ready;

    const int tid = threadIdx.x;
    grid_dep_wait();
    const uint32_t n = load_count(active, g.capacity, g.dev_err);
    const uint32_t ntiles = (n + MT_TILE - 1) / MT_TILE;
    const void *src[MT_ARRAYS] = {vx, vy, vz, rng0, rng1, rng2, rng3};

    auto issue = [&](uint32_t tile, int stage) {
        const uint32_t t0 = tile * MT_TILE;
        const uint32_t cnt = min((uint32_t)MT_TILE, n - t0);
        const uint32_t bytes = ((cnt + 3u) & ~3u) * 4u;
        mbar_arrive_expect_tx(&bar[stage], MT_ARRAYS * bytes);
#pragma unroll
        for (int a = 0; a < MT_ARRAYS; ++a)
            bulk_load(in + (stage * MT_ARRAYS + a) * MT_TILE, static_cast<const uint32_t *>(src[a]) + t0, bytes,
                      &bar[stage]);
    };

    const GlobalTable table{sigma_tot};
    // Drains the collider queue: one collider per thread, full warps.
    auto drain = [&]() {
        const uint32_t qn = s_q;
        if (coll && tid == 0 && qn) atomicAdd(coll, (unsigned long long)qn);  // collision events (measurement)
        for (uint32_t q = tid; q < qn; q += MCC_THREADS) {
            const uint32_t i = queue[0 * MT_QCAP + q];
            Xoshiro128p rs{queue[1 * MT_QCAP + q], queue[2 * MT_QCAP + q], queue[3 * MT_QCAP + q],
                           queue[4 * MT_QCAP + q]};
            const float vxi = vx[i], vyi = vy[i], vzi = vz[i];
            uint32_t ev;
            if (ION) {
                const IonTest t = test_ion(vxi, vyi, vzi, rs, table, g);
                ev = collide_ion(i, t.idx, vxi, vyi, vzi, t.vxa, t.vya, t.vza, rs, cs, vx, vy, vz, g);
            } else {
                const Test t = test_electron(vxi, vyi, vzi, rs, table, g);
                ev = collide_electron(0u, i, t.idx, vxi, vyi, vzi, rs, cs, x, vx, vy, vz, ix, ivx, ivy, ivz, alive_e,
                                      alive_i, g, dep_e, dep_i);
            }
            rng0[i] = rs.s0;
            rng1[i] = rs.s1;
            rng2[i] = rs.s2;
            rng3[i] = rs.s3;
            if (EVENTS) events[i] = (uint8_t)ev;
        }
        __syncthreads();
        if (tid == 0) s_q = 0;
        __syncthreads();
    };

    if (tid == 0) {
        for (int s = 0; s < stages; ++s) mbar_init(&bar[s], 1);
        fence_mbar_init();
        s_q = 0;
    }
    __syncthreads();
    if (tid == 0) {
        for (int s = 0; s < stages; ++s) {
            const uint32_t tile = blockIdx.x + (uint32_t)s * gridDim.x;
            if (tile < ntiles) issue(tile, s);
        }
    }

    uint32_t it = 0;
    for (uint32_t tile = blockIdx.x; tile < ntiles; tile += gridDim.x, ++it) {
        const int s = (int)(it % (uint32_t)stages);
        const uint32_t parity = (it / (uint32_t)stages) & 1u;
        if (tid == 0) {
            const int ok = mbar_wait_bounded(&bar[s], parity) ? 1 : 0;
            if (!ok) set_dev_err(g.dev_err, CUDAPIC_DEVERR_TIMEOUT);
            s_ready = ok;
        }
        __syncthreads();
        if (!s_ready) return;
        const uint32_t t0 = tile * MT_TILE;
        const uint32_t cnt = min((uint32_t)MT_TILE, n - t0);
        const uint32_t *b = in + s * MT_ARRAYS * MT_TILE;
#pragma unroll
        for (int u = 0; u < MT_U; ++u) {
            const uint32_t j = (uint32_t)u * MCC_THREADS + tid;
            if (j < cnt) {
                const uint32_t i = t0 + j;
                const uint32_t q0 = b[3 * MT_TILE + j], q1 = b[4 * MT_TILE + j], q2 = b[5 * MT_TILE + j],
                               q3 = b[6 * MT_TILE + j];
                Xoshiro128p rs{q0, q1, q2, q3};
                const float vxi = __uint_as_float(b[0 * MT_TILE + j]);
                const float vyi = __uint_as_float(b[1 * MT_TILE + j]);
                const float vzi = __uint_as_float(b[2 * MT_TILE + j]);
                bool collide;
                if (ION) collide = ion_collides(vxi, vyi, vzi, rs, table, g, ion_k);
                else collide = test_electron(vxi, vyi, vzi, rs, table, g).collide;
                if (collide) {
                    const uint32_t q = atomicAdd(&s_q, 1u);
                    queue[0 * MT_QCAP + q] = i;
                    queue[1 * MT_QCAP + q] = q0;
                    queue[2 * MT_QCAP + q] = q1;
                    queue[3 * MT_QCAP + q] = q2;
                    queue[4 * MT_QCAP + q] = q3;
                } else {
                    rng0[i] = rs.s0;
                    rng1[i] = rs.s1;
                    rng2[i] = rs.s2;
                    rng3[i] = rs.s3;
                    if (EVENTS) events[i] = 0;
                }
            }
        }
        __syncthreads();  // stage consumed; queue count visible
        if (tid == 0) {
            const uint32_t next = tile + (uint32_t)stages * gridDim.x;
            if (next < ntiles) issue(next, s);
        }
        if (s_q > (uint32_t)MT_QFLUSH) drain();
    }
    __syncthreads();
    if (s_q > 0) drain();
}

// ------------------------------------------------------------------ resident-table kernels
//
// One 1024-thread CTA per SM, no bulk copies and no block barrier in the
// main loop:
//  * the first MR_RESIDENT entries of sigma_tot (energies below 32.768 eV,
//    where almost every particle sits) are copied into shared memory once
//    per launch; the collision-frequency gather becomes a shared load
//    (higher energies still read the global table);
//  * each thread issues the 7 loads of MR_U particles before any compute;
//  * colliders go to a queue private to their warp (slot and RNG state
//    before the test); whenever it holds 32 the warp drains 32 of them, one
//    per lane -- only __syncwarp, no block-wide synchronisation.
// Plain loads: no alignment requirement on any pointer.

constexpr int MR_THREADS = 1024;
constexpr int MR_WARPS = MR_THREADS / 32;
constexpr int MR_U = 2;                        // particles per thread and iteration
constexpr uint32_t MR_RESIDENT = 32768;        // sigma_tot entries kept in shared memory
constexpr int MR_QCAP = 32 + 32 * MR_U;        // a warp drains at 32; one iteration adds <= 64
constexpr size_t MR_SMEM = MR_RESIDENT * sizeof(float) + (size_t)MR_WARPS * 5 * MR_QCAP * sizeof(uint32_t);

template <bool ION, bool EVENTS>
__global__ void __launch_bounds__(MR_THREADS, 1)
    check_collisions_resident_kernel(const float *__restrict__ sigma_tot, const float *__restrict__ cs,
                                     const uint32_t *__restrict__ active, float *x, float *vx, float *vy,
                                     float *vz, uint32_t *rng0, uint32_t *rng1, uint32_t *rng2, uint32_t *rng3,
                                     float *ix, float *ivx, float *ivy, float *ivz, uint32_t *alive_e,
                                     uint32_t *alive_i, uint8_t *events, const __grid_constant__ cudapic_grid g,
                                     float *dep_e, float *dep_i, unsigned long long *coll, float ion_k) {
    extern __shared__ __align__(128) unsigned char smem[];
    float *tab = reinterpret_cast<float *>(smem);
    const int tid = threadIdx.x;
    const int lane = tid & 31;
    const int warp = tid >> 5;
    uint32_t *wq = reinterpret_cast<uint32_t *>(tab + MR_RESIDENT) + (size_t)warp * 5 * MR_QCAP;  // [5][QCAP]
    const unsigned lt = lanemask_lt();

    // the table is read before the wait: under PDL (the driver) it was
    // written when the state was created, long before any dependent grid
    for (uint32_t k = tid; k < MR_RESIDENT; k += MR_THREADS) tab[k] = __ldg(sigma_tot + k);
    __syncthreads();
    grid_dep_wait();
    const ResidentTable table{sigma_tot, tab, MR_RESIDENT};
    const uint32_t n = load_count(active, g.capacity, g.dev_err);

    auto drain = [&](uint32_t first, uint32_t count) {  // lanes < count take entries first + lane
        if (coll && lane == 0) atomicAdd(coll, (unsigned long long)count);  // collision events (measurement)
        if ((uint32_t)lane < count) {
            const uint32_t q = first + lane;
            const uint32_t i = wq[0 * MR_QCAP + q];
            Xoshiro128p rs{wq[1 * MR_QCAP + q], wq[2 * MR_QCAP + q], wq[3 * MR_QCAP + q], wq[4 * MR_QCAP + q]};
            const float vxi = vx[i], vyi = vy[i], vzi = vz[i];
            uint32_t ev;
            if (ION) {
                const IonTest t = test_ion(vxi, vyi, vzi, rs, table, g);
                ev = collide_ion(i, t.idx, vxi, vyi, vzi, t.vxa, t.vya, t.vza, rs, cs, vx, vy, vz, g);
            } else {
                const Test t = test_electron(vxi, vyi, vzi, rs, table, g);
                ev = collide_electron(0u, i, t.idx, vxi, vyi, vzi, rs, cs, x, vx, vy, vz, ix, ivx, ivy, ivz, alive_e,
                                      alive_i, g, dep_e, dep_i);
            }
            rng0[i] = rs.s0;
            rng1[i] = rs.s1;
            rng2[i] = rs.s2;
            rng3[i] = rs.s3;
            if (EVENTS) events[i] = (uint8_t)ev;
        }
        __syncwarp();
    };

    uint32_t qn = 0;  // entries in this warp's queue (warp-uniform)
    const uint32_t step = gridDim.x * (uint32_t)(MR_THREADS * MR_U);
    for (uint32_t base = blockIdx.x * (uint32_t)(MR_THREADS * MR_U); base < n; base += step) {
        uint32_t s[MR_U][4];
        float v[MR_U][3];
#pragma unroll
        for (int u = 0; u < MR_U; ++u) {
            const uint32_t i = base + (uint32_t)u * MR_THREADS + tid;
            if (i < n) {
                s[u][0] = rng0[i];
                s[u][1] = rng1[i];
                s[u][2] = rng2[i];
                s[u][3] = rng3[i];
                v[u][0] = vx[i];
                v[u][1] = vy[i];
                v[u][2] = vz[i];
            }
        }
#pragma unroll
        for (int u = 0; u < MR_U; ++u) {
            const uint32_t i = base + (uint32_t)u * MR_THREADS + tid;
            bool collide = false;
            if (i < n) {
                Xoshiro128p rs{s[u][0], s[u][1], s[u][2], s[u][3]};
                if (ION) collide = ion_collides(v[u][0], v[u][1], v[u][2], rs, table, g, ion_k);
                else collide = test_electron(v[u][0], v[u][1], v[u][2], rs, table, g).collide;
                if (!collide) {
                    rng0[i] = rs.s0;
                    rng1[i] = rs.s1;
                    rng2[i] = rs.s2;
                    rng3[i] = rs.s3;
                    if (EVENTS) events[i] = 0;
                }
            }
            const unsigned m = __ballot_sync(0xffffffffu, collide);
            if (collide) {
                const uint32_t q = qn + __popc(m & lt);
                wq[0 * MR_QCAP + q] = i;
                wq[1 * MR_QCAP + q] = s[u][0];
                wq[2 * MR_QCAP + q] = s[u][1];
                wq[3 * MR_QCAP + q] = s[u][2];
                wq[4 * MR_QCAP + q] = s[u][3];
            }
            qn += __popc(m);
        }
        __syncwarp();
        while (qn >= 32) {  // full-warp drains from the top of the queue
            qn -= 32;
            drain(qn, 32);
        }
    }
    if (qn) drain(0, qn);
}

// accumulate_eepf, Rust-CUDA/src/main.rs:1301-1339: per-block shared
// histogram, one global atomic per non-empty bin and block.
__global__ void __launch_bounds__(256)
    accumulate_eepf_kernel(const float *__restrict__ x, const float *__restrict__ vx, const float *__restrict__ vy,
                           const float *__restrict__ vz, const float *__restrict__ efield,
                           const uint32_t *__restrict__ active_e, uint32_t *__restrict__ eepf,
                           const cudapic_grid g, double *esum, unsigned long long *ecount) {
    __shared__ uint32_t h[N_EEPF];
    for (uint32_t k = threadIdx.x; k < N_EEPF; k += blockDim.x) h[k] = 0;
    __syncthreads();
    grid_dep_wait();
    const uint32_t n = load_count(active_e, g.capacity, g.dev_err);
    double e_sum = 0.0;
    unsigned long long e_cnt = 0;
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const float xi = x[i];
        if (xi <= g.min_x || xi >= g.max_x) continue;
        const float pos = xi * g.inv_dx;
        const int p = cell_of(pos, g.n_g);
        const float c2 = pos - (float)p;
        const float e_x = (1.0f - c2) * __ldg(efield + p) + c2 * __ldg(efield + p + 1);
        const float mvx = vx[i] - 0.5f * e_x * g.eepf_half_kick;
        const float vyi = vy[i], vzi = vz[i];
        const float v2 = mvx * mvx + vyi * vyi + vzi * vzi;
        const float energy = g.half_me_over_e * v2;
        const float binf = energy / DE_EEPF_F;
        if (binf < (float)N_EEPF) atomicAdd(&h[(uint32_t)binf], 1u);
        e_sum += (double)energy;
        ++e_cnt;
    }
    if (esum) {  // mean energy of the sampled electrons (the report's centre energy)
        for (int o = 16; o > 0; o >>= 1) {
            e_sum += __shfl_down_sync(0xffffffffu, e_sum, o);
            e_cnt += __shfl_down_sync(0xffffffffu, e_cnt, o);
        }
        if ((threadIdx.x & 31) == 0 && e_cnt) {
            atomicAdd(esum, e_sum);
            atomicAdd(ecount, e_cnt);
        }
    }
    __syncthreads();
    for (uint32_t k = threadIdx.x; k < N_EEPF; k += blockDim.x)
        if (h[k]) atomicAdd(&eepf[k], h[k]);
}

namespace {

bool tma_ready(uint32_t capacity, std::initializer_list<const void *> ptrs) {
    if (capacity % 4u) return false;
    for (const void *p : ptrs)
        if (!aligned16(p)) return false;
    return true;
}

template <bool ION, bool EVENTS>
int launch_tma(const float *sigma_tot, const float *cs, const uint32_t *active, float *x, float *vx, float *vy,
               float *vz, uint32_t *r0, uint32_t *r1, uint32_t *r2, uint32_t *r3, float *ix, float *ivx, float *ivy,
               float *ivz, uint32_t *alive_e, uint32_t *alive_i, uint8_t *events, const cudapic_grid &g,
               cudaStream_t stream, float *dep_e, float *dep_i, unsigned long long *coll, float ion_k) {
    auto kern = check_collisions_tma_kernel<ION, EVENTS>;
    const cudapic_tuning t = tuning();
    const int stages = std::min(std::max(t.mcc_stages, 2), MT_MAX_STAGES);
    const size_t smem = mcc_tma_smem_bytes(stages);
    CUDAPIC_CHECK(check_cuda(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem),
                             "cudaFuncSetAttribute(check_collisions)"));
    int per_sm = 0;
    CUDAPIC_CHECK(check_cuda(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, MCC_THREADS, smem),
                             "occupancy(check_collisions)"));
    per_sm = std::min(std::max(per_sm, 1), t.mcc_ctas_per_sm);
    const uint64_t tiles_max = ((uint64_t)g.capacity + MT_TILE - 1) / MT_TILE;
    const unsigned grid = persistent_grid(per_sm, tiles_max);
    return launch_kernel(ION ? "check_collisions_i" : "check_collisions_e", kern, dim3(grid), dim3(MCC_THREADS), smem,
                         stream, sigma_tot, cs, active, x, vx, vy, vz, r0, r1, r2, r3, ix, ivx, ivy, ivz, alive_e,
                         alive_i, events, g, stages, dep_e, dep_i, coll, ion_k);
}

template <bool ION, bool EVENTS>
int launch_resident(const float *sigma_tot, const float *cs, const uint32_t *active, float *x, float *vx, float *vy,
                    float *vz, uint32_t *r0, uint32_t *r1, uint32_t *r2, uint32_t *r3, float *ix, float *ivx,
                    float *ivy, float *ivz, uint32_t *alive_e, uint32_t *alive_i, uint8_t *events,
                    const cudapic_grid &g, cudaStream_t stream, float *dep_e, float *dep_i,
                    unsigned long long *coll, float ion_k) {
    auto kern = check_collisions_resident_kernel<ION, EVENTS>;
    if (MR_SMEM > (size_t)max_smem_optin()) return fail(CUDAPIC_ERR_NOT_SUPPORTED, "check_collisions: shared memory");
    CUDAPIC_CHECK(check_cuda(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)MR_SMEM),
                             "cudaFuncSetAttribute(check_collisions resident)"));
    const uint64_t chunks = ((uint64_t)g.capacity + MR_THREADS * MR_U - 1) / (MR_THREADS * MR_U);
    return launch_kernel(ION ? "check_collisions_i" : "check_collisions_e", kern, dim3(persistent_grid(1, chunks)),
                         dim3(MR_THREADS), MR_SMEM, stream, sigma_tot, cs, active, x, vx, vy, vz, r0, r1, r2, r3, ix,
                         ivx, ivy, ivz, alive_e, alive_i, events, g, dep_e, dep_i, coll, ion_k);
}

// Variant choice: the bulk-copy kernel needs 16-byte aligned planes and a
// capacity that is a multiple of 4; the resident-table kernel takes anything.
template <bool ION>
int launch_collisions(const float *sigma_tot, const float *cs, const uint32_t *active, float *x, float *vx,
                      float *vy, float *vz, uint32_t *r0, uint32_t *r1, uint32_t *r2, uint32_t *r3, float *ix,
                      float *ivx, float *ivy, float *ivz, uint32_t *alive_e, uint32_t *alive_i, uint8_t *events,
                      const cudapic_grid &g, cudaStream_t stream, float *dep_e, float *dep_i,
                      unsigned long long *coll, float ion_k = INFINITY) {
    const bool bulk = tuning().mcc_variant == 2 && tma_ready(g.capacity, {vx, vy, vz, r0, r1, r2, r3});
    if (bulk) {
        if (events)
            return launch_tma<ION, true>(sigma_tot, cs, active, x, vx, vy, vz, r0, r1, r2, r3, ix, ivx, ivy, ivz,
                                         alive_e, alive_i, events, g, stream, dep_e, dep_i, coll, ion_k);
        return launch_tma<ION, false>(sigma_tot, cs, active, x, vx, vy, vz, r0, r1, r2, r3, ix, ivx, ivy, ivz,
                                      alive_e, alive_i, nullptr, g, stream, dep_e, dep_i, coll, ion_k);
    }
    if (events)
        return launch_resident<ION, true>(sigma_tot, cs, active, x, vx, vy, vz, r0, r1, r2, r3, ix, ivx, ivy, ivz,
                                          alive_e, alive_i, events, g, stream, dep_e, dep_i, coll, ion_k);
    return launch_resident<ION, false>(sigma_tot, cs, active, x, vx, vy, vz, r0, r1, r2, r3, ix, ivx, ivy, ivz,
                                       alive_e, alive_i, nullptr, g, stream, dep_e, dep_i, coll, ion_k);
}

}  // namespace

int launch_collisions_e(const float *total_cs_e, const float *cs, const uint32_t *active_e, float *x, float *vx,
                        float *vy, float *vz, uint32_t *rng0, uint32_t *rng1, uint32_t *rng2, uint32_t *rng3,
                        float *i_x, float *i_vx, float *i_vy, float *i_vz, uint32_t *alive_e, uint32_t *alive_i,
                        uint8_t *events, const cudapic_grid &g, cudaStream_t stream, float *dep_e, float *dep_i,
                        unsigned long long *coll) {
    return launch_collisions<false>(total_cs_e, cs, active_e, x, vx, vy, vz, rng0, rng1, rng2, rng3, i_x, i_vx, i_vy,
                                    i_vz, alive_e, alive_i, events, g, stream, dep_e, dep_i, coll);
}

int launch_collisions_i(const float *total_cs_i, const float *cs, const uint32_t *active_i, float *vx, float *vy,
                        float *vz, uint32_t *rng0, uint32_t *rng1, uint32_t *rng2, uint32_t *rng3, uint8_t *events,
                        const cudapic_grid &g, cudaStream_t stream, unsigned long long *coll, float ion_k) {
    return launch_collisions<true>(total_cs_i, cs, active_i, nullptr, vx, vy, vz, rng0, rng1, rng2, rng3, nullptr,
                                   nullptr, nullptr, nullptr, nullptr, nullptr, events, g, stream, nullptr, nullptr,
                                   coll, ion_k);
}

float ion_reject_k(float sigma_max_i, const cudapic_grid &g) {
    if (!(sigma_max_i > 0.0f) || !(g.dt_i > 0.0f) || !std::isfinite(sigma_max_i)) return INFINITY;
    const double k = (double)sigma_max_i * (double)g.dt_i * (1.0 + 1e-5);
    return std::nextafter((float)k, INFINITY);
}

int launch_eepf(const float *x, const float *vx, const float *vy, const float *vz, const float *efield,
                const uint32_t *active_e, uint32_t *eepf, const cudapic_grid &g, cudaStream_t stream,
                double *esum, unsigned long long *ecount) {
    const uint64_t need = ((uint64_t)g.capacity + 255) / 256;
    const unsigned grid = (unsigned)std::max<uint64_t>(1, std::min<uint64_t>((uint64_t)sm_count() * 2, need));
    return launch_kernel("accumulate_eepf", accumulate_eepf_kernel, dim3(grid), dim3(256), 0, stream, x, vx, vy, vz,
                         efield, active_e, eepf, g, esum, ecount);
}

}  // namespace cudapic

using namespace cudapic;

#define CUDAPIC_E_ARGS_NONNULL                                                                              \
    (total_cs_e && cs && active_e && x && vx && vy && vz && rng0 && rng1 && rng2 && rng3 && i_x && i_vx && \
     i_vy && i_vz && alive_e && alive_i)

extern "C" int cudapic_check_collisions_e(const float *total_cs_e, const float *cs, const uint32_t *active_e,
                                          float *x, float *vx, float *vy, float *vz, uint32_t *rng0,
                                          uint32_t *rng1, uint32_t *rng2, uint32_t *rng3, float *i_x, float *i_vx,
                                          float *i_vy, float *i_vz, uint32_t *alive_e, uint32_t *alive_i,
                                          const cudapic_grid *grid, cudapic_stream_t stream) {
    CUDAPIC_CHECK(validate_grid(grid));
    CUDAPIC_REQUIRE(CUDAPIC_E_ARGS_NONNULL, "check_collisions_e: null pointer");
    return launch_collisions_e(total_cs_e, cs, active_e, x, vx, vy, vz, rng0, rng1, rng2, rng3, i_x, i_vx, i_vy,
                               i_vz, alive_e, alive_i, nullptr, *grid, (cudaStream_t)stream);
}

extern "C" int cudapic_check_collisions_e_events(const float *total_cs_e, const float *cs,
                                                 const uint32_t *active_e, float *x, float *vx, float *vy,
                                                 float *vz, uint32_t *rng0, uint32_t *rng1, uint32_t *rng2,
                                                 uint32_t *rng3, float *i_x, float *i_vx, float *i_vy,
                                                 float *i_vz, uint32_t *alive_e, uint32_t *alive_i,
                                                 uint8_t *events, const cudapic_grid *grid,
                                                 cudapic_stream_t stream) {
    CUDAPIC_CHECK(validate_grid(grid));
    CUDAPIC_REQUIRE(CUDAPIC_E_ARGS_NONNULL && events, "check_collisions_e_events: null pointer");
    return launch_collisions_e(total_cs_e, cs, active_e, x, vx, vy, vz, rng0, rng1, rng2, rng3, i_x, i_vx, i_vy,
                               i_vz, alive_e, alive_i, events, *grid, (cudaStream_t)stream);
}

extern "C" int cudapic_check_collisions_e_deposit(const float *total_cs_e, const float *cs,
                                                  const uint32_t *active_e, float *x, float *vx, float *vy,
                                                  float *vz, uint32_t *rng0, uint32_t *rng1, uint32_t *rng2,
                                                  uint32_t *rng3, float *i_x, float *i_vx, float *i_vy,
                                                  float *i_vz, uint32_t *alive_e, uint32_t *alive_i,
                                                  float *e_next_density, float *i_next_density,
                                                  const cudapic_grid *grid, cudapic_stream_t stream) {
    CUDAPIC_CHECK(validate_grid(grid));
    CUDAPIC_REQUIRE(CUDAPIC_E_ARGS_NONNULL, "check_collisions_e_deposit: null pointer");
    return launch_collisions_e(total_cs_e, cs, active_e, x, vx, vy, vz, rng0, rng1, rng2, rng3, i_x, i_vx, i_vy,
                               i_vz, alive_e, alive_i, nullptr, *grid, (cudaStream_t)stream, e_next_density,
                               i_next_density);
}

extern "C" int cudapic_check_collisions_i(const float *total_cs_i, const float *cs, const uint32_t *active_i,
                                          float *vx, float *vy, float *vz, uint32_t *rng0, uint32_t *rng1,
                                          uint32_t *rng2, uint32_t *rng3, const cudapic_grid *grid,
                                          cudapic_stream_t stream) {
    CUDAPIC_CHECK(validate_grid(grid));
    CUDAPIC_REQUIRE(total_cs_i && cs && active_i && vx && vy && vz && rng0 && rng1 && rng2 && rng3,
                    "check_collisions_i: null pointer");
    return launch_collisions_i(total_cs_i, cs, active_i, vx, vy, vz, rng0, rng1, rng2, rng3, nullptr, *grid,
                               (cudaStream_t)stream);
}

extern "C" int cudapic_check_collisions_i_events(const float *total_cs_i, const float *cs,
                                                 const uint32_t *active_i, float *vx, float *vy, float *vz,
                                                 uint32_t *rng0, uint32_t *rng1, uint32_t *rng2, uint32_t *rng3,
                                                 uint8_t *events, const cudapic_grid *grid,
                                                 cudapic_stream_t stream) {
    CUDAPIC_CHECK(validate_grid(grid));
    CUDAPIC_REQUIRE(total_cs_i && cs && active_i && vx && vy && vz && rng0 && rng1 && rng2 && rng3 && events,
                    "check_collisions_i_events: null pointer");
    return launch_collisions_i(total_cs_i, cs, active_i, vx, vy, vz, rng0, rng1, rng2, rng3, events, *grid,
                               (cudaStream_t)stream);
}

extern "C" int cudapic_check_collisions_i_bounded(const float *total_cs_i, const float *cs,
                                                  const uint32_t *active_i, float *vx, float *vy, float *vz,
                                                  uint32_t *rng0, uint32_t *rng1, uint32_t *rng2, uint32_t *rng3,
                                                  float sigma_max_i, uint8_t *events, const cudapic_grid *grid,
                                                  cudapic_stream_t stream) {
    CUDAPIC_CHECK(validate_grid(grid));
    CUDAPIC_REQUIRE(total_cs_i && cs && active_i && vx && vy && vz && rng0 && rng1 && rng2 && rng3,
                    "check_collisions_i_bounded: null pointer");
    CUDAPIC_REQUIRE(sigma_max_i >= 0.0f, "check_collisions_i_bounded: sigma_max_i must be the largest entry of total_cs_i");
    return launch_collisions_i(total_cs_i, cs, active_i, vx, vy, vz, rng0, rng1, rng2, rng3, events, *grid,
                               (cudaStream_t)stream, nullptr, ion_reject_k(sigma_max_i, *grid));
}

extern "C" int cudapic_accumulate_eepf(const float *x, const float *vx, const float *vy, const float *vz,
                                       const float *efield, const uint32_t *active_e, uint32_t *eepf,
                                       const cudapic_grid *grid, cudapic_stream_t stream) {
    CUDAPIC_CHECK(validate_grid(grid));
    CUDAPIC_REQUIRE(x && vx && vy && vz && efield && active_e && eepf, "accumulate_eepf: null pointer");
    return launch_eepf(x, vx, vy, vz, efield, active_e, eepf, *grid, (cudaStream_t)stream);
}
