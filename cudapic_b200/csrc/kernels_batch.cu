// kernels_batch.cu -- the particle kernels of a batch of discharges.
//
// The reference steps one discharge per process (Rust-CUDA/src/main.rs:
// 1725-1808); a parameter sweep of small discharges leaves most of a B200
// idle between launches.  Here one persistent launch per kernel of the step
// covers every discharge of a batch:
//  * the particles of all discharges form one index space, each discharge's
//    count rounded up to a multiple of 4 (so every segment starts 16-byte
//    aligned); CTA c owns an equal contiguous share of it, which cuts into at
//    most a few discharges: its segments;
//  * the particle planes of all discharges live in one pool: the plane bases
//    are launch parameters, a discharge is an element offset into them;
//  * per segment the CTA loads that discharge's descriptor (offset, grid
//    constants, buffers, tables) into shared memory and runs the same tile
//    pipeline as the one-discharge fused step (step.cuh), with the
//    discharge's own slot counters, density and E-field;
//  * each discharge's count is published by the last CTA to finish it (its
//    own ticket, expecting the CTAs whose shares meet the discharge).
// The plan (a prefix over the counts) is recomputed by every CTA from the
// counts the batched Poisson kernel wrote, so no extra launch is needed.
#include <algorithm>

#include "batch_internal.h"
#include "inplace.cuh"
#include "internal.h"
#include "step.cuh"

namespace cudapic {

namespace {

__device__ __forceinline__ uint32_t round4(uint32_t n) { return (n + 3u) & ~3u; }

// A shared word read by a volatile load (never kept in a register across code
// that does not need it).
__device__ __forceinline__ uint32_t lds_volatile(const uint32_t *p) {
    uint32_t v;
    asm volatile("ld.shared.u32 %0, [%1];" : "=r"(v) : "r"(smem_addr(p)));
    return v;
}

// P[d] = sum_{k<d} round4(count(k)) for d in [0, D]; one call by the whole
// CTA (ES_THREADS threads), which synchronises before returning.
template <typename Count>
__device__ __forceinline__ void plan_prefix(Count count, uint32_t D, uint32_t *P, uint32_t *wsum) {
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const uint32_t per = (D + ES_THREADS - 1) / ES_THREADS;
    uint32_t sum = 0;
    for (uint32_t j = 0; j < per; ++j) {
        const uint32_t d = (uint32_t)tid * per + j;
        if (d < D) sum += round4(count(d));
    }
    uint32_t incl = sum;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const uint32_t t = __shfl_up_sync(0xffffffffu, incl, o);
        if (lane >= o) incl += t;
    }
    if (lane == 31) wsum[warp] = incl;
    __syncthreads();
    if (warp == 0) {
        uint32_t w = lane < ES_WARPS ? wsum[lane] : 0u;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const uint32_t t = __shfl_up_sync(0xffffffffu, w, o);
            if (lane >= o) w += t;
        }
        if (lane < ES_WARPS) wsum[lane] = w;
    }
    __syncthreads();
    uint32_t run = incl - sum + (warp > 0 ? wsum[warp - 1] : 0u);
    for (uint32_t j = 0; j < per; ++j) {
        const uint32_t d = (uint32_t)tid * per + j;
        if (d < D) {
            P[d] = run;
            run += round4(count(d));
        }
    }
    if (tid == 0) P[D] = wsum[ES_WARPS - 1];
    __syncthreads();
}

// Smallest d with P[d + 1] > x (D when there is none).
__device__ __forceinline__ uint32_t first_discharge(const uint32_t *P, uint32_t D, uint32_t x) {
    uint32_t lo = 0, hi = D;
    while (lo < hi) {
        const uint32_t mid = (lo + hi) >> 1;
        if (P[mid + 1] > x) hi = mid;
        else lo = mid + 1;
    }
    return lo;
}

// The CTA's share [beg, end) of the batch's index space (a multiple of 4 long).
__device__ __forceinline__ void cta_share(uint32_t total, uint32_t &chunk, uint32_t &beg, uint32_t &end) {
    chunk = ((total + gridDim.x - 1) / gridDim.x + 3u) & ~3u;
    beg = min(total, blockIdx.x * chunk);
    end = min(total, beg + chunk);
}

// Publishes a discharge's count: the CTA whose ticket is the last of the
// `expected` CTAs that processed the discharge stores min(*src, capacity)
// into *dst and clears *src and the ticket (publish_count with a count).
__device__ __forceinline__ void publish_count_of(uint32_t *ticket, uint32_t *dst, uint32_t *src, uint32_t capacity,
                                                 uint32_t expected) {
    __threadfence();
    __syncthreads();
    if (threadIdx.x == 0) {
        const uint32_t t = atomicAdd(ticket, 1u);
        if (t == expected - 1) {
            __threadfence();
            const uint32_t v = atomicExch(src, 0u);
            *dst = v < capacity ? v : capacity;
            *ticket = 0u;
        }
    }
}

}  // namespace

// MCC: the fused electron step of every discharge; !MCC: the ion push with
// the deposit of the next ion density.  The plane bases are launch
// parameters (one pool for all discharges); per segment only the discharge's
// offset, grid constants and a few buffers differ.  MINB: resident CTAs per
// SM the register allocation is bounded for (cudapic_tuning.step_ctas_per_sm);
// MEAS: the electrode and collision counters of a measurement window.
template <int U, bool MCC, int MINB, bool MEAS>
__global__ void __launch_bounds__(ES_THREADS, MINB)
    batch_step_kernel(const __grid_constant__ StepPlanes pl, const BatchDisc *__restrict__ desc,
                      const uint32_t *__restrict__ counts, uint32_t D, const StepRoles r, uint32_t ef_pad,
                      int stages, int copies, uint32_t epoch) {
    extern __shared__ __align__(128) unsigned char smem[];
    __shared__ uint32_t offs[3][StepShape<U, MCC>::NSEG];
    __shared__ uint32_t s_base[3];
    __shared__ uint32_t wsum[ES_WARPS];
    __shared__ StepDisc s_dc;
    __shared__ cudapic_grid s_g;
    __shared__ uint32_t s_d, s_off;
    __shared__ uint32_t ccnt[3][StepShape<U, MCC>::NSEG];
    const StepSmem<U, MCC> sm(smem, stages, copies, ef_pad, offs, s_base, ccnt);
    uint32_t *P = reinterpret_cast<uint32_t *>(sm.end(stages));  // [D + 1]
    step_smem_init(sm, stages, copies, ef_pad);
    grid_dep_wait();
    plan_prefix([&](uint32_t d) { return counts[d]; }, D, P, wsum);
    uint32_t it = 0;
    bool ok = true;
    uint32_t d;
    {
        uint32_t chunk, beg, end;
        cta_share(P[D], chunk, beg, end);
        d = first_discharge(P, D, beg);
    }
    // Nothing of the plan stays in registers across a segment (the tile
    // loop needs them all): the share is recomputed from the plan and the
    // discharge index reloaded from shared memory after each segment.
    for (;; ++d) {
        uint32_t chunk, beg, end;
        cta_share(P[D], chunk, beg, end);
        if (d >= D || P[d] >= end) break;
        const uint32_t n = counts[d];
        const uint32_t lo = max(beg, P[d]) - P[d];
        const uint32_t hi = min(end, P[d] + n) - P[d];
        if (lo >= hi) continue;
        if (threadIdx.x == 0) {
            const BatchDisc &dd = desc[d];
            s_d = d;
            s_off = dd.off;
            s_g = dd.g;
            StepDisc dc;
            dc.efield = dd.efield;
            dc.sigma_tot = MCC ? dd.sigma_tot_e : dd.sigma_tot_i;
            dc.cs = dd.cs;
            dc.sigma_max = dd.sigma_max_e;
            dc.factor = MCC ? dd.g.factor_e : dd.g.factor_i;
            dc.dt = MCC ? dd.g.dt_e : dd.g.dt_i;
            dc.alive = dd.counters + (MCC ? 2 : 5);
            dc.n_i = dd.counters + 1;
            dc.dens = MCC ? dd.e_dens[r.dens] : dd.i_dens[r.dens];
            dc.dens_i = dd.i_dens[r.dens_i];
            dc.wall = MEAS ? dd.wall + (MCC ? 0 : 1) : nullptr;
            dc.coll = MEAS && MCC ? dd.mcount : nullptr;
            s_dc = dc;
        }
        __syncthreads();
        if (ok) {
            // the grid constants in registers: the tile loop's shared-memory
            // stores would otherwise force reloads of s_g at every use
            const cudapic_grid g = s_g;
            uint32_t live = 0;
            ok = step_segment<U, MCC, true, MEAS>(pl, s_dc, g, s_g, s_off, lo, hi, sm, stages, copies, ef_pad, epoch,
                                                  it, live);
            add_work(s_g.work, live);
        }
        d = lds_volatile(&s_d);
        {
            uint32_t chunk2, beg2, end2;
            cta_share(P[D], chunk2, beg2, end2);
            const uint32_t n2 = counts[d];
            const uint32_t expected = (P[d] + n2 - 1) / chunk2 - P[d] / chunk2 + 1;
            uint32_t *ctr = desc[d].counters;
            publish_count_of(ctr + 6, ctr + (MCC ? 0 : 1), ctr + (MCC ? 2 : 5), s_g.capacity, expected);
        }
        __syncthreads();  // s_dc, s_g, s_d and s_off are rewritten for the next segment
    }
}

// The in-place electron step of every discharge (inplace.cuh), stream pass:
// the batch's concatenated electron slots cut into equal per-CTA shares as
// in batch_step_kernel, each segment run with that discharge's field,
// tables, next density and collider list (the discharge's range of the
// other sides' planes).  No count changes: nothing is published.
template <bool MEAS>
__global__ void __launch_bounds__(IP_THREADS, 4)
    batch_inplace_kernel(const __grid_constant__ InplacePlanes pl, const __grid_constant__ CollList list,
                         const BatchDisc *__restrict__ desc, const uint32_t *__restrict__ counts, uint32_t D,
                         int dens_role, uint32_t ef_pad, int copies, uint32_t epoch, uint32_t pf) {
    extern __shared__ __align__(128) unsigned char smem[];
    __shared__ uint32_t wsum[ES_WARPS];
    __shared__ StepDisc s_dc;
    __shared__ cudapic_grid s_g;
    __shared__ uint32_t s_d, s_off;
    const InplaceSmem sm(smem, copies, ef_pad);
    uint32_t *P = reinterpret_cast<uint32_t *>(sm.end());  // [D + 1]
    inplace_smem_init(sm, copies, ef_pad);
    grid_dep_wait();
    plan_prefix([&](uint32_t d) { return counts[d]; }, D, P, wsum);
    uint32_t d;
    {
        uint32_t chunk, beg, end;
        cta_share(P[D], chunk, beg, end);
        d = first_discharge(P, D, beg);
    }
    for (;; ++d) {
        uint32_t chunk, beg, end;
        cta_share(P[D], chunk, beg, end);
        if (d >= D || P[d] >= end) break;
        const uint32_t n = counts[d];
        const uint32_t lo = max(beg, P[d]) - P[d];
        const uint32_t hi = min(end, P[d] + n) - P[d];
        if (lo >= hi) continue;
        if (threadIdx.x == 0) {
            const BatchDisc &dd = desc[d];
            s_d = d;
            s_off = dd.off;
            s_g = dd.g;
            StepDisc dc;
            dc.efield = dd.efield;
            dc.sigma_tot = dd.sigma_tot_e;
            dc.cs = dd.cs;
            dc.sigma_max = dd.sigma_max_e;
            dc.factor = dd.g.factor_e;
            dc.dt = dd.g.dt_e;
            dc.alive = dd.counters + CTR_COLL_COUNT;   // the collider count
            dc.n_i = nullptr;
            dc.dens = dd.e_dens[dens_role];
            dc.dens_i = nullptr;
            dc.wall = MEAS ? dd.wall : nullptr;
            dc.coll = nullptr;
            s_dc = dc;
        }
        __syncthreads();
        {
            const cudapic_grid g = s_g;
            const uint32_t off = s_off;
            const CollList mine{list.slot + off, list.vx + off, list.vy + off, list.vz + off,
                                list.r0 + off,   list.r1 + off, list.r2 + off, list.r3 + off};
            uint32_t live = 0;
            inplace_segment<true, MEAS>(pl, s_dc, g, s_g, off, lo, hi, sm, copies, ef_pad, epoch, mine,
                                        dcp<true>(s_dc.alive), live, pf);
            add_work(s_g.work, live);
        }
        d = lds_volatile(&s_d);
        __syncthreads();  // s_dc, s_g, s_d and s_off are rewritten for the next segment
    }
}

// The in-place electron step of every discharge, scatter pass: the listed
// colliders of all discharges (each discharge's count clamped to its
// capacity) cut into per-CTA shares; each segment scatters with that
// discharge's table, counters and next densities.  The last CTA of the
// launch adds the collision counts (measurement) and empties every list.
template <bool MEAS>
__global__ void __launch_bounds__(IP_THREADS)
    batch_scatter_kernel(const __grid_constant__ InplacePlanes pl, const __grid_constant__ CollList list,
                         const BatchDisc *__restrict__ desc, uint32_t D, int dens_role, int dens_i_role,
                         uint32_t *ticket) {
    extern __shared__ __align__(16) uint32_t sc_smem[];
    uint32_t *P = sc_smem;  // [D + 1]
    __shared__ uint32_t wsum[ES_WARPS];
    grid_dep_wait();
    auto count = [&](uint32_t d) {
        const BatchDisc &dd = desc[d];
        return min(*(volatile uint32_t *)(dd.counters + CTR_COLL_COUNT), dd.g.capacity);
    };
    plan_prefix(count, D, P, wsum);  // the counts do not change until the last CTA has its ticket
    // the batch's records in chunks of 32, chunk c to CTA c mod gridDim (no
    // block barrier per discharge); each lane finds its discharge in the plan.
    // The plan rounds every count up to a multiple of 4: an index past the
    // discharge's own count (at most 3 per discharge) is skipped, its record
    // slot holds nothing of this step.
    const uint32_t lane = threadIdx.x & 31u, warp = threadIdx.x >> 5;
    const uint32_t total = P[D];
    const uint32_t chunks = (total + 31u) / 32u, per_pass = gridDim.x * (blockDim.x >> 5);
    for (uint32_t c = blockIdx.x + warp * gridDim.x; c < chunks; c += per_pass) {
        const uint32_t k = c * 32u + lane;
        if (k < total) {
            uint32_t lo = 0, hi = D;  // the last d with P[d] <= k: P[d] <= k < P[d + 1]
            while (hi - lo > 1u) {
                const uint32_t mid = (lo + hi) >> 1;
                if (P[mid] <= k) lo = mid;
                else hi = mid;
            }
            const uint32_t kd = k - P[lo];
            if (kd < count(lo)) {
                const BatchDisc &dd = desc[lo];
                inplace_scatter(pl, list, dd.off, kd, dd.cs, dd.counters + 0, dd.counters + 1, dd.g,
                                dd.e_dens[dens_role], dd.i_dens[dens_i_role]);
            }
        }
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        __threadfence();  // one per CTA: its spawns before its ticket
        const uint32_t t = atomicAdd(ticket, 1u);
        P[0] = t == gridDim.x - 1;
    }
    __syncthreads();
    if (P[0]) {  // the last CTA: every list has been read
        __threadfence();
        for (uint32_t d = threadIdx.x; d < D; d += IP_THREADS) {
            const BatchDisc &dd = desc[d];
            uint32_t *c = dd.counters + CTR_COLL_COUNT;
            if (MEAS) atomicAdd(dd.mcount, (unsigned long long)min(*c, dd.g.capacity));
            *c = 0u;
        }
        if (threadIdx.x == 0) *ticket = 0u;
    }
}

// check_collisions_i / collision_i (Rust-CUDA/src/main.rs:1167-1292) of every
// discharge, in place.  Plain coalesced loads; colliders go to warp-private
// queues (slot and RNG state before the test) drained 32 at a time, as in
// the resident-table kernel of kernels_mcc.cu, with each discharge's table
// read from global memory.
constexpr int BC_U = 2;
constexpr int BC_QCAP = 32 + 32 * BC_U;

struct IonCollIO {
    float *vx, *vy, *vz;
    uint32_t *rng0, *rng1, *rng2, *rng3;
    const float *sigma_tot, *cs;
    unsigned long long *coll;
    float ion_k;
};

__global__ void __launch_bounds__(ES_THREADS)
    batch_collisions_i_kernel(const __grid_constant__ SidePlanes ions, const BatchDisc *__restrict__ desc,
                              uint32_t D, int measure) {
    extern __shared__ __align__(16) uint32_t bc_smem[];
    uint32_t *P = bc_smem;                                   // [D + 1]
    __shared__ uint32_t queue[ES_WARPS][5][BC_QCAP];
    __shared__ uint32_t wsum[ES_WARPS];
    __shared__ IonCollIO s_io;
    __shared__ cudapic_grid s_g;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const unsigned lt = lanemask_lt();
    grid_dep_wait();
    auto count = [&](uint32_t d) {
        const BatchDisc &dd = desc[d];
        return min(*(volatile uint32_t *)(dd.counters + 1), dd.g.capacity);
    };
    plan_prefix(count, D, P, wsum);
    uint32_t chunk, beg, end;
    cta_share(P[D], chunk, beg, end);
    uint32_t (*wq)[BC_QCAP] = queue[warp];
    for (uint32_t d = first_discharge(P, D, beg); d < D && P[d] < end; ++d) {
        const uint32_t n = count(d);  // unchanged during the kernel
        const uint32_t lo = max(beg, P[d]) - P[d];
        const uint32_t hi = min(end, P[d] + n) - P[d];
        if (lo >= hi) continue;
        const BatchDisc &dd = desc[d];
        if (tid == 0) {
            s_g = dd.g;
            IonCollIO io;
            io.vx = ions.vx + dd.off;
            io.vy = ions.vy + dd.off;
            io.vz = ions.vz + dd.off;
            io.rng0 = ions.rng0 + dd.off;
            io.rng1 = ions.rng1 + dd.off;
            io.rng2 = ions.rng2 + dd.off;
            io.rng3 = ions.rng3 + dd.off;
            io.sigma_tot = dd.sigma_tot_i;
            io.cs = dd.cs;
            io.coll = measure ? dd.mcount + 1 : nullptr;
            io.ion_k = dd.ion_k;
            s_io = io;
        }
        __syncthreads();
        const IonCollIO &io = s_io;
        const cudapic_grid &g = s_g;
        const GlobalTable table{io.sigma_tot};
        auto drain = [&](uint32_t first, uint32_t cnt) {
            if (io.coll && lane == 0) atomicAdd(io.coll, (unsigned long long)cnt);
            if ((uint32_t)lane < cnt) {
                const uint32_t q = first + lane;
                const uint32_t i = wq[0][q];
                Xoshiro128p rs{wq[1][q], wq[2][q], wq[3][q], wq[4][q]};
                const float vxi = io.vx[i], vyi = io.vy[i], vzi = io.vz[i];
                const IonTest t = test_ion(vxi, vyi, vzi, rs, table, g);
                collide_ion(i, t.idx, vxi, vyi, vzi, t.vxa, t.vya, t.vza, rs, io.cs, io.vx, io.vy, io.vz, g);
                io.rng0[i] = rs.s0;
                io.rng1[i] = rs.s1;
                io.rng2[i] = rs.s2;
                io.rng3[i] = rs.s3;
            }
            __syncwarp();
        };
        uint32_t qn = 0;
        for (uint32_t b0 = lo; b0 < hi; b0 += ES_THREADS * BC_U) {
            uint32_t s[BC_U][4];
            float v[BC_U][3];
#pragma unroll
            for (int u = 0; u < BC_U; ++u) {
                const uint32_t i = b0 + (uint32_t)u * ES_THREADS + tid;
                if (i < hi) {
                    s[u][0] = io.rng0[i];
                    s[u][1] = io.rng1[i];
                    s[u][2] = io.rng2[i];
                    s[u][3] = io.rng3[i];
                    v[u][0] = io.vx[i];
                    v[u][1] = io.vy[i];
                    v[u][2] = io.vz[i];
                }
            }
#pragma unroll
            for (int u = 0; u < BC_U; ++u) {
                const uint32_t i = b0 + (uint32_t)u * ES_THREADS + tid;
                bool collide = false;
                if (i < hi) {
                    Xoshiro128p rs{s[u][0], s[u][1], s[u][2], s[u][3]};
                    collide = ion_collides(v[u][0], v[u][1], v[u][2], rs, table, g, io.ion_k);
                    if (!collide) {
                        io.rng0[i] = rs.s0;
                        io.rng1[i] = rs.s1;
                        io.rng2[i] = rs.s2;
                        io.rng3[i] = rs.s3;
                    }
                }
                const unsigned m = __ballot_sync(0xffffffffu, collide);
                if (collide) {
                    const uint32_t q = qn + __popc(m & lt);
                    wq[0][q] = i;
                    wq[1][q] = s[u][0];
                    wq[2][q] = s[u][1];
                    wq[3][q] = s[u][2];
                    wq[4][q] = s[u][3];
                }
                qn += __popc(m);
            }
            __syncwarp();
            while (qn >= 32) {
                qn -= 32;
                drain(qn, 32);
            }
        }
        if (qn) drain(0, qn);
        __syncthreads();  // s_io and s_g are rewritten for the next segment
    }
}

// accumulate_eepf (Rust-CUDA/src/main.rs:1301-1339) of every discharge with
// the centre-energy sums of the report; one shared histogram per segment.
__global__ void __launch_bounds__(ES_THREADS)
    batch_eepf_kernel(const __grid_constant__ SidePlanes electrons, const BatchDisc *__restrict__ desc, uint32_t D) {
    extern __shared__ __align__(16) uint32_t be_smem[];
    uint32_t *P = be_smem;  // [D + 1]
    __shared__ uint32_t hist[N_EEPF];
    __shared__ uint32_t wsum[ES_WARPS];
    const int tid = threadIdx.x;
    for (uint32_t k = tid; k < N_EEPF; k += ES_THREADS) hist[k] = 0u;
    grid_dep_wait();
    auto count = [&](uint32_t d) {
        const BatchDisc &dd = desc[d];
        return min(*(volatile uint32_t *)(dd.counters + 0), dd.g.capacity);
    };
    plan_prefix(count, D, P, wsum);
    uint32_t chunk, beg, end;
    cta_share(P[D], chunk, beg, end);
    for (uint32_t d = first_discharge(P, D, beg); d < D && P[d] < end; ++d) {
        const uint32_t n = count(d);  // unchanged during the kernel
        const uint32_t lo = max(beg, P[d]) - P[d];
        const uint32_t hi = min(end, P[d] + n) - P[d];
        if (lo >= hi) continue;
        const BatchDisc &dd = desc[d];
        const cudapic_grid &g = dd.g;
        const float *x = electrons.x + dd.off, *vx = electrons.vx + dd.off, *vy = electrons.vy + dd.off,
                    *vz = electrons.vz + dd.off;
        const float *ef = dd.efield;
        const float min_x = g.min_x, max_x = g.max_x, inv_dx = g.inv_dx, kick = g.eepf_half_kick;
        const float half_me = g.half_me_over_e;
        const uint32_t n_g = g.n_g;
        double e_sum = 0.0;
        unsigned long long e_cnt = 0;
        for (uint32_t i = lo + tid; i < hi; i += ES_THREADS) {
            const float xi = x[i];
            if (xi <= min_x || xi >= max_x) continue;
            const float pos = xi * inv_dx;
            const int p = cell_of(pos, n_g);
            const float c2 = pos - (float)p;
            const float e_x = (1.0f - c2) * __ldg(ef + p) + c2 * __ldg(ef + p + 1);
            const float mvx = vx[i] - 0.5f * e_x * kick;
            const float vyi = vy[i], vzi = vz[i];
            const float v2 = mvx * mvx + vyi * vyi + vzi * vzi;
            const float energy = half_me * v2;
            const float binf = energy / DE_EEPF_F;
            if (binf < (float)N_EEPF) atomicAdd(&hist[(uint32_t)binf], 1u);
            e_sum += (double)energy;
            ++e_cnt;
        }
        for (int o = 16; o > 0; o >>= 1) {
            e_sum += __shfl_down_sync(0xffffffffu, e_sum, o);
            e_cnt += __shfl_down_sync(0xffffffffu, e_cnt, o);
        }
        if ((tid & 31) == 0 && e_cnt) {
            atomicAdd(dd.esum, e_sum);
            atomicAdd(dd.mcount + 2, e_cnt);
        }
        __syncthreads();
        for (uint32_t k = tid; k < N_EEPF; k += ES_THREADS) {
            if (hist[k]) {
                atomicAdd(&dd.eepf[k], hist[k]);
                hist[k] = 0u;
            }
        }
        __syncthreads();
    }
}

namespace {

template <int U, bool MCC, int MINB, bool MEAS>
int launch_batch_step_t(const StepPlanes &pl, const BatchDisc *desc, const uint32_t *counts, uint32_t D,
                        uint64_t cap_sum, uint32_t max_n_g, const StepRoles &r, cudaStream_t stream,
                        const cudapic_tuning &t) {
    constexpr int TILE = StepShape<U, MCC>::TILE;
    int stages = std::min(std::max(t.step_stages, 2), ES_MAX_STAGES);
    int copies = std::max(1, std::min(t.density_copies, ES_WARPS));
    const uint32_t ef_pad = (max_n_g + 3u) & ~3u;
    const size_t plan = (size_t)(D + 1) * sizeof(uint32_t);
    auto bytes = [&]() { return step_smem_bytes<U, MCC>(stages, copies, ef_pad) + plan; };
    const size_t budget = (size_t)max_smem_optin();
    while (bytes() > budget && stages > 2) --stages;
    // below 4 copies the f32 histogram (copies = 0) takes over: 8 B per node
    auto fewer = [&]() { copies = copies / 2 < 4 ? 0 : copies / 2; };
    while (bytes() > budget && copies > 0) fewer();
    if (bytes() > budget) return fail(CUDAPIC_ERR_ARG, "batch step: n_g too large");
    auto kern = batch_step_kernel<U, MCC, MINB, MEAS>;
    int per_sm = 0;
    auto occupancy = [&]() {
        CUDAPIC_CHECK(check_cuda(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes()),
                                 "cudaFuncSetAttribute(batch step)"));
        return check_cuda(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, ES_THREADS, bytes()),
                          "occupancy(batch step)");
    };
    CUDAPIC_CHECK(occupancy());
    // large grids: fewer histogram copies rather than fewer CTAs per SM
    while (per_sm < t.step_ctas_per_sm && copies > 0) {
        fewer();
        CUDAPIC_CHECK(occupancy());
    }
    const size_t smem = bytes();
    per_sm = std::min(std::max(per_sm, 1), t.step_ctas_per_sm);
    const unsigned grid = persistent_grid(per_sm, (cap_sum + TILE - 1) / TILE);
    const uint32_t per_tile = copies ? (uint32_t)((ES_WARPS + copies - 1) / copies) * U * 32u : 1u;
    const uint32_t epoch = copies ? std::max(1u, DEP_MAX_PER_COPY / per_tile) : 0xffffffffu;
    return launch_kernel(MCC ? "batch_step_electrons" : "batch_push_ions", kern, dim3(grid), dim3(ES_THREADS), smem,
                         stream, pl, desc, counts, D, r, ef_pad, stages, copies, epoch);
}

}  // namespace

template <bool MEAS>
int launch_batch_step_m(bool mcc, const StepPlanes &pl, const BatchDisc *desc, const uint32_t *counts, uint32_t D,
                        uint64_t cap_sum, uint32_t max_n_g, const StepRoles &r, cudaStream_t stream,
                        const cudapic_tuning &t) {
    const bool three = t.step_ctas_per_sm >= 3;
    if (mcc) {
        if (t.step_rows == 4)
            return three ? launch_batch_step_t<4, true, 3, MEAS>(pl, desc, counts, D, cap_sum, max_n_g, r, stream, t)
                         : launch_batch_step_t<4, true, 2, MEAS>(pl, desc, counts, D, cap_sum, max_n_g, r, stream, t);
        if (t.step_rows == 1)
            return three ? launch_batch_step_t<1, true, 3, MEAS>(pl, desc, counts, D, cap_sum, max_n_g, r, stream, t)
                         : launch_batch_step_t<1, true, 2, MEAS>(pl, desc, counts, D, cap_sum, max_n_g, r, stream, t);
        return three ? launch_batch_step_t<2, true, 3, MEAS>(pl, desc, counts, D, cap_sum, max_n_g, r, stream, t)
                     : launch_batch_step_t<2, true, 2, MEAS>(pl, desc, counts, D, cap_sum, max_n_g, r, stream, t);
    }
    return t.step_rows == 4
               ? launch_batch_step_t<4, false, 3, MEAS>(pl, desc, counts, D, cap_sum, max_n_g, r, stream, t)
               : launch_batch_step_t<2, false, 3, MEAS>(pl, desc, counts, D, cap_sum, max_n_g, r, stream, t);
}

int launch_batch_step(bool mcc, const StepPlanes &pl, const BatchDisc *desc, const uint32_t *counts, uint32_t D,
                      uint64_t cap_sum, uint32_t max_n_g, const StepRoles &r, cudaStream_t stream) {
    if (D == 0 || D > BATCH_MAX_DISCHARGES) return fail(CUDAPIC_ERR_ARG, "batch step: bad discharge count");
    const cudapic_tuning t = tuning();
    if (r.measure) return launch_batch_step_m<true>(mcc, pl, desc, counts, D, cap_sum, max_n_g, r, stream, t);
    return launch_batch_step_m<false>(mcc, pl, desc, counts, D, cap_sum, max_n_g, r, stream, t);
}

int launch_batch_inplace(const InplacePlanes &pl, const CollList &list, const BatchDisc *desc, const uint32_t *counts,
                         uint32_t D, uint64_t cap_sum, uint32_t max_n_g, const StepRoles &r, cudaStream_t stream) {
    if (D == 0 || D > BATCH_MAX_DISCHARGES) return fail(CUDAPIC_ERR_ARG, "batch in-place step: bad discharge count");
    const cudapic_tuning t = tuning();
    const uint32_t ef_pad = (max_n_g + 3u) & ~3u;
    const size_t plan = (size_t)(D + 1) * sizeof(uint32_t);
    int copies = t.inplace_copies < 0 ? 0 : std::max(1, std::min(t.inplace_copies, IP_WARPS));  // 0: f32
    auto bytes = [&]() { return inplace_smem_bytes(copies, ef_pad) + plan; };
    const size_t budget = (size_t)max_smem_optin();
    while (bytes() > budget && copies > 0) copies = copies / 2 < 4 ? 0 : copies / 2;
    if (bytes() > budget) return fail(CUDAPIC_ERR_ARG, "batch in-place step: n_g too large");
    auto kern = r.measure ? batch_inplace_kernel<true> : batch_inplace_kernel<false>;
    int per_sm = 0;
    auto occupancy = [&]() {
        CUDAPIC_CHECK(check_cuda(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes()),
                                 "cudaFuncSetAttribute(batch in-place step)"));
        return check_cuda(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, IP_THREADS, bytes()),
                          "occupancy(batch in-place step)");
    };
    CUDAPIC_CHECK(occupancy());
    // large grids: fewer copies rather than fewer CTAs; below 4 copies the
    // drains would come every few rounds, so the f32 histogram takes over
    while (per_sm < t.inplace_ctas_per_sm && copies > 0) {
        copies = copies / 2 < 4 ? 0 : copies / 2;
        CUDAPIC_CHECK(occupancy());
    }
    per_sm = std::min(std::max(per_sm, 1), t.inplace_ctas_per_sm);
    const unsigned grid = persistent_grid(per_sm, (cap_sum + IP_ROUND - 1) / IP_ROUND);
    const uint32_t per_round = copies ? (uint32_t)((IP_WARPS + copies - 1) / copies) * 32u * IP_ROW : 1u;
    const uint32_t epoch = copies ? std::max(1u, DEP_MAX_PER_COPY / per_round) : 0xffffffffu;
    return launch_kernel("batch_inplace_electrons", kern, dim3(grid), dim3(IP_THREADS), bytes(), stream, pl, list,
                         desc, counts, D, r.dens, ef_pad, copies, epoch, (uint32_t)std::max(t.inplace_prefetch, 0));
}

int launch_batch_scatter(const InplacePlanes &pl, const CollList &list, const BatchDisc *desc, uint32_t D,
                         uint64_t cap_sum, const StepRoles &r, uint32_t *ticket, cudaStream_t stream) {
    if (D == 0 || D > BATCH_MAX_DISCHARGES) return fail(CUDAPIC_ERR_ARG, "batch scatter: bad discharge count");
    const size_t plan = (size_t)(D + 1) * sizeof(uint32_t);
    auto kern = r.measure ? batch_scatter_kernel<true> : batch_scatter_kernel<false>;
    const unsigned grid = persistent_grid(tuning().scatter_ctas_per_sm, (cap_sum + IP_THREADS - 1) / IP_THREADS);
    return launch_kernel("batch_scatter_electrons", kern, dim3(grid), dim3(IP_THREADS), plan, stream, pl, list, desc,
                         D, r.dens, r.dens_i, ticket);
}

int launch_batch_collisions_i(const SidePlanes &ions, const BatchDisc *desc, uint32_t D, uint64_t cap_sum,
                              int measure, cudaStream_t stream) {
    if (D == 0 || D > BATCH_MAX_DISCHARGES) return fail(CUDAPIC_ERR_ARG, "batch collisions: bad discharge count");
    const size_t smem = (size_t)(D + 1) * sizeof(uint32_t);
    const unsigned grid = persistent_grid(4, (cap_sum + ES_THREADS * BC_U - 1) / (ES_THREADS * BC_U));
    return launch_kernel("batch_collisions_i", batch_collisions_i_kernel, dim3(grid), dim3(ES_THREADS), smem, stream,
                         ions, desc, D, measure);
}

int launch_batch_eepf(const SidePlanes &electrons, const BatchDisc *desc, uint32_t D, uint64_t cap_sum,
                      cudaStream_t stream) {
    if (D == 0 || D > BATCH_MAX_DISCHARGES) return fail(CUDAPIC_ERR_ARG, "batch eepf: bad discharge count");
    const size_t smem = (size_t)(D + 1) * sizeof(uint32_t);
    const unsigned grid = persistent_grid(2, (cap_sum + ES_THREADS - 1) / ES_THREADS);
    return launch_kernel("batch_eepf", batch_eepf_kernel, dim3(grid), dim3(ES_THREADS), smem, stream, electrons, desc,
                         D);
}

}  // namespace cudapic
