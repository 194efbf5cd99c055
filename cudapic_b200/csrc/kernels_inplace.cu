// kernels_inplace.cu -- the in-place electron step of one discharge
// (inplace.cuh): the stream pass and the scatter pass as two persistent
// kernels, their launchers (shared with the driver) and the C entry points;
// plus eduPIC's same-step collisions of new electrons (a driver option).
//
// Reference: the electron half of a time step, move_and_compact
// (Rust-CUDA/src/main.rs:566-678) + check_collisions_e / collision_e
// (:971-1165) + the next step's get_density (:356-406), as the compacting
// fused step (kernels_step.cu) does it, but with every electron kept in its
// slot: no compaction, 56 B of HBM traffic per electron (x, v, RNG read;
// x, vx, RNG written) against 64 B, plus the colliders' records and their
// scattered velocities.
#include <algorithm>
#include <type_traits>

#include "batch_internal.h"
#include "inplace.cuh"
#include "internal.h"
#include "poisson.cuh"

namespace cudapic {

template <bool MEAS>
__global__ void __launch_bounds__(IP_THREADS, 4)
    electron_inplace_kernel(const InplacePlanes pl, const float *__restrict__ efield,
                            const float *__restrict__ sigma_tot_e, const float *__restrict__ cs, float sigma_max,
                            const uint32_t *n_active,
                            const CollList list, uint32_t *count, float *dens_e,
                            const __grid_constant__ cudapic_grid g, uint32_t ef_pad, int copies, uint32_t epoch,
                            cudapic_wall_counters *wall, uint32_t *spawn_from, uint32_t pf) {
    extern __shared__ __align__(128) unsigned char smem[];
    const InplaceSmem sm(smem, copies, ef_pad);
    inplace_smem_init(sm, copies, ef_pad);
    grid_dep_wait();
    const uint32_t n = load_count(n_active, g.capacity, g.dev_err);
    // the first slot the scatter pass can give a spawned electron (n_e does not change in this pass)
    if (spawn_from && blockIdx.x == 0 && threadIdx.x == 0) *spawn_from = n;
    // balanced contiguous shares, multiples of 4 (16-byte aligned loads)
    const uint32_t chunk = ((n + gridDim.x - 1) / gridDim.x + 3u) & ~3u;
    const uint32_t beg = min(n, blockIdx.x * chunk);
    const uint32_t end = min(n, beg + chunk);
    StepDisc dc;
    dc.efield = efield;
    dc.sigma_tot = sigma_tot_e;
    dc.cs = cs;
    dc.sigma_max = sigma_max;
    dc.factor = g.factor_e;
    dc.dt = g.dt_e;
    dc.alive = nullptr;
    dc.n_i = nullptr;
    dc.dens = dens_e;
    dc.dens_i = nullptr;
    dc.wall = wall;
    dc.coll = nullptr;
    uint32_t live = 0;
    inplace_segment<false, MEAS>(pl, dc, g, g, 0u, beg, end, sm, copies, ef_pad, epoch, list, count, live, pf);
    add_work(g.work, live);
}

// SOLVE: 0, or the last CTA also solves the next step's field (1: FP64
// scans, 2: f32 scans) with the solve kernel's own shape for N_G <= 1024
// (one node per thread, so the sums are added in the same order and the
// field is bit-identical to the separate kernel's): CTAs of 1024 threads,
// dynamic shared memory n_g x the scan type.
constexpr int SC_SOLVE_THREADS = 1024;

template <int SOLVE>
__global__ void __launch_bounds__(SOLVE ? SC_SOLVE_THREADS : IP_THREADS)
    electron_scatter_kernel(const InplacePlanes pl, const CollList list, const float *__restrict__ cs,
                            uint32_t *count, uint32_t *ticket, uint32_t *n_e, uint32_t *n_i,
                            const __grid_constant__ cudapic_grid g, float *dens_e, float *dens_i,
                            unsigned long long *coll, const PoissonAhead ahead) {
    __shared__ uint32_t s_last;
    grid_dep_wait();
    const uint32_t n = min(*count, g.capacity);  // read before this CTA takes its ticket
    // chunks of 32 consecutive records, chunk c to CTA c % gridDim (a warp
    // reads its records coalesced, and a few thousand colliders still reach
    // every SM instead of the first few CTAs)
    const uint32_t lane = threadIdx.x & 31u, warp = threadIdx.x >> 5;
    const uint32_t chunks = (n + 31u) / 32u, per_pass = gridDim.x * (blockDim.x >> 5);
    for (uint32_t c = blockIdx.x + warp * gridDim.x; c < chunks; c += per_pass) {
        const uint32_t k = c * 32u + lane;
        if (k < n) inplace_scatter(pl, list, 0u, k, cs, n_e, n_i, g, dens_e, dens_i);
    }
    // the last CTA counts the collisions and empties the list for the next
    // step (every CTA read the count before its ticket: no fence needed for
    // that; one per CTA orders its spawns and deposits before the ticket)
    __syncthreads();
    if (threadIdx.x == 0) {
        __threadfence();
        const uint32_t t = atomicAdd(ticket, 1u);
        s_last = t == gridDim.x - 1;
        if (s_last) {
            __threadfence();
            if (coll) atomicAdd(coll, (unsigned long long)n);
            *count = 0u;
            *ticket = 0u;
        }
    }
    if (SOLVE) {
        __syncthreads();
        if (s_last)  // every deposit of this step is in: the next step's solve (clears its collectors)
            poisson_body<typename std::conditional<SOLVE == 1, double, float>::type, 1>(
                ahead.e_density, ahead.i_density, ahead.pot, ahead.efield, 0.0f, ahead.pot0_table,
                ahead.step_counter, g, ahead.zero_a, ahead.zero_b);
    }
}

// eduPIC's semantics for electrons born in a step (C/eduPIC.cc:669-703: its
// collision loop runs up to the N_e that the ionizations of the same loop
// keep raising, so a new electron is tested -- and may collide and ionize --
// in the step of its birth; the GPU reference tests it only from the next
// step, Rust-CUDA/src/main.rs:992).  One CTA tests the electrons appended
// since *spawn_from (one draw of each new slot's stream, the exact test) and
// scatters the colliders, in rounds until no new slot appears (at most 64).
__global__ void __launch_bounds__(IP_THREADS)
    spawn_collide_kernel(const InplacePlanes pl, const float *__restrict__ sigma_tot_e,
                         const float *__restrict__ cs, const uint32_t *spawn_from, uint32_t *n_e, uint32_t *n_i,
                         const __grid_constant__ cudapic_grid g, float *dens_e, float *dens_i,
                         unsigned long long *coll) {
    __shared__ uint32_t s_lo, s_hi;
    grid_dep_wait();
    if (threadIdx.x == 0) {
        s_lo = *spawn_from;
        s_hi = min(*(volatile uint32_t *)n_e, g.capacity);
    }
    __syncthreads();
    for (int round = 0; round < 64; ++round) {
        const uint32_t lo = s_lo, hi = s_hi;
        if (lo >= hi) break;
        uint32_t collided = 0;
        for (uint32_t k = lo + threadIdx.x; k < hi; k += IP_THREADS) {
            Xoshiro128p rs{pl.rng0[k], pl.rng1[k], pl.rng2[k], pl.rng3[k]};
            const float vxi = pl.vx[k], vyi = pl.vy[k], vzi = pl.vz[k];
            const Test t = test_electron(vxi, vyi, vzi, rs, GlobalTable{sigma_tot_e}, g);
            if (t.collide) {
                collide_electron_t<true>(0u, k, t.idx, vxi, vyi, vzi, rs, cs, pl.x, pl.vx, pl.vy, pl.vz, pl.ix,
                                         pl.ivx, pl.ivy, pl.ivz, n_e, n_i, g, dens_e, dens_i);
                ++collided;
            }
            pl.rng0[k] = rs.s0;
            pl.rng1[k] = rs.s1;
            pl.rng2[k] = rs.s2;
            pl.rng3[k] = rs.s3;
        }
        if (coll) {
            const uint32_t c = __reduce_add_sync(0xffffffffu, collided);
            if ((threadIdx.x & 31) == 0 && c) atomicAdd(coll, (unsigned long long)c);
        }
        __threadfence();
        __syncthreads();
        if (threadIdx.x == 0) {
            s_lo = hi;
            s_hi = min(*(volatile uint32_t *)n_e, g.capacity);
        }
        __syncthreads();
    }
}

int launch_spawn_collide(const InplacePlanes &pl, const float *sigma_tot_e, const float *cs,
                         const uint32_t *spawn_from, uint32_t *n_e, uint32_t *n_i, const cudapic_grid &g,
                         cudaStream_t stream, float *dens_e, float *dens_i, unsigned long long *coll) {
    return launch_kernel("spawn_collide_e", spawn_collide_kernel, dim3(1), dim3(IP_THREADS), 0, stream, pl,
                         sigma_tot_e, cs, spawn_from, n_e, n_i, g, dens_e, dens_i, coll);
}

bool inplace_eligible(const void *const *planes, int count, uint32_t capacity) {
    return electron_step_eligible(planes, count, capacity);
}

int launch_electron_inplace(const InplacePlanes &pl, const float *efield, const float *sigma_tot_e, const float *cs,
                            float sigma_max, const uint32_t *n_active, const CollList &list, uint32_t *count,
                            float *dens_e, const cudapic_grid &g, cudaStream_t stream, cudapic_wall_counters *wall,
                            uint32_t *spawn_from) {
    if (g.capacity > 0x80000000u)  // a record's slot word keeps bit 31 for the event
        return fail(CUDAPIC_ERR_ARG, "step_electrons_inplace: capacity above 2^31");
    const cudapic_tuning t = tuning();
    const uint32_t ef_pad = (g.n_g + 3u) & ~3u;
    int copies = t.inplace_copies < 0 ? 0 : std::max(1, std::min(t.inplace_copies, IP_WARPS));  // 0: f32
    const size_t budget = (size_t)max_smem_optin();
    while (inplace_smem_bytes(copies, ef_pad) > budget && copies > 0) copies = copies / 2 < 4 ? 0 : copies / 2;
    if (inplace_smem_bytes(copies, ef_pad) > budget)
        return fail(CUDAPIC_ERR_ARG, "step_electrons_inplace: n_g too large");
    auto kern = wall ? electron_inplace_kernel<true> : electron_inplace_kernel<false>;
    int per_sm = 0;
    auto occupancy = [&]() {
        const size_t smem = inplace_smem_bytes(copies, ef_pad);
        CUDAPIC_CHECK(check_cuda(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem),
                                 "cudaFuncSetAttribute(step_electrons_inplace)"));
        return check_cuda(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, IP_THREADS, smem),
                          "occupancy(step_electrons_inplace)");
    };
    CUDAPIC_CHECK(occupancy());
    // large grids: fewer copies rather than fewer CTAs; below 4 copies the
    // drains would come every few rounds, so the f32 histogram takes over
    while (per_sm < t.inplace_ctas_per_sm && copies > 0) {
        copies = copies / 2 < 4 ? 0 : copies / 2;
        CUDAPIC_CHECK(occupancy());
    }
    per_sm = std::min(std::max(per_sm, 1), t.inplace_ctas_per_sm);
    const unsigned grid = persistent_grid(per_sm, ((uint64_t)g.capacity + IP_ROUND - 1) / IP_ROUND);
    // rounds per deposit drain: a copy receives ceil(WARPS / copies) warps x 32 lanes x IP_ROW slots per round
    const uint32_t per_round = copies ? (uint32_t)((IP_WARPS + copies - 1) / copies) * 32u * IP_ROW : 1u;
    const uint32_t epoch = copies ? std::max(1u, DEP_MAX_PER_COPY / per_round) : 0xffffffffu;
    return launch_kernel("step_electrons_inplace", kern, dim3(grid), dim3(IP_THREADS),
                         inplace_smem_bytes(copies, ef_pad), stream, pl, efield, sigma_tot_e, cs, sigma_max, n_active, list,
                         count, dens_e, g, ef_pad, copies, epoch, wall, spawn_from,
                         (uint32_t)std::max(t.inplace_prefetch, 0));
}

int launch_electron_scatter(const InplacePlanes &pl, const CollList &list, const float *cs, uint32_t *count,
                            uint32_t *ticket, uint32_t *n_e, uint32_t *n_i, const cudapic_grid &g,
                            cudaStream_t stream, float *dens_e, float *dens_i, unsigned long long *coll,
                            const PoissonAhead *ahead) {
    // every thread loops over records; CTAs per SM from the tuning (the
    // completion ticket counts them)
    const unsigned grid =
        persistent_grid(tuning().scatter_ctas_per_sm, ((uint64_t)g.capacity + IP_THREADS - 1) / IP_THREADS);
    if (!ahead)
        return launch_kernel("scatter_colliders_e", electron_scatter_kernel<0>, dim3(grid), dim3(IP_THREADS), 0,
                             stream, pl, list, cs, count, ticket, n_e, n_i, g, dens_e, dens_i, coll, PoissonAhead{});
    if (g.n_g > POISSON_AHEAD_MAX_NG) return fail(CUDAPIC_ERR_ARG, "scatter_colliders_e: n_g too large for the solve");
    const bool f32 = (g.flags & CUDAPIC_FLAG_POISSON_F32_SCAN) != 0;
    const size_t smem = (size_t)g.n_g * (f32 ? sizeof(float) : sizeof(double));
    const unsigned grid1 = persistent_grid(1, ((uint64_t)g.capacity + SC_SOLVE_THREADS - 1) / SC_SOLVE_THREADS);
    return launch_kernel("scatter_colliders_e+solve_poisson", f32 ? electron_scatter_kernel<2>
                                                                  : electron_scatter_kernel<1>,
                         dim3(grid1), dim3(SC_SOLVE_THREADS), smem, stream, pl, list, cs, count, ticket, n_e, n_i,
                         g, dens_e, dens_i, coll, *ahead);
}

}  // namespace cudapic

using namespace cudapic;

extern "C" int cudapic_step_electrons_inplace(const float *efield, float *x, float *vx, const float *vy,
                                              const float *vz, uint32_t *rng0, uint32_t *rng1, uint32_t *rng2,
                                              uint32_t *rng3, const float *total_cs_e, const float *cs,
                                              float sigma_max_e,
                                              const uint32_t *n_e, uint32_t *const coll[8], uint32_t *n_colliders,
                                              float *e_next_density, const cudapic_grid *grid,
                                              cudapic_stream_t stream) {
    CUDAPIC_CHECK(validate_grid(grid));
    CUDAPIC_REQUIRE(efield && x && vx && vy && vz && rng0 && rng1 && rng2 && rng3 && total_cs_e && cs && n_e && coll &&
                        n_colliders && e_next_density,
                    "step_electrons_inplace: null pointer");
    for (int k = 0; k < 8; ++k) CUDAPIC_REQUIRE(coll[k], "step_electrons_inplace: null record plane");
    CUDAPIC_REQUIRE(sigma_max_e >= 0.0f, "step_electrons_inplace: sigma_max_e must be the largest entry of total_cs_e");
    const void *planes[8] = {x, vx, vy, vz, rng0, rng1, rng2, rng3};
    CUDAPIC_REQUIRE(inplace_eligible(planes, 8, grid->capacity),
                    "step_electrons_inplace: planes must be 16-byte aligned and capacity a multiple of 4");
    const InplacePlanes pl{x, vx, const_cast<float *>(vy), const_cast<float *>(vz), rng0, rng1, rng2, rng3,
                           nullptr, nullptr, nullptr, nullptr};
    const CollList list{coll[0], reinterpret_cast<float *>(coll[1]), reinterpret_cast<float *>(coll[2]),
                        reinterpret_cast<float *>(coll[3]), coll[4], coll[5], coll[6], coll[7]};
    return launch_electron_inplace(pl, efield, total_cs_e, cs, sigma_max_e, n_e, list, n_colliders, e_next_density,
                                   *grid, (cudaStream_t)stream, nullptr, nullptr);
}

extern "C" int cudapic_scatter_colliders_e(float *x, float *vx, float *vy, float *vz, uint32_t *rng0,
                                           uint32_t *rng1, uint32_t *rng2, uint32_t *rng3, const float *cs,
                                           uint32_t *const coll[8], uint32_t *n_colliders, uint32_t *ticket,
                                           float *i_x, float *i_vx, float *i_vy, float *i_vz, uint32_t *n_e,
                                           uint32_t *n_i, float *e_next_density, float *i_next_density,
                                           const cudapic_grid *grid, cudapic_stream_t stream) {
    CUDAPIC_CHECK(validate_grid(grid));
    CUDAPIC_REQUIRE(x && vx && vy && vz && rng0 && rng1 && rng2 && rng3 && cs && coll && n_colliders && ticket &&
                        i_x && i_vx && i_vy && i_vz && n_e && n_i,
                    "scatter_colliders_e: null pointer");
    for (int k = 0; k < 8; ++k) CUDAPIC_REQUIRE(coll[k], "scatter_colliders_e: null record plane");
    const InplacePlanes pl{x, vx, vy, vz, rng0, rng1, rng2, rng3, i_x, i_vx, i_vy, i_vz};
    const CollList list{coll[0], reinterpret_cast<float *>(coll[1]), reinterpret_cast<float *>(coll[2]),
                        reinterpret_cast<float *>(coll[3]), coll[4], coll[5], coll[6], coll[7]};
    return launch_electron_scatter(pl, list, cs, n_colliders, ticket, n_e, n_i, *grid, (cudaStream_t)stream,
                                   e_next_density, i_next_density, nullptr);
}
