// kernels_inplace.cu -- the in-place electron step of one discharge
// (inplace.cuh): one persistent kernel, its launcher (shared with the
// driver) and the C entry point; plus eduPIC's same-step collisions of new
// electrons (an option of the driver).
//
// Reference: the electron half of a time step, move_and_compact
// (Rust-CUDA/src/main.rs:566-678) + check_collisions_e / collision_e
// (:971-1165) + the next step's get_density (:356-406), as the compacting
// fused step (kernels_step.cu) does it, but with every electron kept in its
// slot: no compaction, 56 B of HBM traffic per electron (x, v, RNG read;
// x, vx, RNG written) against 64 B, plus the colliders' scattered
// velocities and RNG states.
#include <algorithm>

#include "batch_internal.h"
#include "inplace.cuh"
#include "internal.h"

namespace cudapic {

template <bool MEAS>
__global__ void __launch_bounds__(IP_THREADS, 4)
    electron_inplace_kernel(const InplacePlanes pl, const float *__restrict__ efield,
                            const float *__restrict__ sigma_tot_e, const float *__restrict__ cs, float sigma_max,
                            uint32_t *n_e, uint32_t *n_i, uint32_t *spawned, uint32_t *ticket, float *dens_e,
                            float *dens_i, const __grid_constant__ cudapic_grid g, uint32_t ef_pad, int copies,
                            uint32_t epoch, cudapic_wall_counters *wall, unsigned long long *coll,
                            uint32_t *spawn_from) {
    extern __shared__ __align__(128) unsigned char smem[];
    const InplaceSmem sm(smem, copies, ef_pad);
    inplace_smem_init(sm, copies, ef_pad);
    grid_dep_wait();
    // read by every CTA before it takes its ticket; the last one publishes the new count
    const uint32_t n = load_count(n_e, g.capacity, g.dev_err);
    if (spawn_from && blockIdx.x == 0 && threadIdx.x == 0) *spawn_from = n;  // first slot of a spawned electron
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
    dc.alive = spawned;
    dc.n_i = n_i;
    dc.dens = dens_e;
    dc.dens_i = dens_i;
    dc.wall = wall;
    dc.coll = coll;
    uint32_t live = 0;
    inplace_segment<false, MEAS>(pl, dc, g, g, 0u, beg, end, n, sm, copies, ef_pad, epoch, live);
    add_work(g.work, live);
    publish_spawns(ticket, n_e, spawned, n, g.capacity, gridDim.x);
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
                            float sigma_max, uint32_t *n_e, uint32_t *n_i, uint32_t *scratch, float *dens_e,
                            float *dens_i, const cudapic_grid &g, cudaStream_t stream, cudapic_wall_counters *wall,
                            unsigned long long *coll, uint32_t *spawn_from) {
    const cudapic_tuning t = tuning();
    const uint32_t ef_pad = (g.n_g + 3u) & ~3u;
    int copies = std::max(1, std::min(t.inplace_copies, IP_WARPS));
    const size_t budget = (size_t)max_smem_optin();
    while (inplace_smem_bytes(copies, ef_pad) > budget && copies > 0) copies = copies / 2 < 4 ? 0 : copies / 2;
    if (inplace_smem_bytes(copies, ef_pad) > budget)
        return fail(CUDAPIC_ERR_ARG, "step_electrons_inplace: n_g too large");
    const bool meas = wall || coll;
    auto kern = meas ? electron_inplace_kernel<true> : electron_inplace_kernel<false>;
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
                         inplace_smem_bytes(copies, ef_pad), stream, pl, efield, sigma_tot_e, cs, sigma_max, n_e, n_i,
                         scratch, scratch + 1, dens_e, dens_i, g, ef_pad, copies, epoch, wall, coll, spawn_from);
}

}  // namespace cudapic

using namespace cudapic;

extern "C" int cudapic_step_electrons_inplace(const float *efield, float *x, float *vx, float *vy, float *vz,
                                              uint32_t *rng0, uint32_t *rng1, uint32_t *rng2, uint32_t *rng3,
                                              const float *total_cs_e, const float *cs, float sigma_max_e, float *i_x,
                                              float *i_vx, float *i_vy, float *i_vz, uint32_t *n_e, uint32_t *n_i,
                                              uint32_t *scratch, float *e_next_density, float *i_next_density,
                                              const cudapic_grid *grid, cudapic_stream_t stream) {
    CUDAPIC_CHECK(validate_grid(grid));
    CUDAPIC_REQUIRE(efield && x && vx && vy && vz && rng0 && rng1 && rng2 && rng3 && total_cs_e && cs && i_x && i_vx &&
                        i_vy && i_vz && n_e && n_i && scratch && e_next_density && i_next_density,
                    "step_electrons_inplace: null pointer");
    CUDAPIC_REQUIRE(sigma_max_e >= 0.0f, "step_electrons_inplace: sigma_max_e must be the largest entry of total_cs_e");
    const void *planes[8] = {x, vx, vy, vz, rng0, rng1, rng2, rng3};
    CUDAPIC_REQUIRE(inplace_eligible(planes, 8, grid->capacity),
                    "step_electrons_inplace: planes must be 16-byte aligned and capacity a multiple of 4");
    const InplacePlanes pl{x, vx, vy, vz, rng0, rng1, rng2, rng3, i_x, i_vx, i_vy, i_vz};
    return launch_electron_inplace(pl, efield, total_cs_e, cs, sigma_max_e, n_e, n_i, scratch, e_next_density,
                                   i_next_density, *grid, (cudaStream_t)stream, nullptr, nullptr, nullptr);
}
