// kernels_step.cu -- the fused electron step of the driver.
//
// One persistent kernel does, per electron, the work of the reference's
// move_and_compact (Rust-CUDA/src/main.rs:566-678), check_collisions_e /
// collision_e (:971-1165) and the next step's get_density (:356-406):
//   push + absorption -> collision test -> scattering / ionization ->
//   compaction into the other side -> CIC deposit of the new position.
// Two differences from running those kernels in sequence (statistically
// equivalent; the drop-in entry points keep the reference's semantics):
//  * a particle draws from the RNG stream of its SOURCE slot (the slot it
//    occupies when the step starts), not of the slot it is compacted into.
//    Every slot still owns one xoshiro128+ stream, used at most once per
//    step, in the same four SoA planes;
//  * survivors, colliders and spawned electrons share one slot counter, so
//    spawned electrons are interleaved with the survivors.
//
// B200 design (HBM-bound: 16 B of particle and 16 B of RNG state read, the
// same written per survivor -- 64 B against 76 B for push + collisions):
//  * persistent grid, 256 threads, tiles of 512 or 1024 particles; the eight
//    SoA planes of a tile (x, vx, vy, vz, rng0..3: 16 or 32 KB) are staged by
//    cp.async.bulk on an mbarrier pipeline;
//  * certain rejection without the cross-section table: the exact test
//    (mcc.cuh) decides "no collision" whenever u >= fl(a + 5e-7) with
//    a = fl(fl(sigma(E) |v|) dt).  Rounding is monotone, so with sigma_max
//    the largest table entry, u >= fl(fl(fl(sigma_max |v|) dt) + 5e-7)
//    implies it: the energy index and the table gather are skipped for
//    almost every electron, the decision is bit-identical;
//  * every thread waits on the stage's mbarrier itself, so a tile has one
//    block barrier (after the counts), not a barrier for the data as well;
//  * non-colliding survivors store their advanced RNG state in place
//    (coalesced) and are compacted as in move_and_compact: warp ballots, one
//    warp scan per tile, one atomicAdd per tile whose result is consumed a
//    tile later;
//  * colliders are queued per warp by source slot.  A warp with 32 queued
//    re-reads them from the source planes (not written by this kernel),
//    repeats the deterministic push and test and scatters one per lane, so
//    the long scattering path runs on full warps;
//  * every survivor is deposited into the next-step density through 2^-20
//    fixed-point warp-private shared histograms (push.cuh); spawned
//    electrons and ions add to the densities with global atomics;
//  * the last CTA to finish publishes the electron count (StepLink).
#include <algorithm>

#include "internal.h"
#include "step.cuh"

namespace cudapic {

template <int U>
__global__ void __launch_bounds__(ES_THREADS)
    electron_step_kernel(const float *__restrict__ efield, const float *__restrict__ sx,
                         const float *__restrict__ svx, const float *__restrict__ svy,
                         const float *__restrict__ svz, float *dx_, float *dvx, float *dvy, float *dvz,
                         uint32_t *rng0, uint32_t *rng1, uint32_t *rng2, uint32_t *rng3,
                         const float *__restrict__ sigma_tot_e, const float *__restrict__ cs, float sigma_max,
                         float *ix, float *ivx, float *ivy, float *ivz, uint32_t *alive,
                         const uint32_t *n_active, uint32_t *n_i, float *dens_e, float *dens_i,
                         const __grid_constant__ cudapic_grid g, uint32_t ef_pad, int stages, int copies,
                         uint32_t epoch, const StepLink link, cudapic_wall_counters *wall,
                         unsigned long long *coll) {
    extern __shared__ __align__(128) unsigned char smem[];
    // Per tile: (row, warp) counts, then exclusive offsets; the tile's base.
    // Three buffers, because a tile's counts are written while slower warps
    // may still be storing the tile before the previous one.
    __shared__ uint32_t offs[3][StepShape<U, true>::NSEG];
    __shared__ uint32_t s_base[3];
    __shared__ uint32_t ccnt[3][StepShape<U, true>::NSEG];
    const StepSmem<U, true> sm(smem, stages, copies, ef_pad, offs, s_base, ccnt);
    step_smem_init(sm, stages, copies, ef_pad);
    grid_dep_wait();
    // n_active may be link.dst (the no-alloc entry publishes the new count in
    // place): it is read here, before this CTA takes its ticket, and never again
    const uint32_t n = load_count(n_active, g.capacity, g.dev_err);
    // Balanced partition: CTA c owns the particles [beg, end), an equal share
    // (a multiple of 4, so every tile start stays 16-byte aligned) cut into
    // tiles; every CTA then finishes after the same work, whatever n is.
    const uint32_t chunk = ((n + gridDim.x - 1) / gridDim.x + 3u) & ~3u;
    const uint32_t beg = min(n, blockIdx.x * chunk);
    const uint32_t end = min(n, beg + chunk);
    StepPlanes pl;
    pl.sx = sx;
    pl.svx = svx;
    pl.svy = svy;
    pl.svz = svz;
    pl.dx = dx_;
    pl.dvx = dvx;
    pl.dvy = dvy;
    pl.dvz = dvz;
    pl.rng0 = rng0;
    pl.rng1 = rng1;
    pl.rng2 = rng2;
    pl.rng3 = rng3;
    pl.ix = ix;
    pl.ivx = ivx;
    pl.ivy = ivy;
    pl.ivz = ivz;
    StepDisc dc;
    dc.efield = efield;
    dc.sigma_tot = sigma_tot_e;
    dc.cs = cs;
    dc.sigma_max = sigma_max;
    dc.factor = g.factor_e;
    dc.dt = g.dt_e;
    dc.alive = alive;
    dc.n_i = n_i;
    dc.dens = dens_e;
    dc.dens_i = dens_i;
    dc.wall = wall;
    dc.coll = coll;
    uint32_t it = 0, live = 0;
    step_segment<U, true, false, true>(pl, dc, g, g, 0u, beg, end, sm, stages, copies, ef_pad, epoch, it, live);
    add_work(g.work, live);
    publish_count(link.ticket, link.dst, link.src, link.clear_src, g.capacity);
}

bool electron_step_eligible(const void *const *planes, int count, uint32_t capacity) {
    if (capacity % 4u) return false;
    for (int k = 0; k < count; ++k)
        if (!aligned16(planes[k])) return false;
    return true;
}

namespace {

template <int U>
int launch_electron_step_t(const float *efield, const float *sx, const float *svx, const float *svy,
                           const float *svz, float *dx_, float *dvx, float *dvy, float *dvz, uint32_t *rng0,
                           uint32_t *rng1, uint32_t *rng2, uint32_t *rng3, const float *sigma_tot_e, const float *cs,
                           float sigma_max_e, float *ix, float *ivx, float *ivy, float *ivz, uint32_t *alive,
                           const uint32_t *n_active, uint32_t *n_i, float *dens_e, float *dens_i,
                           const cudapic_grid &g, cudaStream_t stream, const StepLink &link,
                           cudapic_wall_counters *wall, unsigned long long *coll, const cudapic_tuning &t) {
    constexpr int ES_TILE = StepShape<U, true>::TILE;
    int stages = std::min(std::max(t.step_stages, 2), ES_MAX_STAGES);
    int copies = std::max(1, std::min(t.density_copies, ES_WARPS));
    const uint32_t ef_pad = (g.n_g + 3u) & ~3u;
    auto bytes = [&]() { return step_smem_bytes<U, true>(stages, copies, ef_pad); };
    const size_t budget = (size_t)max_smem_optin();
    while (bytes() > budget && stages > 2) --stages;
    // below 4 copies the f32 histogram (copies = 0) takes over: 8 B per node
    auto fewer = [&]() { copies = copies / 2 < 4 ? 0 : copies / 2; };
    while (bytes() > budget && copies > 0) fewer();
    if (bytes() > budget) return fail(CUDAPIC_ERR_ARG, "step_electrons: n_g too large");
    auto kern = electron_step_kernel<U>;
    int per_sm = 0;
    auto occupancy = [&]() {
        CUDAPIC_CHECK(check_cuda(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes()),
                                 "cudaFuncSetAttribute(step_electrons)"));
        return check_cuda(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, ES_THREADS, bytes()),
                          "occupancy(step_electrons)");
    };
    CUDAPIC_CHECK(occupancy());
    // large grids: fewer histogram copies rather than fewer CTAs per SM (the
    // copies only spread atomic conflicts, which a large grid spreads by itself)
    while (per_sm < t.step_ctas_per_sm && copies > 0) {
        fewer();
        CUDAPIC_CHECK(occupancy());
    }
    const size_t smem = bytes();
    per_sm = std::min(std::max(per_sm, 1), t.step_ctas_per_sm);
    const uint64_t tiles_max = ((uint64_t)g.capacity + ES_TILE - 1) / ES_TILE;
    const unsigned grid = persistent_grid(per_sm, tiles_max);
    // tiles per deposit drain: a copy receives ceil(WARPS / copies) warps x 128 particles per tile
    const uint32_t per_tile = copies ? (uint32_t)((ES_WARPS + copies - 1) / copies) * U * 32u : 1u;
    const uint32_t epoch = copies ? std::max(1u, DEP_MAX_PER_COPY / per_tile) : 0xffffffffu;
    return launch_kernel("step_electrons", kern, dim3(grid), dim3(ES_THREADS), smem, stream, efield, sx, svx, svy, svz,
                         dx_, dvx, dvy, dvz, rng0, rng1, rng2, rng3, sigma_tot_e, cs, sigma_max_e, ix, ivx, ivy, ivz,
                         alive, n_active, n_i, dens_e, dens_i, g, ef_pad, stages, copies, epoch, link, wall, coll);
}

}  // namespace

int launch_electron_step(const float *efield, const float *sx, const float *svx, const float *svy, const float *svz,
                         float *dx_, float *dvx, float *dvy, float *dvz, uint32_t *rng0, uint32_t *rng1,
                         uint32_t *rng2, uint32_t *rng3, const float *sigma_tot_e, const float *cs, float sigma_max_e,
                         float *ix, float *ivx, float *ivy, float *ivz, uint32_t *alive, const uint32_t *n_active,
                         uint32_t *n_i, float *dens_e, float *dens_i, const cudapic_grid &g, cudaStream_t stream,
                         const StepLink &link, cudapic_wall_counters *wall, unsigned long long *coll) {
    const void *planes[8] = {sx, svx, svy, svz, rng0, rng1, rng2, rng3};
    if (!electron_step_eligible(planes, 8, g.capacity)) return CUDAPIC_ERR_NOT_SUPPORTED;
    const cudapic_tuning t = tuning();
    auto launch = t.step_rows == 4   ? launch_electron_step_t<4>
                  : t.step_rows == 1 ? launch_electron_step_t<1>
                                     : launch_electron_step_t<2>;
    return launch(efield, sx, svx, svy, svz, dx_, dvx, dvy, dvz, rng0, rng1, rng2, rng3, sigma_tot_e, cs, sigma_max_e,
                  ix, ivx, ivy, ivz, alive, n_active, n_i, dens_e, dens_i, g, stream, link, wall, coll, t);
}

}  // namespace cudapic

using namespace cudapic;

extern "C" int cudapic_step_electrons(const float *efield, const float *src_x, const float *src_vx,
                                      const float *src_vy, const float *src_vz, float *dst_x, float *dst_vx,
                                      float *dst_vy, float *dst_vz, uint32_t *rng0, uint32_t *rng1, uint32_t *rng2,
                                      uint32_t *rng3, const float *total_cs_e, const float *cs, float sigma_max_e,
                                      float *i_x, float *i_vx, float *i_vy, float *i_vz, uint32_t *alive_counter,
                                      const uint32_t *n_e, uint32_t *n_i, float *e_next_density,
                                      float *i_next_density, const cudapic_grid *grid, cudapic_stream_t stream) {
    CUDAPIC_CHECK(validate_grid(grid));
    CUDAPIC_REQUIRE(efield && src_x && src_vx && src_vy && src_vz && dst_x && dst_vx && dst_vy && dst_vz && rng0 &&
                        rng1 && rng2 && rng3 && total_cs_e && cs && i_x && i_vx && i_vy && i_vz && alive_counter &&
                        n_e && n_i && e_next_density && i_next_density,
                    "step_electrons: null pointer");
    CUDAPIC_REQUIRE(sigma_max_e >= 0.0f, "step_electrons: sigma_max_e must be the largest entry of total_cs_e");
    const int rc = launch_electron_step(efield, src_x, src_vx, src_vy, src_vz, dst_x, dst_vx, dst_vy, dst_vz, rng0,
                                        rng1, rng2, rng3, total_cs_e, cs, sigma_max_e, i_x, i_vx, i_vy, i_vz,
                                        alive_counter, n_e, n_i, e_next_density, i_next_density, *grid,
                                        (cudaStream_t)stream, StepLink());
    if (rc == CUDAPIC_ERR_NOT_SUPPORTED)
        return fail(CUDAPIC_ERR_ARG, "step_electrons: planes must be 16-byte aligned and capacity a multiple of 4");
    return rc;
}
