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

#include "common.cuh"
#include "internal.h"
#include "mcc.cuh"
#include "push.cuh"
#include "tma.cuh"

namespace cudapic {

constexpr int ES_THREADS = 256;
constexpr int ES_WARPS = ES_THREADS / 32;
constexpr int ES_PLANES = 8;                  // x, vx, vy, vz, rng0..3
constexpr int ES_MAX_STAGES = 6;              // pipeline depth: cudapic_tuning.step_stages
// U (cudapic_tuning.step_rows, 2 or 4): particles per thread and tile, so a
// tile holds 256 U particles (8 KB U of staged planes); a warp's collider
// queue holds 31 + 32 U entries at most.
template <int U>
struct StepShape {
    static constexpr int TILE = ES_THREADS * U;
    static constexpr int QCAP = 32 + 32 * U;
    static_assert(U * ES_WARPS <= 32, "one warp scans the (row, warp) counts");
};

// Survivors of one tile held in registers until their base is known.
template <int U>
struct StepOut {
    float x[U], vx[U], vy[U], vz[U];
    uint32_t lane_off[U];
    uint32_t keep;  // bit u: the particle of row u is written by the tile
};

// True unless u certainly exceeds the collision probability at speed
// `velocity` (see the file comment; same operation order as test_electron).
__device__ __forceinline__ bool may_collide(float u, float velocity, float sigma_max, float dt) {
    return u < sigma_max * velocity * dt + 5e-7f;
}

template <int U>
__global__ void __launch_bounds__(ES_THREADS)
    electron_step_kernel(const float *__restrict__ efield, const float *__restrict__ sx,
                         const float *__restrict__ svx, const float *__restrict__ svy,
                         const float *__restrict__ svz, float *dx_, float *dvx, float *dvy, float *dvz,
                         uint32_t *rng0, uint32_t *rng1, uint32_t *rng2, uint32_t *rng3,
                         const float *__restrict__ sigma_tot_e, const float *__restrict__ cs, float sigma_max,
                         float *ix, float *ivx, float *ivy, float *ivz, uint32_t *alive,
                         const uint32_t *__restrict__ n_active, uint32_t *n_i, float *dens_e, float *dens_i,
                         const __grid_constant__ cudapic_grid g, uint32_t ef_pad, int stages, int copies,
                         uint32_t epoch, const StepLink link, cudapic_wall_counters *wall,
                         unsigned long long *coll) {
    constexpr int ES_TILE = StepShape<U>::TILE;
    constexpr int ES_QCAP = StepShape<U>::QCAP;
    constexpr int NSEG = U * ES_WARPS;  // (row, warp) segments of a tile
    extern __shared__ __align__(128) unsigned char smem[];
    uint32_t *in = reinterpret_cast<uint32_t *>(smem);                                   // [stages][8][TILE]
    float *ef = reinterpret_cast<float *>(in + stages * ES_PLANES * ES_TILE);             // [ef_pad]
    unsigned long long *acc = reinterpret_cast<unsigned long long *>(ef + ef_pad);        // [ef_pad]
    uint32_t *hist = reinterpret_cast<uint32_t *>(acc + ef_pad);                          // [copies][ef_pad]
    uint32_t *queue = hist + (uint32_t)copies * ef_pad;                                   // [WARPS][QCAP]
    uint64_t *bar = reinterpret_cast<uint64_t *>(queue + ES_WARPS * ES_QCAP);             // [stages]
    // Per tile: (row, warp) counts, then exclusive offsets; the tile's base.
    // Three buffers, because a tile's counts are written while slower warps
    // may still be storing the tile before the previous one.
    __shared__ uint32_t offs[3][NSEG];
    __shared__ uint32_t s_base[3];

    const int tid = threadIdx.x;
    const int lane = tid & 31;
    const int warp = tid >> 5;
    const unsigned lt = lanemask_lt();
    if (tid == 0) {
        for (int s = 0; s < stages; ++s) mbar_init(&bar[s], 1);
        fence_mbar_init();
    }
    for (uint32_t k = tid; k < (uint32_t)copies * ef_pad; k += ES_THREADS) hist[k] = 0u;
    for (uint32_t k = tid; k < ef_pad; k += ES_THREADS) acc[k] = 0ull;
    grid_dep_wait();
    const uint32_t n = load_count(n_active, g.capacity, g.dev_err);
    // Balanced partition: CTA c owns the particles [beg, end), an equal share
    // (a multiple of 4, so every tile start stays 16-byte aligned) cut into
    // tiles; every CTA then finishes after the same work, whatever n is.
    const uint32_t chunk = ((n + gridDim.x - 1) / gridDim.x + 3u) & ~3u;
    const uint32_t beg = min(n, blockIdx.x * chunk);
    const uint32_t end = min(n, beg + chunk);
    const uint32_t ntiles = (end - beg + ES_TILE - 1) / ES_TILE;  // this CTA's tiles
    const uint32_t *src[ES_PLANES] = {reinterpret_cast<const uint32_t *>(sx), reinterpret_cast<const uint32_t *>(svx),
                                      reinterpret_cast<const uint32_t *>(svy), reinterpret_cast<const uint32_t *>(svz),
                                      rng0, rng1, rng2, rng3};
    if (g.work && blockIdx.x == 0 && tid == 0) atomicAdd(g.work, (unsigned long long)n);

    auto issue = [&](uint32_t tile, int stage) {  // tile: index within this CTA's share
        const uint32_t t0 = beg + tile * ES_TILE;
        const uint32_t cnt = min((uint32_t)ES_TILE, end - t0);
        const uint32_t bytes = ((cnt + 3u) & ~3u) * 4u;  // beg is a multiple of 4; so is the capacity
        mbar_arrive_expect_tx(&bar[stage], ES_PLANES * bytes);
#pragma unroll
        for (int a = 0; a < ES_PLANES; ++a)
            bulk_load(in + (stage * ES_PLANES + a) * ES_TILE, src[a] + t0, bytes, &bar[stage]);
    };

    for (uint32_t k = tid; k < g.n_g; k += ES_THREADS) ef[k] = efield[k];
    uint32_t *h = hist + (uint32_t)(warp % copies) * ef_pad;
    uint32_t *wq = queue + warp * ES_QCAP;
    __syncthreads();
    if (tid == 0) {
        for (int s = 0; s < stages; ++s)
            if ((uint32_t)s < ntiles) issue((uint32_t)s, s);
    }

    // Scatters wq[first, first + count), one collider per lane.
    auto drain = [&](uint32_t first, uint32_t count) {
        if (coll && lane == 0) atomicAdd(coll, (unsigned long long)count);  // collision events (measurement)
        if ((uint32_t)lane < count) {
            const uint32_t i = wq[first + lane];
            const PushResult pr = push_one(sx[i], svx[i], ef, g.factor_e, g.dt_e, g);
            const float vy = svy[i], vz = svz[i];
            Xoshiro128p rs{rng0[i], rng1[i], rng2[i], rng3[i]};
            const Test t = test_electron(pr.vx, vy, vz, rs, GlobalTable{sigma_tot_e}, g);  // collides, as before
            uint32_t slot;
            if (claim_slot(alive, g.capacity, slot)) {
                dx_[slot] = pr.x;
                collide_electron(slot, t.idx, pr.vx, vy, vz, rs, cs, dx_, dvx, dvy, dvz, ix, ivx, ivy, ivz, alive,
                                 n_i, g, dens_e, dens_i);
            } else {
                set_dev_err(g.dev_err, CUDAPIC_DEVERR_SPAWN_E);
            }
            rng0[i] = rs.s0;
            rng1[i] = rs.s1;
            rng2[i] = rs.s2;
            rng3[i] = rs.s3;
        }
        __syncwarp();
    };

    StepOut<U> prev;
    bool have_prev = false;
    uint32_t pending_base = 0;  // warp 0 lane 31: atomicAdd result of the previous tile
    uint32_t qn = 0;            // this warp's queued colliders (warp-uniform)
    uint32_t it = 0;
    for (uint32_t tile = 0; tile < ntiles; ++tile, ++it) {
        if (it != 0 && it % epoch == 0) {  // drain the deposit copies before they can overflow
            __syncthreads();
            dep_drain(hist, copies, ef_pad, acc, g.n_g);
            __syncthreads();
        }
        const int s = (int)(it % (uint32_t)stages);
        const uint32_t parity = (it / (uint32_t)stages) & 1u;
        const uint32_t r3 = it % 3u, p3 = (it + 2u) % 3u;  // buffers of this tile and of the previous one
        // every thread waits for the stage's bulk copies itself (bounded)
        const bool ok = mbar_wait_bounded(&bar[s], parity);
        if (!ok) set_dev_err(g.dev_err, CUDAPIC_DEVERR_TIMEOUT);

        const uint32_t t0 = beg + tile * ES_TILE;
        const uint32_t cnt = ok ? min((uint32_t)ES_TILE, end - t0) : 0u;
        const uint32_t *b = in + s * ES_PLANES * ES_TILE;
        // The rows of a tile are independent; the work is split into phases
        // over all rows so that the scheduler can interleave them.
        StepOut<U> cur;
        cur.keep = 0;
        uint32_t st[U][4];     // RNG states after the test draw
        uint32_t keep = 0, may = 0, coll = 0;  // bit u: row u survives / may collide / collides
        // (1) push (Rust-CUDA/src/main.rs:596-620); rows past the tile's end
        //     push a harmless stand-in and are masked
#pragma unroll
        for (int u = 0; u < U; ++u) {
            const uint32_t j = (uint32_t)u * ES_THREADS + tid;
            const bool valid = j < cnt;
            const float x0 = valid ? __uint_as_float(b[j]) : 0.5f * g.gap;
            const float v0 = valid ? __uint_as_float(b[ES_TILE + j]) : 0.0f;
            const PushResult pr = push_one(x0, v0, ef, g.factor_e, g.dt_e, g);
            if (valid && pr.keep) keep |= 1u << u;
            if (wall) count_wall(wall, false, valid && !pr.keep, pr.x, 0.0f, 0.0f, 0.0f, g.gap);
            cur.x[u] = pr.x;
            cur.vx[u] = pr.vx;
        }
        // (2) test_electron (mcc.cuh, Rust-CUDA/src/main.rs:992-1012) up to the
        //     certain rejection, which needs no table
#pragma unroll
        for (int u = 0; u < U; ++u) {
            const uint32_t j = (uint32_t)u * ES_THREADS + tid;
            cur.vy[u] = __uint_as_float(b[2 * ES_TILE + j]);
            cur.vz[u] = __uint_as_float(b[3 * ES_TILE + j]);
            Xoshiro128p rs{b[4 * ES_TILE + j], b[5 * ES_TILE + j], b[6 * ES_TILE + j], b[7 * ES_TILE + j]};
            const float v2 = cur.vx[u] * cur.vx[u] + cur.vy[u] * cur.vy[u] + cur.vz[u] * cur.vz[u];
            const float velocity = sqrtf(v2);
            const float rnd = rs.uniform();
            if ((keep >> u & 1u) && may_collide(rnd, velocity, sigma_max, g.dt_e)) may |= 1u << u;
            st[u][0] = rs.s0;
            st[u][1] = rs.s1;
            st[u][2] = rs.s2;
            st[u][3] = rs.s3;
        }
        // (3) the exact test where the bound cannot decide (a few per cent)
        if (may) {
#pragma unroll
            for (int u = 0; u < U; ++u) {
                if (may >> u & 1u) {
                    const uint32_t j = (uint32_t)u * ES_THREADS + tid;
                    Xoshiro128p rs{b[4 * ES_TILE + j], b[5 * ES_TILE + j], b[6 * ES_TILE + j], b[7 * ES_TILE + j]};
                    const float v2 = cur.vx[u] * cur.vx[u] + cur.vy[u] * cur.vy[u] + cur.vz[u] * cur.vz[u];
                    const float velocity = sqrtf(v2);
                    const float rnd = rs.uniform();
                    const uint32_t idx = energy_index(g.half_me_over_e * v2);
                    if (collision_draw(rnd, __ldg(sigma_tot_e + idx) * velocity * g.dt_e)) coll |= 1u << u;
                }
            }
        }
        // (4) deposit every survivor; non-colliders store their RNG state and
        //     are compacted, colliders are queued
#pragma unroll
        for (int u = 0; u < U; ++u) {
            const uint32_t j = (uint32_t)u * ES_THREADS + tid;
            const bool kept = keep >> u & 1u;
            const bool collide = coll >> u & 1u;
            const bool stay = kept && !collide;
            if (kept) dep_add(h, cur.x[u], g);  // CIC of the new position, Rust-CUDA/src/main.rs:377-387
            if (stay) {
                const uint32_t i = t0 + j;
                rng0[i] = st[u][0];
                rng1[i] = st[u][1];
                rng2[i] = st[u][2];
                rng3[i] = st[u][3];
            }
            const unsigned m = __ballot_sync(0xffffffffu, stay);
            cur.lane_off[u] = __popc(m & lt);
            if (stay) cur.keep |= 1u << u;
            if (lane == 0) offs[r3][u * ES_WARPS + warp] = __popc(m);
            const unsigned cm = __ballot_sync(0xffffffffu, collide);
            if (collide) wq[qn + __popc(cm & lt)] = t0 + j;
            qn += __popc(cm);
        }
        // publish the previous tile's base (its atomic had this iteration to return)
        if (have_prev && warp == 0 && lane == 31) s_base[p3] = pending_base;
        // the one block barrier of a tile: counts and previous base visible,
        // stage s consumed; a timeout anywhere ends the loop of every thread
        if (__syncthreads_or(!ok)) break;
        if (tid == 0) {
            const uint32_t next = tile + (uint32_t)stages;
            if (next < ntiles) issue(next, s);
        }
        if (have_prev) {
            const uint32_t base = s_base[p3];
#pragma unroll
            for (int u = 0; u < U; ++u) {
                if (prev.keep & (1u << u)) {
                    const uint32_t slot = base + offs[p3][u * ES_WARPS + warp] + prev.lane_off[u];
                    if (slot < g.capacity) {
                        dx_[slot] = prev.x[u];
                        dvx[slot] = prev.vx[u];
                        dvy[slot] = prev.vy[u];
                        dvz[slot] = prev.vz[u];
                    } else {
                        set_dev_err(g.dev_err, CUDAPIC_DEVERR_SPAWN_E);
                    }
                }
            }
        }
        if (warp == 0) {
            const uint32_t v = lane < NSEG ? offs[r3][lane] : 0u;
            uint32_t incl = v;
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
                const uint32_t t = __shfl_up_sync(0xffffffffu, incl, o);
                if (lane >= o) incl += t;
            }
            if (lane < NSEG) offs[r3][lane] = incl - v;
            if (lane == 31) pending_base = incl ? atomicAdd(alive, incl) : 0u;
        }
        prev = cur;
        have_prev = true;
        while (qn >= 32) {  // full-warp drains from the top of the queue
            qn -= 32;
            drain(qn, 32);
        }
    }
    const uint32_t pl = (it + 2u) % 3u;  // buffers of the last tile with survivors held in registers
    if (have_prev && warp == 0 && lane == 31) s_base[pl] = pending_base;
    __syncthreads();
    if (have_prev) {
        const uint32_t base = s_base[pl];
#pragma unroll
        for (int u = 0; u < U; ++u) {
            if (prev.keep & (1u << u)) {
                const uint32_t slot = base + offs[pl][u * ES_WARPS + warp] + prev.lane_off[u];
                if (slot < g.capacity) {
                    dx_[slot] = prev.x[u];
                    dvx[slot] = prev.vx[u];
                    dvy[slot] = prev.vy[u];
                    dvz[slot] = prev.vz[u];
                } else {
                    set_dev_err(g.dev_err, CUDAPIC_DEVERR_SPAWN_E);
                }
            }
        }
    }
    if (qn) drain(0, qn);
    __syncthreads();
    dep_drain(hist, copies, ef_pad, acc, g.n_g);
    __syncthreads();
    dep_flush(acc, dens_e, g);
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
    constexpr int ES_TILE = StepShape<U>::TILE;
    constexpr int ES_QCAP = StepShape<U>::QCAP;
    int stages = std::min(std::max(t.step_stages, 2), ES_MAX_STAGES);
    int copies = std::max(1, std::min(t.density_copies, ES_WARPS));
    const uint32_t ef_pad = (g.n_g + 3u) & ~3u;
    auto bytes = [&]() {
        return (size_t)stages * ES_PLANES * ES_TILE * 4 + (size_t)ef_pad * (4 + 8) + (size_t)copies * ef_pad * 4 +
               (size_t)ES_WARPS * ES_QCAP * 4 + (size_t)stages * sizeof(uint64_t);
    };
    const size_t budget = (size_t)max_smem_optin();
    while (bytes() > budget && stages > 2) --stages;
    while (bytes() > budget && copies > 1) copies = (copies + 1) / 2;
    if (bytes() > budget) return fail(CUDAPIC_ERR_ARG, "step_electrons: n_g too large");
    const size_t smem = bytes();
    auto kern = electron_step_kernel<U>;
    CUDAPIC_CHECK(check_cuda(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem),
                             "cudaFuncSetAttribute(step_electrons)"));
    int per_sm = 0;
    CUDAPIC_CHECK(check_cuda(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, ES_THREADS, smem),
                             "occupancy(step_electrons)"));
    per_sm = std::min(std::max(per_sm, 1), t.step_ctas_per_sm);
    const uint64_t tiles_max = ((uint64_t)g.capacity + ES_TILE - 1) / ES_TILE;
    const unsigned grid = persistent_grid(per_sm, tiles_max);
    // tiles per deposit drain: a copy receives ceil(WARPS / copies) warps x 128 particles per tile
    const uint32_t per_tile = (uint32_t)((ES_WARPS + copies - 1) / copies) * U * 32u;
    const uint32_t epoch = std::max(1u, DEP_MAX_PER_COPY / per_tile);
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
    auto launch = t.step_rows == 4 ? launch_electron_step_t<4> : launch_electron_step_t<2>;
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
