// kernels_push.cu -- leapfrog push + electrode absorption + stream compaction.
//
// Reference: move_and_compact, Rust-CUDA/src/main.rs:566-678.  Per particle:
//   e_x = (1-c2) E[p] + c2 E[p+1]   (CIC gather, p = int(x/dx), c2 = frac)
//   v'  = v + factor e_x,  x' = x + v' dt,  kept iff 0 <= x' <= L,
// survivors appended to dst at a block base from one atomicAdd on
// alive_counter; order across blocks is unspecified (as in the reference).
//
// B200 design (HBM-bound: 16 B read per particle, 16 B written per survivor):
//  * persistent grid, 256 threads, tiles of 1024 particles;
//  * the four SoA input tiles (x, vx, vy, vz: 4 x 4 KB) are staged into
//    shared memory by cp.async.bulk (TMA bulk copies) completing on an
//    mbarrier, four stages deep, so three tiles stream in while one computes;
//  * E[N_G] is held in shared memory for the gathers;
//  * thread t owns particles t, t+256, t+512, t+768 of a tile (conflict-free
//    shared loads); a warp ballot per row gives each surviving lane its rank,
//    one warp scans the 4 x 8 (row, warp) counts, so a (row, warp)'s survivors
//    are written to consecutive slots: coalesced stores straight from
//    registers, no output staging;
//  * two block barriers per tile; the tile's atomicAdd on alive_counter is
//    issued at the end of one iteration and its result consumed in the next,
//    after the next tile's wait and compute, so its latency is hidden.
// Within a tile, survivors keep their order.
// A one-particle-per-thread variant (ballot/popc, the reference's layout)
// serves pointers that are not 16-byte aligned or capacities that are not
// a multiple of 4.
#include "common.cuh"
#include "internal.h"
#include "push.cuh"
#include "tma.cuh"

namespace cudapic {

constexpr int MC_THREADS = 256;
constexpr int MC_WARPS = MC_THREADS / 32;
constexpr int MC_U = 4;                          // particles per thread and tile
constexpr int MC_TILE = MC_THREADS * MC_U;       // 1024
constexpr int MC_MAX_STAGES = 6;                 // pipeline depth: cudapic_tuning.push_stages

// Survivors of one tile held in registers until their base is known.
struct TileOut {
    float x[MC_U], vx[MC_U], vy[MC_U], vz[MC_U];
    uint32_t lane_off[MC_U];
    uint32_t keep;  // bit u: particle of row u survives
};

// DEPOSIT: also deposit every survivor's new position into dens_out (the
// charge density of the next time step), through `copies` warp-private
// fixed-point shared histograms (see dep_add) drained every `epoch` tiles,
// or with copies == 0 (large grids) one f32 histogram (dep_add_f32).
template <bool DEPOSIT>
__global__ void __launch_bounds__(MC_THREADS)
    move_and_compact_tma_kernel(const float *__restrict__ efield, const float *__restrict__ sx,
                                const float *__restrict__ svx, const float *__restrict__ svy,
                                const float *__restrict__ svz, float *__restrict__ dx_,
                                float *__restrict__ dvx, float *__restrict__ dvy, float *__restrict__ dvz,
                                uint32_t *__restrict__ alive, const uint32_t *__restrict__ n_active,
                                float factor, float dt, const cudapic_grid g, uint32_t ef_pad, int stages,
                                float *__restrict__ dens_out, int copies, uint32_t epoch, const StepLink link,
                                cudapic_wall_counters *wall, int wall_ions) {
    extern __shared__ __align__(128) unsigned char smem[];
    float *in = reinterpret_cast<float *>(smem);        // [stages][4][TILE]
    float *ef = in + stages * 4 * MC_TILE;               // [ef_pad]
    unsigned long long *acc = reinterpret_cast<unsigned long long *>(ef + ef_pad);  // [ef_pad] (DEPOSIT)
    float *hf = reinterpret_cast<float *>(acc);  // copies == 0: the f32 histogram [ef_pad] in its place
    uint32_t *hist = !DEPOSIT ? reinterpret_cast<uint32_t *>(acc)
                     : copies ? reinterpret_cast<uint32_t *>(acc + ef_pad)
                              : reinterpret_cast<uint32_t *>(ef + 2u * ef_pad);  // [copies][ef_pad]
    uint64_t *bar = reinterpret_cast<uint64_t *>(hist + (DEPOSIT ? copies * ef_pad : 0));
    __shared__ uint32_t offs[2][MC_U * MC_WARPS];        // counts, then exclusive offsets
    __shared__ uint32_t s_base[2];
    __shared__ int s_ready;

    const int tid = threadIdx.x;
    const int lane = tid & 31;
    const int warp = tid >> 5;
    const unsigned lt = lanemask_lt();
    if (tid == 0) {
        for (int s = 0; s < stages; ++s) mbar_init(&bar[s], 1);
        fence_mbar_init();
    }
    if (DEPOSIT) {
        for (uint32_t k = tid; k < (uint32_t)copies * ef_pad; k += MC_THREADS) hist[k] = 0u;
        if (copies)
            for (uint32_t k = tid; k < ef_pad; k += MC_THREADS) acc[k] = 0ull;
        else
            for (uint32_t k = tid; k < ef_pad; k += MC_THREADS) hf[k] = 0.0f;
    }
    grid_dep_wait();
    const uint32_t n = load_count(n_active, g.capacity, g.dev_err);
    const uint32_t ntiles = (n + MC_TILE - 1) / MC_TILE;
    const float *src[4] = {sx, svx, svy, svz};
    if (g.work && blockIdx.x == 0 && tid == 0) atomicAdd(g.work, (unsigned long long)n);

    auto issue = [&](uint32_t tile, int stage) {
        const uint32_t t0 = tile * MC_TILE;
        const uint32_t cnt = min((uint32_t)MC_TILE, n - t0);
        const uint32_t bytes = ((cnt + 3u) & ~3u) * 4u;   // capacity is a multiple of 4
        mbar_arrive_expect_tx(&bar[stage], 4u * bytes);
#pragma unroll
        for (int a = 0; a < 4; ++a) bulk_load(in + (stage * 4 + a) * MC_TILE, src[a] + t0, bytes, &bar[stage]);
    };

    for (uint32_t k = tid; k < g.n_g; k += MC_THREADS) ef[k] = efield[k];
    uint32_t *h = hist + (uint32_t)(warp % max(copies, 1)) * ef_pad;
    __syncthreads();
    if (tid == 0) {
        for (int s = 0; s < stages; ++s) {
            const uint32_t tile = blockIdx.x + (uint32_t)s * gridDim.x;
            if (tile < ntiles) issue(tile, s);
        }
    }

    TileOut prev;
    bool have_prev = false;
    uint32_t pending_base = 0;  // warp 0 lane 31: atomicAdd result of the previous tile
    uint32_t it = 0;
    for (uint32_t tile = blockIdx.x; tile < ntiles; tile += gridDim.x, ++it) {
        if (DEPOSIT && copies && it != 0 && it % epoch == 0) {  // drain the copies before they can overflow
            __syncthreads();
            dep_drain(hist, copies, ef_pad, acc, g.n_g);
            __syncthreads();
        }
        const int s = (int)(it % (uint32_t)stages);
        const uint32_t parity = (it / (uint32_t)stages) & 1u;
        // (1) the stage's bulk copies have landed (one bounded waiter, uniform verdict)
        if (tid == 0) {
            const int ok = mbar_wait_bounded(&bar[s], parity) ? 1 : 0;
            if (!ok) set_dev_err(g.dev_err, CUDAPIC_DEVERR_TIMEOUT);
            s_ready = ok;
        }
        __syncthreads();
        if (!s_ready) break;  // timed out: flagged; the counts are still published

        const uint32_t t0 = tile * MC_TILE;
        const uint32_t cnt = min((uint32_t)MC_TILE, n - t0);
        const float *bx = in + (s * 4 + 0) * MC_TILE;
        const float *bvx = in + (s * 4 + 1) * MC_TILE;
        const float *bvy = in + (s * 4 + 2) * MC_TILE;
        const float *bvz = in + (s * 4 + 3) * MC_TILE;
        TileOut cur;
        cur.keep = 0;
#pragma unroll
        for (int u = 0; u < MC_U; ++u) {
            const uint32_t j = (uint32_t)u * MC_THREADS + tid;
            bool keep = false;
            cur.x[u] = cur.vx[u] = cur.vy[u] = cur.vz[u] = 0.0f;
            if (j < cnt) {
                const PushResult pr = push_one(bx[j], bvx[j], ef, factor, dt, g);
                keep = pr.keep;
                cur.x[u] = pr.x;
                cur.vx[u] = pr.vx;
                cur.vy[u] = bvy[j];
                cur.vz[u] = bvz[j];
            }
            if (DEPOSIT && keep) {  // CIC of the new position, Rust-CUDA/src/main.rs:377-387
                if (copies) dep_add(h, cur.x[u], g);
                else dep_add_f32(hf, cur.x[u], g);
            }
            if (wall) count_wall(wall, wall_ions, j < cnt && !keep, cur.x[u], cur.vx[u], cur.vy[u], cur.vz[u], g.gap);
            const unsigned m = __ballot_sync(0xffffffffu, keep);
            cur.lane_off[u] = __popc(m & lt);
            if (keep) cur.keep |= 1u << u;
            if (lane == 0) offs[it & 1][u * MC_WARPS + warp] = __popc(m);
        }
        // publish the previous tile's base (its atomic had this iteration to return)
        if (have_prev && warp == 0 && lane == 31) s_base[(it - 1) & 1] = pending_base;
        __syncthreads();  // (2) counts and previous base visible; stage s consumed
        if (tid == 0) {
            const uint32_t next = tile + (uint32_t)stages * gridDim.x;
            if (next < ntiles) issue(next, s);
        }
        if (have_prev) {
            const uint32_t base = s_base[(it - 1) & 1];
#pragma unroll
            for (int u = 0; u < MC_U; ++u) {
                if (prev.keep & (1u << u)) {
                    const uint32_t slot = base + offs[(it - 1) & 1][u * MC_WARPS + warp] + prev.lane_off[u];
                    dx_[slot] = prev.x[u];
                    dvx[slot] = prev.vx[u];
                    dvy[slot] = prev.vy[u];
                    dvz[slot] = prev.vz[u];
                }
            }
        }
        if (warp == 0) {
            const uint32_t v = offs[it & 1][lane];   // MC_U * MC_WARPS == 32
            uint32_t incl = v;
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
                const uint32_t t = __shfl_up_sync(0xffffffffu, incl, o);
                if (lane >= o) incl += t;
            }
            offs[it & 1][lane] = incl - v;
            if (lane == 31) pending_base = incl ? atomicAdd(alive, incl) : 0u;
        }
        prev = cur;
        have_prev = true;
    }
    if (have_prev && warp == 0 && lane == 31) s_base[(it - 1) & 1] = pending_base;
    __syncthreads();
    if (have_prev) {
        const uint32_t base = s_base[(it - 1) & 1];
#pragma unroll
        for (int u = 0; u < MC_U; ++u) {
            if (prev.keep & (1u << u)) {
                const uint32_t slot = base + offs[(it - 1) & 1][u * MC_WARPS + warp] + prev.lane_off[u];
                dx_[slot] = prev.x[u];
                dvx[slot] = prev.vx[u];
                dvy[slot] = prev.vy[u];
                dvz[slot] = prev.vz[u];
            }
        }
    }
    if (DEPOSIT) {  // sum the warp copies, one global atomic per four nodes
        __syncthreads();
        if (copies) {
            dep_drain(hist, copies, ef_pad, acc, g.n_g);
            __syncthreads();
            dep_flush(acc, dens_out, g);
        } else {
            dep_flush_f32(hf, dens_out, g);
        }
    }
    publish_count(link.ticket, link.dst, link.src, link.clear_src, g.capacity);
}

// Reference-layout variant: one particle per thread, warp ballot + popc,
// one atomic per block and iteration.  No alignment requirements.
constexpr int MCS_THREADS = 512;
constexpr int MCS_WARPS = MCS_THREADS / 32;

__global__ void __launch_bounds__(MCS_THREADS)
    move_and_compact_simple_kernel(const float *__restrict__ efield, const float *__restrict__ sx,
                                   const float *__restrict__ svx, const float *__restrict__ svy,
                                   const float *__restrict__ svz, float *__restrict__ dx_,
                                   float *__restrict__ dvx, float *__restrict__ dvy, float *__restrict__ dvz,
                                   uint32_t *__restrict__ alive, const uint32_t *__restrict__ n_active,
                                   float factor, float dt, const cudapic_grid g, cudapic_wall_counters *wall,
                                   int wall_ions) {
    extern __shared__ float ef_s[];
    __shared__ uint32_t wsum[MCS_WARPS];
    __shared__ uint32_t s_base;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    grid_dep_wait();
    for (uint32_t k = tid; k < g.n_g; k += MCS_THREADS) ef_s[k] = efield[k];
    __syncthreads();
    const uint32_t n = load_count(n_active, g.capacity, g.dev_err);
    if (g.work && blockIdx.x == 0 && tid == 0) atomicAdd(g.work, (unsigned long long)n);
    const uint32_t rounds = (n + gridDim.x * MCS_THREADS - 1) / (gridDim.x * MCS_THREADS);
    for (uint32_t rd = 0; rd < rounds; ++rd) {
        const uint32_t i = (rd * gridDim.x + blockIdx.x) * MCS_THREADS + tid;
        PushResult pr = {0.0f, 0.0f, false};
        float vy = 0.0f, vz = 0.0f;
        if (i < n) {
            pr = push_one(sx[i], svx[i], ef_s, factor, dt, g);
            if (pr.keep || wall) {
                vy = svy[i];
                vz = svz[i];
            }
        }
        if (wall) count_wall(wall, wall_ions, i < n && !pr.keep, pr.x, pr.vx, vy, vz, g.gap);
        const unsigned mask = __ballot_sync(0xffffffffu, pr.keep);
        const uint32_t lane_off = __popc(mask & lanemask_lt());
        if (lane == 0) wsum[warp] = __popc(mask);
        __syncthreads();
        if (warp == 0) {
            uint32_t v = lane < MCS_WARPS ? wsum[lane] : 0u;
            uint32_t incl = v;
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
                uint32_t t = __shfl_up_sync(0xffffffffu, incl, o);
                if (lane >= o) incl += t;
            }
            if (lane < MCS_WARPS) wsum[lane] = incl - v;
            if (lane == MCS_WARPS - 1) s_base = incl ? atomicAdd(alive, incl) : 0u;
        }
        __syncthreads();
        if (pr.keep) {
            const uint32_t slot = s_base + wsum[warp] + lane_off;
            dx_[slot] = pr.x;
            dvx[slot] = pr.vx;
            dvy[slot] = vy;
            dvz[slot] = vz;
        }
        __syncthreads();
    }
}

namespace {

size_t tma_smem_bytes(uint32_t n_g, int stages, uint32_t &ef_pad) {
    ef_pad = (n_g + 3u) & ~3u;
    return (size_t)(stages * 4) * MC_TILE * sizeof(float) + (size_t)ef_pad * sizeof(float) +
           (size_t)stages * sizeof(uint64_t);
}

}  // namespace

int launch_move_and_compact(const float *efield, const float *sx, const float *svx, const float *svy,
                            const float *svz, float *dx_, float *dvx, float *dvy, float *dvz, uint32_t *alive,
                            const uint32_t *n_active, float factor, float dt, const cudapic_grid &g,
                            cudaStream_t stream, float *dens_out, const StepLink &link,
                            cudapic_wall_counters *wall, bool wall_ions) {
    const bool tma_ok = aligned16(sx) && aligned16(svx) && aligned16(svy) && aligned16(svz) &&
                        (g.capacity % 4u) == 0u;
    if (tma_ok) {
        const cudapic_tuning t = tuning();
        const bool dep = dens_out != nullptr;
        int copies = dep ? std::max(1, std::min(t.density_copies, MC_WARPS)) : 0;
        int stages = std::min(std::max(t.push_stages, 2), MC_MAX_STAGES);
        uint32_t ef_pad;
        auto bytes = [&](int st) {
            const size_t pad = (g.n_g + 3u) & ~3u;
            return tma_smem_bytes(g.n_g, st, ef_pad) +
                   (!dep ? 0
                    : copies ? pad * sizeof(unsigned long long) + (size_t)copies * pad * sizeof(uint32_t)
                             : pad * sizeof(float));
        };
        // below 4 copies the f32 histogram (copies = 0) takes over
        auto fewer = [&]() { copies = copies / 2 < 4 ? 0 : copies / 2; };
        size_t smem = bytes(stages);
        while (smem > (size_t)max_smem_optin() && stages > 2) smem = bytes(--stages);
        while (dep && smem > (size_t)max_smem_optin() && copies > 0) {
            fewer();
            smem = bytes(stages);
        }
        if (smem > (size_t)max_smem_optin()) return fail(CUDAPIC_ERR_ARG, "move_and_compact: n_g too large");
        auto kern = dep ? move_and_compact_tma_kernel<true> : move_and_compact_tma_kernel<false>;
        int per_sm = 0;
        auto occupancy = [&]() {
            CUDAPIC_CHECK(check_cuda(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem),
                                     "cudaFuncSetAttribute(move_and_compact)"));
            return check_cuda(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, MC_THREADS, smem),
                              "occupancy(move_and_compact)");
        };
        CUDAPIC_CHECK(occupancy());
        // large grids: fewer histogram copies rather than fewer CTAs per SM
        while (dep && per_sm < t.push_ctas_per_sm && copies > 0) {
            fewer();
            smem = bytes(stages);
            CUDAPIC_CHECK(occupancy());
        }
        per_sm = std::min(std::max(per_sm, 1), t.push_ctas_per_sm);
        const uint64_t tiles_max = ((uint64_t)g.capacity + MC_TILE - 1) / MC_TILE;
        const unsigned grid = persistent_grid(per_sm, tiles_max);
        // tiles per drain: a copy receives the particles of ceil(MC_WARPS / copies) warps, MC_U * 32 per tile each
        const uint32_t per_tile = (uint32_t)((MC_WARPS + std::max(copies, 1) - 1) / std::max(copies, 1)) * MC_U * 32u;
        const uint32_t epoch = copies ? std::max(1u, DEP_MAX_PER_COPY / per_tile) : 0xffffffffu;
        return launch_kernel("move_and_compact_tma", kern, dim3(grid), dim3(MC_THREADS), smem, stream, efield, sx, svx,
                             svy, svz, dx_, dvx, dvy, dvz, alive, n_active, factor, dt, g, ef_pad, stages, dens_out,
                             copies, epoch, link, wall, (int)wall_ions);
    }
    if (dens_out || link.ticket) {  // unaligned buffers: separate deposit and count copy
        CUDAPIC_CHECK(launch_move_and_compact(efield, sx, svx, svy, svz, dx_, dvx, dvy, dvz, alive, n_active, factor,
                                              dt, g, stream, nullptr, StepLink(), wall, wall_ions));
        if (dens_out) CUDAPIC_CHECK(cudapic_get_density(dx_, dens_out, alive, &g, (cudapic_stream_t)stream));
        if (link.ticket) {
            CUDAPIC_CHECK(check_cuda(cudaMemcpyAsync(link.dst, link.src, sizeof(uint32_t), cudaMemcpyDeviceToDevice,
                                                     stream), "publish count"));
            if (link.clear_src)
                CUDAPIC_CHECK(check_cuda(cudaMemsetAsync(link.src, 0, sizeof(uint32_t), stream), "clear count"));
        }
        return CUDAPIC_OK;
    }
    const size_t smem = (size_t)g.n_g * sizeof(float);
    if (smem > 48 * 1024)
        CUDAPIC_CHECK(check_cuda(cudaFuncSetAttribute(move_and_compact_simple_kernel,
                                                      cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem),
                                 "cudaFuncSetAttribute(move_and_compact_simple)"));
    const uint64_t blocks_max = ((uint64_t)g.capacity + MCS_THREADS - 1) / MCS_THREADS;
    const unsigned grid = (unsigned)std::max<uint64_t>(1, std::min<uint64_t>((uint64_t)sm_count() * 4, blocks_max));
    return launch_kernel("move_and_compact_simple", move_and_compact_simple_kernel, dim3(grid), dim3(MCS_THREADS), smem,
                         stream, efield, sx, svx, svy, svz, dx_, dvx, dvy, dvz, alive, n_active, factor, dt, g, wall,
                         (int)wall_ions);
}

}  // namespace cudapic

using namespace cudapic;

extern "C" int cudapic_move_and_compact(const float *efield, const float *src_x, const float *src_vx,
                                        const float *src_vy, const float *src_vz, float *dst_x, float *dst_vx,
                                        float *dst_vy, float *dst_vz, uint32_t *alive_counter,
                                        const uint32_t *n_active, float factor, float dt,
                                        const cudapic_grid *grid, cudapic_stream_t stream) {
    CUDAPIC_CHECK(validate_grid(grid));
    CUDAPIC_REQUIRE(efield && src_x && src_vx && src_vy && src_vz && dst_x && dst_vx && dst_vy && dst_vz &&
                        alive_counter && n_active,
                    "move_and_compact: null pointer");
    CUDAPIC_REQUIRE(src_x != dst_x && src_vx != dst_vx && src_vy != dst_vy && src_vz != dst_vz,
                    "move_and_compact: src and dst must be distinct buffers");
    return launch_move_and_compact(efield, src_x, src_vx, src_vy, src_vz, dst_x, dst_vx, dst_vy, dst_vz,
                                   alive_counter, n_active, factor, dt, *grid, (cudaStream_t)stream);
}

extern "C" int cudapic_move_and_compact_deposit(const float *efield, const float *src_x, const float *src_vx,
                                                const float *src_vy, const float *src_vz, float *dst_x,
                                                float *dst_vx, float *dst_vy, float *dst_vz,
                                                uint32_t *alive_counter, const uint32_t *n_active, float factor,
                                                float dt, float *next_density, const cudapic_grid *grid,
                                                cudapic_stream_t stream) {
    CUDAPIC_CHECK(validate_grid(grid));
    CUDAPIC_REQUIRE(efield && src_x && src_vx && src_vy && src_vz && dst_x && dst_vx && dst_vy && dst_vz &&
                        alive_counter && n_active && next_density,
                    "move_and_compact_deposit: null pointer");
    CUDAPIC_REQUIRE(src_x != dst_x && src_vx != dst_vx && src_vy != dst_vy && src_vz != dst_vz,
                    "move_and_compact_deposit: src and dst must be distinct buffers");
    return launch_move_and_compact(efield, src_x, src_vx, src_vy, src_vz, dst_x, dst_vx, dst_vy, dst_vz,
                                   alive_counter, n_active, factor, dt, *grid, (cudaStream_t)stream, next_density);
}

extern "C" int cudapic_move_and_compact_wall(const float *efield, const float *src_x, const float *src_vx,
                                             const float *src_vy, const float *src_vz, float *dst_x, float *dst_vx,
                                             float *dst_vy, float *dst_vz, uint32_t *alive_counter,
                                             const uint32_t *n_active, float factor, float dt,
                                             cudapic_wall_counters *wall, int ions, const cudapic_grid *grid,
                                             cudapic_stream_t stream) {
    CUDAPIC_CHECK(validate_grid(grid));
    CUDAPIC_REQUIRE(efield && src_x && src_vx && src_vy && src_vz && dst_x && dst_vx && dst_vy && dst_vz &&
                        alive_counter && n_active && wall,
                    "move_and_compact_wall: null pointer");
    CUDAPIC_REQUIRE(src_x != dst_x && src_vx != dst_vx && src_vy != dst_vy && src_vz != dst_vz,
                    "move_and_compact_wall: src and dst must be distinct buffers");
    return launch_move_and_compact(efield, src_x, src_vx, src_vy, src_vz, dst_x, dst_vx, dst_vy, dst_vz,
                                   alive_counter, n_active, factor, dt, *grid, (cudaStream_t)stream, nullptr,
                                   StepLink(), wall, ions != 0);
}
