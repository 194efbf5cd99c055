// kernels_push.cu -- leapfrog push + electrode absorption + stream compaction.
//
// Reference: move_and_compact, Rust-CUDA/src/main.rs:566-678.  Per particle:
//   e_x = (1-c2) E[p] + c2 E[p+1]   (CIC gather, p = int(x/dx), c2 = frac)
//   v'  = v + factor e_x,  x' = x + v' dt,  kept iff 0 <= x' <= L,
// survivors appended to dst at a block base from one atomicAdd on
// alive_counter; order across blocks is unspecified (as in the reference).
//
// B200 design (HBM-bound, 16 B read + 16 B written per survivor):
//  * persistent grid, 256 threads, tiles of 2048 particles;
//  * the four SoA input tiles (x, vx, vy, vz: 4 x 8 KB) are staged into
//    shared memory by cp.async.bulk (TMA bulk copies) on an mbarrier,
//    double-buffered so the next tile streams in while this one computes;
//  * the field E[N_G] sits in shared memory for the gathers;
//  * each thread takes 4 consecutive particles of each 1024-particle row
//    (conflict-free float4 shared loads); per-thread survivor counts of
//    both rows are packed into one int and scanned once across the block
//    (warp shuffles + one warp over the 8 warp totals);
//  * one atomicAdd per tile on alive_counter;
//  * survivors are compacted into a shared output tile, then written with
//    fully coalesced stores.
// A simple one-particle-per-thread variant (ballot/popc, reference layout)
// serves pointers that are not 16-byte aligned or capacities that are not
// a multiple of 4.
#include "common.cuh"
#include "internal.h"
#include "tma.cuh"

namespace cudapic {

constexpr int MC_THREADS = 256;
constexpr int MC_WARPS = MC_THREADS / 32;
constexpr int MC_ROW = MC_THREADS * 4;   // 1024 particles per row
constexpr int MC_TILE = 2 * MC_ROW;      // 2048 particles per tile
constexpr int MC_STAGES = 2;

struct PushResult {
    float x, vx;
    bool keep;
};

__device__ __forceinline__ PushResult push_one(float xi, float vxi, const float *ef, float factor, float dt,
                                               const cudapic_grid &g) {
    float pos = xi * g.inv_dx;
    if (!(pos >= 0.0f && pos < (float)g.n_g - 0.5f)) set_dev_err(g.dev_err, CUDAPIC_DEVERR_POSITION);
    int p = cell_of(pos, g.n_g);
    float c2 = pos - (float)p;
    float e_x = (1.0f - c2) * ef[p] + c2 * ef[p + 1];
    PushResult r;
    r.vx = vxi + factor * e_x;
    r.x = xi + r.vx * dt;
    r.keep = r.x >= 0.0f && r.x <= g.gap;
    return r;
}

__global__ void __launch_bounds__(MC_THREADS)
    move_and_compact_tma_kernel(const float *__restrict__ efield, const float *__restrict__ sx,
                                const float *__restrict__ svx, const float *__restrict__ svy,
                                const float *__restrict__ svz, float *__restrict__ dx_,
                                float *__restrict__ dvx, float *__restrict__ dvy, float *__restrict__ dvz,
                                uint32_t *__restrict__ alive, const uint32_t *__restrict__ n_active,
                                float factor, float dt, const cudapic_grid g, uint32_t ef_pad) {
    extern __shared__ __align__(128) unsigned char smem[];
    float *in = reinterpret_cast<float *>(smem);            // [STAGES][4][TILE]
    float *out = in + MC_STAGES * 4 * MC_TILE;               // [4][TILE]
    float *ef = out + 4 * MC_TILE;                           // [ef_pad]
    uint64_t *bar = reinterpret_cast<uint64_t *>(ef + ef_pad);
    __shared__ uint32_t wsum[MC_WARPS];
    __shared__ uint32_t s_base, s_tot0, s_total;
    __shared__ int s_ready;

    const int tid = threadIdx.x;
    const int lane = tid & 31;
    const int warp = tid >> 5;
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

    if (tid == 0) {
#pragma unroll
        for (int s = 0; s < MC_STAGES; ++s) mbar_init(&bar[s], 1);
        fence_mbar_init();
    }
    for (uint32_t k = tid; k < g.n_g; k += MC_THREADS) ef[k] = efield[k];
    __syncthreads();
    if (tid == 0) {
        for (int s = 0; s < MC_STAGES; ++s) {
            uint32_t tile = blockIdx.x + (uint32_t)s * gridDim.x;
            if (tile < ntiles) issue(tile, s);
        }
    }

    uint32_t it = 0;
    for (uint32_t tile = blockIdx.x; tile < ntiles; tile += gridDim.x, ++it) {
        const int s = (int)(it % MC_STAGES);
        const uint32_t parity = (it / MC_STAGES) & 1u;
        // One thread waits (bounded) on the stage's barrier and publishes the
        // verdict, so that a timeout makes the whole CTA leave together.
        if (tid == 0) {
            int ok = mbar_wait_bounded(&bar[s], parity) ? 1 : 0;
            if (!ok) {
                set_dev_err(g.dev_err, CUDAPIC_DEVERR_TIMEOUT);
                // the other stage's copy, if one was issued, must land before exit
                if (tile + gridDim.x < ntiles) mbar_wait_bounded(&bar[s ^ 1], ((it + 1) / MC_STAGES) & 1u);
            }
            s_ready = ok;
        }
        __syncthreads();
        if (!s_ready) return;
        const uint32_t t0 = tile * MC_TILE;
        const uint32_t cnt = min((uint32_t)MC_TILE, n - t0);
        const float *bx = in + (s * 4 + 0) * MC_TILE;
        const float *bvx = in + (s * 4 + 1) * MC_TILE;
        const float *bvy = in + (s * 4 + 2) * MC_TILE;
        const float *bvz = in + (s * 4 + 3) * MC_TILE;

        float ox[8], ovx[8], ovy[8], ovz[8];
        uint32_t keep = 0;
#pragma unroll
        for (int r = 0; r < 2; ++r) {
            const uint32_t j = (uint32_t)r * MC_ROW + 4u * (uint32_t)tid;
            const float4 X = *reinterpret_cast<const float4 *>(bx + j);
            const float4 VX = *reinterpret_cast<const float4 *>(bvx + j);
            const float4 VY = *reinterpret_cast<const float4 *>(bvy + j);
            const float4 VZ = *reinterpret_cast<const float4 *>(bvz + j);
            const float xs[4] = {X.x, X.y, X.z, X.w};
            const float vxs[4] = {VX.x, VX.y, VX.z, VX.w};
            const float vys[4] = {VY.x, VY.y, VY.z, VY.w};
            const float vzs[4] = {VZ.x, VZ.y, VZ.z, VZ.w};
#pragma unroll
            for (int q = 0; q < 4; ++q) {
                const int o = r * 4 + q;
                if (j + q < cnt) {
                    PushResult pr = push_one(xs[q], vxs[q], ef, factor, dt, g);
                    ox[o] = pr.x;
                    ovx[o] = pr.vx;
                    ovy[o] = vys[q];
                    ovz[o] = vzs[q];
                    if (pr.keep) keep |= 1u << o;
                } else {
                    ox[o] = ovx[o] = ovy[o] = ovz[o] = 0.0f;
                }
            }
        }
        const uint32_t packed = (uint32_t)__popc(keep & 0xfu) | ((uint32_t)__popc(keep >> 4) << 16);
        uint32_t incl = packed;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            uint32_t v = __shfl_up_sync(0xffffffffu, incl, o);
            if (lane >= o) incl += v;
        }
        if (lane == 31) wsum[warp] = incl;
        __syncthreads();  // (A) stage s fully read; warp totals visible
        if (tid == 0) {
            const uint32_t next = tile + (uint32_t)MC_STAGES * gridDim.x;
            if (next < ntiles) issue(next, s);
        }
        if (warp == 0) {
            uint32_t w = lane < MC_WARPS ? wsum[lane] : 0u;
#pragma unroll
            for (int o = 1; o < MC_WARPS; o <<= 1) {
                uint32_t v = __shfl_up_sync(0xffffffffu, w, o);
                if (lane >= o) w += v;
            }
            if (lane < MC_WARPS) wsum[lane] = w;
            if (lane == MC_WARPS - 1) {
                const uint32_t tot0 = w & 0xffffu;
                const uint32_t total = tot0 + (w >> 16);
                s_tot0 = tot0;
                s_total = total;
                s_base = total ? atomicAdd(alive, total) : 0u;
            }
        }
        __syncthreads();  // (B)
        const uint32_t excl = incl - packed + (warp > 0 ? wsum[warp - 1] : 0u);
        uint32_t off0 = excl & 0xffffu;
        uint32_t off1 = s_tot0 + (excl >> 16);
#pragma unroll
        for (int o = 0; o < 8; ++o) {
            if (keep & (1u << o)) {
                const uint32_t dst = o < 4 ? off0++ : off1++;
                out[0 * MC_TILE + dst] = ox[o];
                out[1 * MC_TILE + dst] = ovx[o];
                out[2 * MC_TILE + dst] = ovy[o];
                out[3 * MC_TILE + dst] = ovz[o];
            }
        }
        __syncthreads();  // (C)
        const uint32_t total = s_total;
        const uint32_t base = s_base;
        for (uint32_t j = tid; j < total; j += MC_THREADS) {
            dx_[base + j] = out[0 * MC_TILE + j];
            dvx[base + j] = out[1 * MC_TILE + j];
            dvy[base + j] = out[2 * MC_TILE + j];
            dvz[base + j] = out[3 * MC_TILE + j];
        }
    }
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
                                   float factor, float dt, const cudapic_grid g) {
    extern __shared__ float ef[];
    __shared__ uint32_t wsum[MCS_WARPS];
    __shared__ uint32_t s_base;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    for (uint32_t k = tid; k < g.n_g; k += MCS_THREADS) ef[k] = efield[k];
    __syncthreads();
    const uint32_t n = load_count(n_active, g.capacity, g.dev_err);
    if (g.work && blockIdx.x == 0 && tid == 0) atomicAdd(g.work, (unsigned long long)n);
    const uint32_t rounds = (n + gridDim.x * MCS_THREADS - 1) / (gridDim.x * MCS_THREADS);
    for (uint32_t rd = 0; rd < rounds; ++rd) {
        const uint32_t i = (rd * gridDim.x + blockIdx.x) * MCS_THREADS + tid;
        PushResult pr = {0.0f, 0.0f, false};
        float vy = 0.0f, vz = 0.0f;
        if (i < n) {
            pr = push_one(sx[i], svx[i], ef, factor, dt, g);
            if (pr.keep) {
                vy = svy[i];
                vz = svz[i];
            }
        }
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

size_t tma_smem_bytes(uint32_t n_g, uint32_t &ef_pad) {
    ef_pad = (n_g + 3u) & ~3u;
    return (size_t)(MC_STAGES * 4 + 4) * MC_TILE * sizeof(float) + (size_t)ef_pad * sizeof(float) +
           MC_STAGES * sizeof(uint64_t);
}

}  // namespace

int launch_move_and_compact(const float *efield, const float *sx, const float *svx, const float *svy,
                            const float *svz, float *dx_, float *dvx, float *dvy, float *dvz, uint32_t *alive,
                            const uint32_t *n_active, float factor, float dt, const cudapic_grid &g,
                            cudaStream_t stream) {
    const bool tma_ok = aligned16(sx) && aligned16(svx) && aligned16(svy) && aligned16(svz) &&
                        (g.capacity % 4u) == 0u;
    if (tma_ok) {
        uint32_t ef_pad;
        const size_t smem = tma_smem_bytes(g.n_g, ef_pad);
        if (smem > (size_t)max_smem_optin()) return fail(CUDAPIC_ERR_ARG, "move_and_compact: n_g too large");
        CUDAPIC_CHECK(check_cuda(cudaFuncSetAttribute(move_and_compact_tma_kernel,
                                                      cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem),
                                 "cudaFuncSetAttribute(move_and_compact)"));
        int per_sm = 0;
        CUDAPIC_CHECK(check_cuda(cudaOccupancyMaxActiveBlocksPerMultiprocessor(
                                     &per_sm, move_and_compact_tma_kernel, MC_THREADS, smem),
                                 "occupancy(move_and_compact)"));
        per_sm = std::max(per_sm, 1);
        const uint64_t tiles_max = ((uint64_t)g.capacity + MC_TILE - 1) / MC_TILE;
        const unsigned grid = (unsigned)std::max<uint64_t>(1, std::min<uint64_t>((uint64_t)sm_count() * per_sm,
                                                                                tiles_max));
        move_and_compact_tma_kernel<<<grid, MC_THREADS, smem, stream>>>(efield, sx, svx, svy, svz, dx_, dvx, dvy,
                                                                         dvz, alive, n_active, factor, dt, g,
                                                                         ef_pad);
        return check_launch("move_and_compact_tma");
    }
    const size_t smem = (size_t)g.n_g * sizeof(float);
    if (smem > 48 * 1024)
        CUDAPIC_CHECK(check_cuda(cudaFuncSetAttribute(move_and_compact_simple_kernel,
                                                      cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem),
                                 "cudaFuncSetAttribute(move_and_compact_simple)"));
    const uint64_t blocks_max = ((uint64_t)g.capacity + MCS_THREADS - 1) / MCS_THREADS;
    const unsigned grid = (unsigned)std::max<uint64_t>(1, std::min<uint64_t>((uint64_t)sm_count() * 4, blocks_max));
    move_and_compact_simple_kernel<<<grid, MCS_THREADS, smem, stream>>>(efield, sx, svx, svy, svz, dx_, dvx, dvy,
                                                                        dvz, alive, n_active, factor, dt, g);
    return check_launch("move_and_compact_simple");
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
