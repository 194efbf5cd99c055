// kernels_density.cu -- charge deposition (get_density) and its accumulator.
//
// Reference: get_density, Rust-CUDA/src/main.rs:356-406 (one N_G shared
// histogram per 512-thread block updated with shared f32 atomics, flushed
// with one global atomic per non-zero node and block).
//
// B200 design:
//  * persistent grid (SMs x resident CTAs, whole clusters), float4 loads of x;
//  * warp-privatised shared histograms: warp w adds into copy (w % copies),
//    so concurrent shared atomics of different warps never contend on the
//    same word;
//  * the shared-atomic pipe bounds this kernel.  Measured on B200 with
//    random nodes: 32-bit integer adds about 11.5 lane-updates per clock per
//    SM, f32 adds 3.8, 64-bit adds 2.0.  So the default arithmetic is 2^-20
//    fixed point: weights 2^20 - r and r, r = round(rem 2^20), added with
//    32-bit integer atomics and drained into a 64-bit per-CTA accumulator
//    before a copy can overflow (a weight's quantum 2^-21 is below the f32
//    rounding of x * inv_dx the reference already carries; the sums are
//    exact and order-independent within a cluster);
//  * CUDAPIC_FLAG_DEPOSIT_F32: the reference's f32 weights (1-rem) W, rem W
//    added with shared f32 atomics;
//  * CUDAPIC_FLAG_DEPOSIT_FIXED_POINT: 32.32 fixed point, round(rem * 2^32)
//    (exact for every pos >= 1), summed with 64-bit integer atomics;
//  * copies are summed inside the CTA, then the CTAs of a thread-block
//    cluster sum their histograms through distributed shared memory, and one
//    CTA per cluster adds each node (boundary nodes doubled) to the f32
//    density with one global atomic.
// CTA size, copies, cluster size and CTAs per SM come from cudapic_tuning.
// HBM traffic: 4 B per particle (x) plus the flush.
#include <cooperative_groups.h>

#include <algorithm>

#include "common.cuh"
#include "internal.h"

namespace cg = cooperative_groups;

namespace cudapic {

using u64 = unsigned long long;

__device__ __forceinline__ float cic_fraction(float xv, const cudapic_grid &g, int &p) {
    const float pos = xv * g.inv_dx;
    if (!(pos >= 0.0f && pos < (float)g.n_g - 0.5f)) set_dev_err(g.dev_err, CUDAPIC_DEVERR_POSITION);
    p = cell_of(pos, g.n_g);
    return pos - (float)p;
}

// reference arithmetic: c1 = (1-rem) W, c2 = rem W in f32 (Rust-CUDA/src/main.rs:377-387)
__device__ __forceinline__ void deposit_one(float xv, float *h, const cudapic_grid &g) {
    int p;
    const float rem = cic_fraction(xv, g, p);
    atomicAdd(&h[p], (1.0f - rem) * g.weight_factor);
    atomicAdd(&h[p + 1], rem * g.weight_factor);
}

// fixed point: weights 2^32 - r and r, r = round(rem 2^32)
__device__ __forceinline__ void deposit_one(float xv, u64 *h, const cudapic_grid &g) {
    int p;
    const float rem = cic_fraction(xv, g, p);
    const u64 r = __float2ull_rn(rem * 4294967296.0f);
    atomicAdd(&h[p], (1ull << 32) - r);
    atomicAdd(&h[p + 1], r);
}

__device__ __forceinline__ float node_value(float s, const cudapic_grid &) { return s; }
__device__ __forceinline__ float node_value(u64 s, const cudapic_grid &g) {
    return (float)((double)s * (g.weight_factor_d * 0x1p-32));
}

template <int BLOCK, bool VEC, typename Acc>
__global__ void __launch_bounds__(BLOCK)
    get_density_kernel(const float *__restrict__ x, float *__restrict__ density,
                       const uint32_t *__restrict__ n_active, const cudapic_grid g, int copies) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    Acc *hist = reinterpret_cast<Acc *>(smem_raw);
    const uint32_t n_g = g.n_g;
    const int tid = threadIdx.x;
    for (uint32_t k = tid; k < (uint32_t)copies * n_g; k += BLOCK) hist[k] = Acc(0);
    __syncthreads();
    grid_dep_wait();

    const uint32_t n = load_count(n_active, g.capacity, g.dev_err);
    Acc *h = hist + (uint32_t)((tid >> 5) % copies) * n_g;
    const uint32_t stride = gridDim.x * BLOCK;
    const uint32_t start = blockIdx.x * BLOCK + tid;
    if (VEC) {
        const uint32_t n4 = n >> 2;
        const float4 *x4 = reinterpret_cast<const float4 *>(x);
        for (uint32_t j = start; j < n4; j += stride) {
            const float4 v = x4[j];
            deposit_one(v.x, h, g);
            deposit_one(v.y, h, g);
            deposit_one(v.z, h, g);
            deposit_one(v.w, h, g);
        }
        for (uint32_t i = (n4 << 2) + start; i < n; i += stride) deposit_one(x[i], h, g);
    } else {
        for (uint32_t i = start; i < n; i += stride) deposit_one(x[i], h, g);
    }
    __syncthreads();

    // sum the warp copies into copy 0
    if (copies > 1) {
        for (uint32_t k = tid; k < n_g; k += BLOCK) {
            Acc s = hist[k];
            for (int c = 1; c < copies; ++c) s += hist[(uint32_t)c * n_g + k];
            hist[k] = s;
        }
    }

    // cluster reduction through distributed shared memory, then flush
    cg::cluster_group cluster = cg::this_cluster();
    cluster.sync();
    const unsigned rank = cluster.block_rank();
    const unsigned csize = cluster.num_blocks();
    const uint32_t chunk = (n_g + csize - 1) / csize;
    const uint32_t k0 = rank * chunk;
    const uint32_t k1 = min(n_g, k0 + chunk);
    for (uint32_t k = k0 + tid; k < k1; k += BLOCK) {
        Acc s = Acc(0);
        for (unsigned q = 0; q < csize; ++q) {
            const Acc *remote = cluster.map_shared_rank(hist, q);
            s += remote[k];
        }
        if (s != Acc(0)) {
            float v = node_value(s, g);
            if (k == 0 || k == n_g - 1) v *= 2.0f;
            atomicAdd(&density[k], v);
        }
    }
    cluster.sync();
}

// Default arithmetic: weights 2^20 - r and r, r = round(rem 2^20), added with
// 32-bit integer shared atomics into warp-private copies.  A node of a copy
// gains at most 2^20 per particle of that copy, so the copies are drained
// into the CTA's 64-bit accumulator `acc` every `epoch` rounds of the grid
// loop, before 2^12 - 1 particles can have reached one copy.
constexpr uint32_t DX_Q = 20;
constexpr uint32_t DX_MAX_PER_COPY = (1u << (32 - DX_Q)) - 1;

__device__ __forceinline__ void deposit_fx(float xv, uint32_t *h, const cudapic_grid &g) {
    int p;
    const float rem = cic_fraction(xv, g, p);
    const uint32_t r = min(__float2uint_rn(rem * (float)(1u << DX_Q)), 1u << DX_Q);  // rem <= 1 + ulp at x = L
    atomicAdd(&h[p], (1u << DX_Q) - r);
    atomicAdd(&h[p + 1], r);
}

__device__ __forceinline__ void drain_fx(uint32_t *hist, int copies, uint32_t n_g, u64 *acc, int block) {
    for (uint32_t k = threadIdx.x; k < n_g; k += block) {
        u64 v = acc[k];
        for (int c = 0; c < copies; ++c) {
            v += hist[(uint32_t)c * n_g + k];
            hist[(uint32_t)c * n_g + k] = 0u;
        }
        acc[k] = v;
    }
}

template <int BLOCK, bool VEC>
__global__ void __launch_bounds__(BLOCK)
    get_density_fx_kernel(const float *__restrict__ x, float *__restrict__ density,
                          const uint32_t *__restrict__ n_active, const cudapic_grid g, int copies,
                          uint32_t acc_pad, uint32_t epoch) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    u64 *acc = reinterpret_cast<u64 *>(smem_raw);                // [acc_pad]
    uint32_t *hist = reinterpret_cast<uint32_t *>(acc + acc_pad);  // [copies][n_g]
    const uint32_t n_g = g.n_g;
    const int tid = threadIdx.x;
    for (uint32_t k = tid; k < (uint32_t)copies * n_g; k += BLOCK) hist[k] = 0u;
    for (uint32_t k = tid; k < n_g; k += BLOCK) acc[k] = 0ull;
    __syncthreads();
    grid_dep_wait();

    const uint32_t n = load_count(n_active, g.capacity, g.dev_err);
    uint32_t *h = hist + (uint32_t)((tid >> 5) % copies) * n_g;
    const uint64_t stride = (uint64_t)gridDim.x * BLOCK;
    const uint64_t start = (uint64_t)blockIdx.x * BLOCK + tid;
    const uint64_t nv = VEC ? (n >> 2) : n;            // float4 items or particles
    const uint32_t rounds = (uint32_t)((nv + stride - 1) / stride);
    for (uint32_t r = 0; r < rounds; ++r) {            // uniform trip count: drains need the whole CTA
        if (r != 0 && r % epoch == 0) {
            __syncthreads();
            drain_fx(hist, copies, n_g, acc, BLOCK);
            __syncthreads();
        }
        const uint64_t j = (uint64_t)r * stride + start;
        if (j < nv) {
            if (VEC) {
                const float4 v = reinterpret_cast<const float4 *>(x)[j];
                deposit_fx(v.x, h, g);
                deposit_fx(v.y, h, g);
                deposit_fx(v.z, h, g);
                deposit_fx(v.w, h, g);
            } else {
                deposit_fx(x[j], h, g);
            }
        }
    }
    if (VEC) {  // the last n % 4 particles, one per thread
        const uint64_t i = (nv << 2) + start;
        if (i < n) deposit_fx(x[i], h, g);
    }
    __syncthreads();
    drain_fx(hist, copies, n_g, acc, BLOCK);

    // cluster reduction of the accumulators through distributed shared memory, then flush
    cg::cluster_group cluster = cg::this_cluster();
    cluster.sync();
    const unsigned rank = cluster.block_rank();
    const unsigned csize = cluster.num_blocks();
    const uint32_t chunk = (n_g + csize - 1) / csize;
    const uint32_t k0 = rank * chunk;
    const uint32_t k1 = min(n_g, k0 + chunk);
    const double w = g.weight_factor_d * (1.0 / (double)(1u << DX_Q));
    for (uint32_t k = k0 + tid; k < k1; k += BLOCK) {
        u64 s = 0ull;
        for (unsigned q = 0; q < csize; ++q) s += cluster.map_shared_rank(acc, q)[k];
        if (s != 0ull) {
            float v = (float)((double)s * w);
            if (k == 0 || k == n_g - 1) v *= 2.0f;
            atomicAdd(&density[k], v);
        }
    }
    cluster.sync();
}

// accumulate_density, Rust-CUDA/src/main.rs:1294-1299.
__global__ void accumulate_density_kernel(const float *__restrict__ density, double *__restrict__ cumul,
                                          uint32_t n_g) {
    grid_dep_wait();
    uint32_t k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k < n_g) cumul[k] += (double)density[k];
}

namespace {

// Cluster launch of a density kernel on a persistent grid of whole clusters.
template <typename Kern, typename... Args>
int launch_clustered(Kern kern, int block, size_t smem, const cudapic_grid &g, const cudapic_tuning &t,
                     cudaStream_t stream, Args... args) {
    CUDAPIC_CHECK(check_cuda(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem),
                             "cudaFuncSetAttribute(get_density)"));
    cudaLaunchConfig_t cfg = {};
    cudaLaunchAttribute attr[2];
    attr[0].id = cudaLaunchAttributeClusterDimension;
    attr[0].val.clusterDim.x = (unsigned)t.density_cluster;
    attr[0].val.clusterDim.y = 1;
    attr[0].val.clusterDim.z = 1;
    cfg.blockDim = dim3(block);
    cfg.dynamicSmemBytes = smem;
    cfg.stream = stream;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    const int cl = t.density_cluster;
    int max_clusters = 0;
    cfg.gridDim = dim3(cl * 64);
    CUDAPIC_CHECK(check_cuda(cudaOccupancyMaxActiveClusters(&max_clusters, kern, &cfg),
                             "cudaOccupancyMaxActiveClusters(get_density)"));
    if (max_clusters < 1) return fail(CUDAPIC_ERR_NOT_SUPPORTED, "get_density: no resident cluster");
    const uint64_t want = (uint64_t)sm_count() * (uint64_t)t.density_ctas_per_sm / (uint64_t)cl;
    const uint64_t need = ((uint64_t)g.capacity + 4ull * block - 1) / (4ull * block);
    const uint64_t clusters = std::min(std::min((uint64_t)max_clusters, std::max<uint64_t>(1, want)),
                                       std::max<uint64_t>(1, (need + cl - 1) / cl));
    cfg.gridDim = dim3((unsigned)(clusters * cl));
    if (pdl_enabled()) {
        attr[1].id = cudaLaunchAttributeProgrammaticStreamSerialization;
        attr[1].val.programmaticStreamSerializationAllowed = 1;
        cfg.numAttrs = 2;
    }
    CUDAPIC_CHECK(check_cuda(cudaLaunchKernelEx(&cfg, kern, args...), "launch get_density"));
    return CUDAPIC_OK;
}

template <int BLOCK, bool VEC, typename Acc>
int launch_density_t(const float *x, float *density, const uint32_t *n_active, const cudapic_grid &g,
                     const cudapic_tuning &t, cudaStream_t stream) {
    const size_t per_copy = (size_t)g.n_g * sizeof(Acc);
    const size_t budget = (size_t)max_smem_optin();
    if (per_copy > budget) return fail(CUDAPIC_ERR_ARG, "get_density: n_g too large for one shared histogram");
    int copies = std::min(t.density_copies, BLOCK / 32);
    copies = (int)std::min<size_t>((size_t)copies, std::max<size_t>(1, budget / per_copy));
    return launch_clustered(get_density_kernel<BLOCK, VEC, Acc>, BLOCK, per_copy * (size_t)copies, g, t, stream, x,
                            density, n_active, g, copies);
}

constexpr int DX_NO_FIT = -1;  // not a status: the fixed-point histograms do not fit in shared memory

template <int BLOCK, bool VEC>
int launch_density_fx(const float *x, float *density, const uint32_t *n_active, const cudapic_grid &g,
                      const cudapic_tuning &t, cudaStream_t stream) {
    constexpr int WARPS = BLOCK / 32;
    const uint32_t acc_pad = (g.n_g + 1u) & ~1u;
    const size_t fixed = (size_t)acc_pad * sizeof(u64);
    const size_t per_copy = (size_t)g.n_g * sizeof(uint32_t);
    const size_t budget = (size_t)max_smem_optin();
    int copies = std::min(t.density_copies, WARPS);
    while (copies > 1 && fixed + per_copy * copies > budget) --copies;
    // particles one copy receives per round: ceil(WARPS / copies) warps x 32 lanes x (4 or 1)
    auto per_round = [&](int c) { return (uint32_t)((WARPS + c - 1) / c) * 32u * (VEC ? 4u : 1u); };
    const uint32_t tail = VEC ? 3u : 0u;                   // the n % 4 particles after the last round
    while (copies < WARPS && per_round(copies) + tail > DX_MAX_PER_COPY) ++copies;
    if (fixed + per_copy * copies > budget || per_round(copies) + tail > DX_MAX_PER_COPY) return DX_NO_FIT;
    const uint32_t epoch = std::max(1u, (DX_MAX_PER_COPY - tail) / per_round(copies));
    const size_t smem = fixed + per_copy * copies;
    return launch_clustered(get_density_fx_kernel<BLOCK, VEC>, BLOCK, smem, g, t, stream, x, density, n_active, g,
                            copies, acc_pad, epoch);
}

template <bool VEC>
int launch_density_fx_any(const float *x, float *density, const uint32_t *n_active, const cudapic_grid &g,
                          cudaStream_t stream) {
    const cudapic_tuning t = tuning();
    switch (t.density_threads) {
    case 256: return launch_density_fx<256, VEC>(x, density, n_active, g, t, stream);
    case 1024: return launch_density_fx<1024, VEC>(x, density, n_active, g, t, stream);
    default: return launch_density_fx<512, VEC>(x, density, n_active, g, t, stream);
    }
}

template <bool VEC, typename Acc>
int launch_density_acc(const float *x, float *density, const uint32_t *n_active, const cudapic_grid &g,
                       cudaStream_t stream) {
    const cudapic_tuning t = tuning();
    switch (t.density_threads) {
    case 256: return launch_density_t<256, VEC, Acc>(x, density, n_active, g, t, stream);
    case 1024: return launch_density_t<1024, VEC, Acc>(x, density, n_active, g, t, stream);
    default: return launch_density_t<512, VEC, Acc>(x, density, n_active, g, t, stream);
    }
}

template <bool VEC>
int launch_density(const float *x, float *density, const uint32_t *n_active, const cudapic_grid &g,
                   cudaStream_t stream) {
    if (g.flags & CUDAPIC_FLAG_DEPOSIT_FIXED_POINT) return launch_density_acc<VEC, u64>(x, density, n_active, g, stream);
    if (!(g.flags & CUDAPIC_FLAG_DEPOSIT_F32)) {
        const int rc = launch_density_fx_any<VEC>(x, density, n_active, g, stream);
        if (rc != DX_NO_FIT) return rc;   // histograms too large for shared memory: f32 below
    }
    return launch_density_acc<VEC, float>(x, density, n_active, g, stream);
}

}  // namespace
}  // namespace cudapic

using namespace cudapic;

extern "C" int cudapic_get_density(const float *x, float *density, const uint32_t *n_active,
                                   const cudapic_grid *grid, cudapic_stream_t stream) {
    CUDAPIC_CHECK(validate_grid(grid));
    CUDAPIC_REQUIRE(x && density && n_active, "get_density: null pointer");
    if (aligned16(x)) return launch_density<true>(x, density, n_active, *grid, (cudaStream_t)stream);
    return launch_density<false>(x, density, n_active, *grid, (cudaStream_t)stream);
}

extern "C" int cudapic_accumulate_density(const float *density, double *cumul, const cudapic_grid *grid,
                                          cudapic_stream_t stream) {
    CUDAPIC_CHECK(validate_grid(grid));
    CUDAPIC_REQUIRE(density && cumul, "accumulate_density: null pointer");
    const int block = 256;
    return launch_kernel("accumulate_density", accumulate_density_kernel, dim3((grid->n_g + block - 1) / block),
                         dim3(block), 0, (cudaStream_t)stream, density, cumul, grid->n_g);
}
