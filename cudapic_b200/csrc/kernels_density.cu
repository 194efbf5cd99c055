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
//  * default arithmetic: the reference's f32 weights (1-rem) W, rem W added
//    with shared f32 atomics (about 1.5 lane-updates per clock per SM on
//    B200: the bound of this kernel);
//  * CUDAPIC_FLAG_DEPOSIT_FIXED_POINT: the CIC fraction rem = pos - p (an f32
//    in [0, 1)) becomes the 32.32 fixed-point integer round(rem * 2^32) --
//    exact for every pos >= 1 -- and the node weights 2^32 - r and r are
//    summed with 64-bit integer shared atomics: exact and order-independent
//    within a cluster, about 25 % slower;
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

// accumulate_density, Rust-CUDA/src/main.rs:1294-1299.
__global__ void accumulate_density_kernel(const float *__restrict__ density, double *__restrict__ cumul,
                                          uint32_t n_g) {
    uint32_t k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k < n_g) cumul[k] += (double)density[k];
}

namespace {

template <int BLOCK, bool VEC, typename Acc>
int launch_density_t(const float *x, float *density, const uint32_t *n_active, const cudapic_grid &g,
                     const cudapic_tuning &t, cudaStream_t stream) {
    const size_t per_copy = (size_t)g.n_g * sizeof(Acc);
    const size_t budget = (size_t)max_smem_optin();
    if (per_copy > budget) return fail(CUDAPIC_ERR_ARG, "get_density: n_g too large for one shared histogram");
    int copies = std::min(t.density_copies, BLOCK / 32);
    copies = (int)std::min<size_t>((size_t)copies, std::max<size_t>(1, budget / per_copy));
    const size_t smem = per_copy * (size_t)copies;
    auto kern = get_density_kernel<BLOCK, VEC, Acc>;
    CUDAPIC_CHECK(check_cuda(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem),
                             "cudaFuncSetAttribute(get_density)"));
    cudaLaunchConfig_t cfg = {};
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeClusterDimension;
    attr[0].val.clusterDim.x = (unsigned)t.density_cluster;
    attr[0].val.clusterDim.y = 1;
    attr[0].val.clusterDim.z = 1;
    cfg.blockDim = dim3(BLOCK);
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
    const uint64_t need = ((uint64_t)g.capacity + 4ull * BLOCK - 1) / (4ull * BLOCK);
    const uint64_t clusters = std::min(std::min((uint64_t)max_clusters, std::max<uint64_t>(1, want)),
                                       std::max<uint64_t>(1, (need + cl - 1) / cl));
    cfg.gridDim = dim3((unsigned)(clusters * cl));
    CUDAPIC_CHECK(check_cuda(cudaLaunchKernelEx(&cfg, kern, x, density, n_active, g, copies), "launch get_density"));
    return CUDAPIC_OK;
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
    accumulate_density_kernel<<<(grid->n_g + block - 1) / block, block, 0, (cudaStream_t)stream>>>(
        density, cumul, grid->n_g);
    return check_launch("accumulate_density");
}
