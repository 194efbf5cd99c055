// kernels_density.cu -- charge deposition (get_density) and its accumulator.
//
// Reference: get_density, Rust-CUDA/src/main.rs:356-406 (one N_G shared
// histogram per 512-thread block updated with shared f32 atomics, flushed
// with one global atomic per non-zero node and block).
//
// B200 design:
//  * persistent grid (SM count x resident clusters), float4 loads of x;
//  * warp-privatised shared histograms: warp w adds into copy (w % copies),
//    so concurrent shared atomics of different warps never contend on the
//    same word; `copies` is as many N_G-float copies as fit in 64 KB;
//  * copies are summed inside the CTA, then a thread-block cluster of
//    DENS_CLUSTER CTAs sums its CTAs' histograms through distributed shared
//    memory, and only one CTA per cluster touches each global node: the
//    global flush costs (grid / DENS_CLUSTER) x N_G atomics instead of
//    grid x N_G.
// HBM traffic: 4 B per particle (x) plus the flush.
#include <cooperative_groups.h>

#include "common.cuh"
#include "internal.h"

namespace cg = cooperative_groups;

namespace cudapic {

constexpr int DENS_BLOCK = 512;
constexpr int DENS_CLUSTER = 4;
constexpr int DENS_SMEM_BUDGET = 64 * 1024;

__device__ __forceinline__ void deposit_one(float xv, float *h, const cudapic_grid &g) {
    float pos = xv * g.inv_dx;
    if (!(pos >= 0.0f && pos < (float)g.n_g - 0.5f)) set_dev_err(g.dev_err, CUDAPIC_DEVERR_POSITION);
    int p = cell_of(pos, g.n_g);
    float rem = pos - (float)p;
    float c1 = (1.0f - rem) * g.weight_factor;
    float c2 = rem * g.weight_factor;
    atomicAdd(&h[p], c1);
    atomicAdd(&h[p + 1], c2);
}

template <bool VEC>
__global__ void __launch_bounds__(DENS_BLOCK)
    get_density_kernel(const float *__restrict__ x, float *__restrict__ density,
                       const uint32_t *__restrict__ n_active, const cudapic_grid g, int copies) {
    extern __shared__ float hist[];
    const uint32_t n_g = g.n_g;
    const int tid = threadIdx.x;
    for (uint32_t k = tid; k < (uint32_t)copies * n_g; k += DENS_BLOCK) hist[k] = 0.0f;
    __syncthreads();

    const uint32_t n = load_count(n_active, g.capacity, g.dev_err);
    float *h = hist + (uint32_t)((tid >> 5) % copies) * n_g;
    const uint32_t stride = gridDim.x * DENS_BLOCK;
    uint32_t start = blockIdx.x * DENS_BLOCK + tid;
    if (VEC) {
        const uint32_t n4 = n >> 2;
        const float4 *x4 = reinterpret_cast<const float4 *>(x);
        for (uint32_t j = start; j < n4; j += stride) {
            float4 v = x4[j];
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
        for (uint32_t k = tid; k < n_g; k += DENS_BLOCK) {
            float s = hist[k];
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
    for (uint32_t k = k0 + tid; k < k1; k += DENS_BLOCK) {
        float s = 0.0f;
        for (unsigned q = 0; q < csize; ++q) {
            const float *remote = cluster.map_shared_rank(hist, q);
            s += remote[k];
        }
        if (s != 0.0f) {
            if (k == 0 || k == n_g - 1) s *= 2.0f;
            atomicAdd(&density[k], s);
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

struct DensityLaunch {
    int grid = 0;
    int copies = 1;
    size_t smem = 0;
};

template <bool VEC>
int launch_density(const float *x, float *density, const uint32_t *n_active, const cudapic_grid &g,
                   cudaStream_t stream) {
    DensityLaunch L;
    const size_t per_copy = (size_t)g.n_g * sizeof(float);
    L.copies = (int)std::min<size_t>(DENS_BLOCK / 32, std::max<size_t>(1, DENS_SMEM_BUDGET / per_copy));
    L.smem = per_copy * (size_t)L.copies;
    if (L.smem > (size_t)max_smem_optin())
        return fail(CUDAPIC_ERR_ARG, "get_density: n_g too large for one shared histogram");
    auto kern = get_density_kernel<VEC>;
    CUDAPIC_CHECK(check_cuda(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                                  (int)L.smem),
                             "cudaFuncSetAttribute(get_density)"));
    cudaLaunchConfig_t cfg = {};
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeClusterDimension;
    attr[0].val.clusterDim.x = DENS_CLUSTER;
    attr[0].val.clusterDim.y = 1;
    attr[0].val.clusterDim.z = 1;
    cfg.blockDim = dim3(DENS_BLOCK);
    cfg.dynamicSmemBytes = L.smem;
    cfg.stream = stream;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    // grid: resident clusters, but no more CTAs than the capacity needs
    int max_clusters = 0;
    cfg.gridDim = dim3(DENS_CLUSTER * 64);
    CUDAPIC_CHECK(check_cuda(cudaOccupancyMaxActiveClusters(&max_clusters, kern, &cfg),
                             "cudaOccupancyMaxActiveClusters(get_density)"));
    if (max_clusters < 1) return fail(CUDAPIC_ERR_NOT_SUPPORTED, "get_density: no resident cluster");
    uint64_t need = ((uint64_t)g.capacity + 4ull * DENS_BLOCK - 1) / (4ull * DENS_BLOCK);
    uint64_t clusters = std::min<uint64_t>((uint64_t)max_clusters,
                                           std::max<uint64_t>(1, (need + DENS_CLUSTER - 1) / DENS_CLUSTER));
    cfg.gridDim = dim3((unsigned)(clusters * DENS_CLUSTER));
    CUDAPIC_CHECK(check_cuda(cudaLaunchKernelEx(&cfg, kern, x, density, n_active, g, L.copies),
                             "launch get_density"));
    return CUDAPIC_OK;
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
