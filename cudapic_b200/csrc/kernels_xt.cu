// kernels_xt.cu -- spatio-temporal (XT) diagnostics of the measurement window.
//
// Reference: the measurement branches of eduPIC's do_one_cycle
// (C/eduPIC.cc:557-576 electrons, :599-614 ions, :705-715 grid quantities),
// with norm_all_xt (:864-903) applied on the host (state.cpp).  Step t of the
// RF period adds to column j = t / N_BIN (N_BIN = 20 steps) of [N_G][N_XT]
// FP64 arrays (eduPIC's xt_distr layout):
//  * per electron at its position before the push, with the CIC weights
//    c1 = 1 - c2 (node p) and c2 (node p + 1): counter += c, ue += c v,
//    meanee += c E, ioniz_rate += c sigma_ion(E) |v| DT_E n_gas, where
//    v = vx + 1/2 factor_e e_x is the x-velocity at the time of x and E the
//    energy [eV] of (v, vy, vz);
//  * per ion on an ion step the same without the rate (factor_i);
//  * per node: the potential, the field and both densities of the step.
// The arithmetic of a particle is f32 (the kernels' precision, like the
// push that follows); eduPIC works in double.
//
// B200 design: persistent CTAs of 512 threads; each CTA sums its particles
// into f32 shared histograms of the 4 (electrons) or 3 (ions) quantities
// and adds every non-empty node to the FP64 column with one global atomic,
// so the long accumulation is FP64 while the per-step partial sums are f32.
// The batched variant walks each CTA's share of the batch's concatenated
// particles discharge by discharge (one flush per segment).
#include "batch_internal.h"
#include "common.cuh"
#include "internal.h"

namespace cudapic {

namespace {

constexpr int XT_THREADS = 512;

// Column of the step just solved: the Poisson kernel advanced the step counter.
__device__ __forceinline__ uint32_t xt_column(const uint32_t *step_counter, uint32_t n_t) {
    const uint32_t t = (*step_counter + n_t - 1u) % n_t;
    return t / XT_BIN;
}

// Adds the particles [lo, hi) of the planes to the CTA's shared histograms
// h[q * n_g + node].
template <bool ION>
__device__ __forceinline__ void xt_accumulate(const float *__restrict__ x, const float *__restrict__ vx,
                                              const float *__restrict__ vy, const float *__restrict__ vz,
                                              uint32_t lo, uint32_t hi, const float *__restrict__ ef,
                                              const float *__restrict__ cs_ion, const cudapic_grid &g, float *h) {
    const uint32_t n_g = g.n_g;
    const float factor = ION ? g.factor_i : g.factor_e;
    const float half_m = ION ? HALF_MI_OVER_E : g.half_me_over_e;
    const float rate_scale = (float)((double)g.dt_e * g.gas_density);
    for (uint32_t i = lo + threadIdx.x; i < hi; i += blockDim.x) {
        if (slot_dead(x[i])) continue;  // emptied by an in-place electron step
        const float pos = x[i] * g.inv_dx;
        const int p = cell_of(pos, n_g);
        const float c2 = pos - (float)p;
        const float c1 = 1.0f - c2;
        const float e_x = c1 * __ldg(ef + p) + c2 * __ldg(ef + p + 1);
        const float v = vx[i] + 0.5f * factor * e_x;
        const float vyi = vy[i], vzi = vz[i];
        const float v2 = v * v + vyi * vyi + vzi * vzi;
        const float energy = half_m * v2;
        atomicAdd(&h[p], c1);
        atomicAdd(&h[p + 1], c2);
        atomicAdd(&h[n_g + p], c1 * v);
        atomicAdd(&h[n_g + p + 1], c2 * v);
        atomicAdd(&h[2 * n_g + p], c1 * energy);
        atomicAdd(&h[2 * n_g + p + 1], c2 * energy);
        if (!ION) {
            const float t = fminf(energy / DE_CS_F + 0.5f, (float)(CS_RANGES - 1));
            const float rate = __ldg(cs_ion + (uint32_t)t) * sqrtf(v2) * rate_scale;
            atomicAdd(&h[3 * n_g + p], c1 * rate);
            atomicAdd(&h[3 * n_g + p + 1], c2 * rate);
        }
    }
}

// Adds the CTA's histograms to column col of the quantities q0 .. q0 + Q - 1
// of xt ([quantity][n_g][n_xt] doubles) and clears them.
__device__ __forceinline__ void xt_flush(float *h, int Q, double *xt, int q0, uint32_t n_g, uint32_t n_xt,
                                         uint32_t col) {
    __syncthreads();
    const size_t plane = (size_t)n_g * n_xt;
    for (uint32_t k = threadIdx.x; k < (uint32_t)Q * n_g; k += blockDim.x) {
        const float v = h[k];
        if (v != 0.0f) {
            const uint32_t q = k / n_g, node = k % n_g;
            atomicAdd(&xt[(size_t)(q0 + q) * plane + (size_t)node * n_xt + col], (double)v);
        }
        h[k] = 0.0f;
    }
    __syncthreads();
}

template <bool ION>
__global__ void __launch_bounds__(XT_THREADS)
    xt_particles_kernel(const float *__restrict__ x, const float *__restrict__ vx, const float *__restrict__ vy,
                        const float *__restrict__ vz, const uint32_t *__restrict__ n_active,
                        const float *__restrict__ efield, const float *__restrict__ cs,
                        const uint32_t *__restrict__ step_counter, const cudapic_grid g, uint32_t n_xt, double *xt) {
    extern __shared__ float xt_h[];  // [Q][n_g]
    constexpr int Q = ION ? 3 : 4;
    for (uint32_t k = threadIdx.x; k < Q * g.n_g; k += blockDim.x) xt_h[k] = 0.0f;
    __syncthreads();
    grid_dep_wait();
    const uint32_t n = load_count(n_active, g.capacity, g.dev_err);
    const uint32_t col = xt_column(step_counter, g.n_t);
    const uint32_t chunk = (n + gridDim.x - 1) / gridDim.x;
    const uint32_t lo = min(n, blockIdx.x * chunk), hi = min(n, lo + chunk);
    xt_accumulate<ION>(x, vx, vy, vz, lo, hi, efield, cs + 2 * CS_RANGES, g, xt_h);
    xt_flush(xt_h, Q, xt, ION ? XT_COUNT_I : XT_COUNT_E, g.n_g, n_xt, col);
}

__global__ void __launch_bounds__(256)
    xt_grid_kernel(const float *__restrict__ pot, const float *__restrict__ efield,
                   const float *__restrict__ e_density, const float *__restrict__ i_density,
                   const uint32_t *__restrict__ step_counter, const cudapic_grid g, uint32_t n_xt, double *xt) {
    grid_dep_wait();
    const uint32_t col = xt_column(step_counter, g.n_t);
    const size_t plane = (size_t)g.n_g * n_xt;
    for (uint32_t p = blockIdx.x * blockDim.x + threadIdx.x; p < g.n_g; p += gridDim.x * blockDim.x) {
        const size_t at = (size_t)p * n_xt + col;
        xt[XT_POT * plane + at] += (double)pot[p];
        xt[XT_EFIELD * plane + at] += (double)efield[p];
        xt[XT_NE * plane + at] += (double)e_density[p];
        xt[XT_NI * plane + at] += (double)i_density[p];
    }
}

// Batched: CTA c takes an equal share of the batch's concatenated particles
// of one species (pooled planes `sp`), discharge by discharge.
template <bool ION>
__global__ void __launch_bounds__(XT_THREADS)
    batch_xt_particles_kernel(const __grid_constant__ SidePlanes sp, const BatchDisc *__restrict__ desc,
                              uint32_t D) {
    extern __shared__ float bxt_h[];  // [Q][largest n_g]
    constexpr int Q = ION ? 3 : 4;
    __shared__ uint32_t cnt[BATCH_MAX_DISCHARGES];
    __shared__ uint32_t pfx[BATCH_MAX_DISCHARGES + 1];
    const int lane = threadIdx.x & 31;
    grid_dep_wait();
    // the plan: prefix of the discharges' counts (read from their counters)
    for (uint32_t d = threadIdx.x; d < D; d += blockDim.x) {
        const BatchDisc &dd = desc[d];
        cnt[d] = min(*(volatile const uint32_t *)(dd.counters + (ION ? 1 : 0)), dd.g.capacity);
    }
    __syncthreads();
    if (threadIdx.x < 32) {  // warp 0: each lane sums a block of the counts, then the warp scans the blocks
        const uint32_t per = (D + 31) / 32, a = min(D, lane * per), b = min(D, a + per);
        uint32_t sum = 0;
        for (uint32_t d = a; d < b; ++d) sum += cnt[d];
        uint32_t incl = sum;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const uint32_t t = __shfl_up_sync(0xffffffffu, incl, o);
            if (lane >= o) incl += t;
        }
        uint32_t run = incl - sum;
        for (uint32_t d = a; d < b; ++d) {
            pfx[d] = run;
            run += cnt[d];
        }
        if (lane == 31) pfx[D] = incl;
    }
    __syncthreads();
    const uint32_t total = pfx[D];
    const uint32_t chunk = (total + gridDim.x - 1) / gridDim.x;
    const uint32_t beg = min(total, blockIdx.x * chunk), end = min(total, beg + chunk);
    for (uint32_t d = 0; d < D; ++d) {
        const uint32_t a = max(beg, pfx[d]), b = min(end, pfx[d + 1]);
        if (a >= b) continue;
        const BatchDisc &dd = desc[d];
        if (!dd.xt) continue;
        const uint32_t n_g = dd.g.n_g;
        for (uint32_t k = threadIdx.x; k < Q * n_g; k += blockDim.x) bxt_h[k] = 0.0f;
        __syncthreads();
        xt_accumulate<ION>(sp.x + dd.off, sp.vx + dd.off, sp.vy + dd.off, sp.vz + dd.off, a - pfx[d], b - pfx[d],
                           dd.efield, dd.cs + 2 * CS_RANGES, dd.g, bxt_h);
        xt_flush(bxt_h, Q, dd.xt, ION ? XT_COUNT_I : XT_COUNT_E, n_g, dd.n_xt, xt_column(dd.counters + 3, dd.g.n_t));
    }
}

}  // namespace

int launch_xt_particles(bool ions, const float *x, const float *vx, const float *vy, const float *vz,
                        const uint32_t *n_active, const float *efield, const float *cs, const uint32_t *step_counter,
                        const cudapic_grid &g, uint32_t n_xt, double *xt, cudaStream_t stream) {
    const size_t smem = (size_t)(ions ? 3 : 4) * g.n_g * sizeof(float);
    if (smem > (size_t)max_smem_optin()) return fail(CUDAPIC_ERR_ARG, "xt: n_g too large");
    auto kern = ions ? xt_particles_kernel<true> : xt_particles_kernel<false>;
    CUDAPIC_CHECK(check_cuda(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem),
                             "cudaFuncSetAttribute(xt)"));
    const unsigned grid = persistent_grid(1, ((uint64_t)g.capacity + XT_THREADS - 1) / XT_THREADS);
    return launch_kernel(ions ? "xt_ions" : "xt_electrons", kern, dim3(grid), dim3(XT_THREADS), smem, stream, x, vx,
                         vy, vz, n_active, efield, cs, step_counter, g, n_xt, xt);
}

int launch_xt_grid(const float *pot, const float *efield, const float *e_density, const float *i_density,
                   const uint32_t *step_counter, const cudapic_grid &g, uint32_t n_xt, double *xt,
                   cudaStream_t stream) {
    return launch_kernel("xt_grid", xt_grid_kernel, dim3((g.n_g + 255) / 256), dim3(256), 0, stream, pot, efield,
                         e_density, i_density, step_counter, g, n_xt, xt);
}

int launch_batch_xt_particles(bool ions, const SidePlanes &sp, const BatchDisc *desc, uint32_t D, uint32_t max_n_g,
                              uint64_t cap_sum, cudaStream_t stream) {
    if (D == 0 || D > BATCH_MAX_DISCHARGES) return fail(CUDAPIC_ERR_ARG, "batch xt: bad discharge count");
    const size_t smem = (size_t)(ions ? 3 : 4) * max_n_g * sizeof(float);
    if (smem > (size_t)max_smem_optin() - sizeof(uint32_t) * (BATCH_MAX_DISCHARGES + 1))
        return fail(CUDAPIC_ERR_ARG, "batch xt: n_g too large");
    auto kern = ions ? batch_xt_particles_kernel<true> : batch_xt_particles_kernel<false>;
    CUDAPIC_CHECK(check_cuda(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem),
                             "cudaFuncSetAttribute(batch xt)"));
    const unsigned grid = persistent_grid(1, (cap_sum + XT_THREADS - 1) / XT_THREADS);
    return launch_kernel(ions ? "batch_xt_ions" : "batch_xt_electrons", kern, dim3(grid), dim3(XT_THREADS), smem,
                         stream, sp, desc, D);
}

}  // namespace cudapic
