// push.cuh -- leapfrog push of one particle and the fixed-point deposit
// helpers shared by move_and_compact (kernels_push.cu) and the fused
// electron step (kernels_step.cu).
//
// Reference: move_and_compact, Rust-CUDA/src/main.rs:566-678 (push) and
// get_density, :356-406 (CIC weights).
#pragma once
#include "common.cuh"

namespace cudapic {

// One particle (Rust-CUDA/src/main.rs:596-620):
//   e_x = (1-c2) E[p] + c2 E[p+1]   (CIC gather, p = int(x/dx), c2 = frac)
//   v'  = v + factor e_x,  x' = x + v' dt,  kept iff 0 <= x' <= L.
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

// push_one with the hot constants passed in (registers of the caller); the
// error word is read from `gm` only for a position out of range.
__device__ __forceinline__ PushResult push_one_c(float xi, float vxi, const float *ef, float factor, float dt,
                                                 float inv_dx, uint32_t n_g, float gap, const cudapic_grid &gm) {
    float pos = xi * inv_dx;
    if (!(pos >= 0.0f && pos < (float)n_g - 0.5f)) set_dev_err(gm.dev_err, CUDAPIC_DEVERR_POSITION);
    int p = cell_of(pos, n_g);
    float c2 = pos - (float)p;
    float e_x = (1.0f - c2) * ef[p] + c2 * ef[p + 1];
    PushResult r;
    r.vx = vxi + factor * e_x;
    r.x = xi + r.vx * dt;
    r.keep = r.x >= 0.0f && r.x <= gap;
    return r;
}

// Boundary check of C/eduPIC.cc:623-667 for one row of a warp (every lane
// calls it): particles with a pushed position x < 0 count at the powered
// electrode, x > L at the grounded one, one atomic per electrode and row;
// with ions, the energy 1/2 M v^2 / e of an absorbed ion goes to the 1 eV bin
// of that electrode's IFED (below 200 eV).
__device__ __forceinline__ void count_wall(cudapic_wall_counters *w, bool ions, bool valid, float x, float vx,
                                           float vy, float vz, float gap) {
    const bool at_pow = valid && x < 0.0f;
    const bool at_gnd = valid && x > gap;
    const unsigned mp = __ballot_sync(0xffffffffu, at_pow);
    const unsigned mg = __ballot_sync(0xffffffffu, at_gnd);
    if ((threadIdx.x & 31) == 0) {
        if (mp) atomicAdd(&w->abs_pow, (unsigned long long)__popc(mp));
        if (mg) atomicAdd(&w->abs_gnd, (unsigned long long)__popc(mg));
    }
    if (ions && (at_pow || at_gnd)) {
        const float e = HALF_MI_OVER_E * (vx * vx + vy * vy + vz * vz);
        if (e < (float)CUDAPIC_N_IFED) atomicAdd(at_pow ? &w->ifed_pow[(int)e] : &w->ifed_gnd[(int)e], 1u);
    }
}

// Fused deposit in 2^-20 fixed point.  A particle at rem = pos - p in [0, 1]
// adds 2^20 - r to node p and r to node p + 1, r = round(rem * 2^20), with
// 32-bit integer shared atomics (on sm_100a several times the throughput of
// f32 or 64-bit shared atomics; the deposit is bound by that pipe).  The
// quantum 2^-21 of a weight is below the f32 rounding of the position
// x * inv_dx that the reference's f32 arithmetic already carries, and the
// integer sums are exact and order-independent.  A node of one histogram
// copy gains at most 2^20 per particle of its copy, so the copies are
// drained into a per-CTA 64-bit accumulator before DEP_MAX_PER_COPY
// particles have reached one copy.
constexpr uint32_t DEP_Q = 20;
constexpr uint32_t DEP_MAX_PER_COPY = (1u << (32 - DEP_Q)) - 1;

__device__ __forceinline__ void dep_add(uint32_t *h, float x, const cudapic_grid &g) {
    const float pos = x * g.inv_dx;
    const int p = cell_of(pos, g.n_g);
    const float rem = pos - (float)p;
    // rem can exceed 1 by an ulp at x = L (pos rounds past N_G - 1): clamp, so no weight is negative
    const uint32_t r = min(__float2uint_rn(rem * (float)(1u << DEP_Q)), 1u << DEP_Q);
    atomicAdd(&h[p], (1u << DEP_Q) - r);
    atomicAdd(&h[p + 1], r);
}

// acc[k] += sum of the copies of node k; the copies are cleared.  Each node is
// owned by one thread: no atomics.  Callers synchronise before and after.
__device__ __forceinline__ void dep_drain(uint32_t *hist, int copies, uint32_t stride, unsigned long long *acc,
                                          uint32_t n_g) {
    for (uint32_t k = threadIdx.x; k < n_g; k += blockDim.x) {
        unsigned long long v = acc[k];
        for (int c = 0; c < copies; ++c) {
            v += hist[(uint32_t)c * stride + k];
            hist[(uint32_t)c * stride + k] = 0u;
        }
        acc[k] = v;
    }
}

// Adds v (nodes k .. k + 3) to dens_out: one 16-byte vector atomic when
// the four nodes exist and dens_out is 16-byte aligned (one L2 operation for
// four nodes: the per-CTA flushes of a large grid are bound by the number of
// global atomics), else one atomic per non-zero node.
__device__ __forceinline__ void red_add4(float *dens_out, uint32_t k, uint32_t n_g, const float (&v)[4], bool vec) {
    if (vec && k + 4u <= n_g) {
        atomicAdd(reinterpret_cast<float4 *>(dens_out + k), make_float4(v[0], v[1], v[2], v[3]));
        return;
    }
#pragma unroll
    for (int u = 0; u < 4; ++u)
        if (k + (uint32_t)u < n_g && v[u] != 0.0f) atomicAdd(&dens_out[k + u], v[u]);
}

// Adds the CTA's accumulated node weights to dens_out, boundary nodes
// doubled, and clears the accumulator (each thread the nodes it flushed:
// four consecutive ones per turn).
__device__ __forceinline__ void dep_flush(unsigned long long *acc, float *dens_out, const cudapic_grid &g) {
    const double w = g.weight_factor_d * (1.0 / (double)(1u << DEP_Q));
    const uint32_t n_g = g.n_g;
    const bool vec = (reinterpret_cast<uintptr_t>(dens_out) & 15u) == 0;
    for (uint32_t k = 4u * threadIdx.x; k < n_g; k += 4u * blockDim.x) {
        float v[4];
        bool any = false;
#pragma unroll
        for (int u = 0; u < 4; ++u) {
            const uint32_t node = k + (uint32_t)u;
            const unsigned long long a = node < n_g ? acc[node] : 0ull;
            if (node < n_g) acc[node] = 0ull;
            v[u] = a ? (float)((double)a * w) : 0.0f;
            if (node == 0 || node == n_g - 1) v[u] *= 2.0f;
            any |= a != 0ull;
        }
        if (any) red_add4(dens_out, k, n_g, v, vec);
    }
}

// The large-grid deposit of the fused kernels: CIC weights (1 - rem, rem)
// of the new position added to one f32 shared histogram per CTA (at
// thousands of nodes the lanes rarely meet on a node, and the fixed-point
// copies would need a drain every few tiles), and the flush of its nodes
// (boundary nodes doubled; four nodes per vector atomic) into dens_out,
// which clears them.
__device__ __forceinline__ void dep_add_f32(float *h, float x, const cudapic_grid &g) {
    const float pos = x * g.inv_dx;
    const int p = cell_of(pos, g.n_g);
    const float rem = fminf(pos - (float)p, 1.0f);
    atomicAdd(&h[p], 1.0f - rem);
    atomicAdd(&h[p + 1], rem);
}

__device__ __forceinline__ void dep_flush_f32(float *h, float *dens_out, const cudapic_grid &g) {
    const uint32_t n_g = g.n_g;
    const bool vec = (reinterpret_cast<uintptr_t>(dens_out) & 15u) == 0;
    for (uint32_t k = 4u * threadIdx.x; k < n_g; k += 4u * blockDim.x) {
        float v[4];
        bool any = false;
#pragma unroll
        for (int u = 0; u < 4; ++u) {
            const uint32_t node = k + (uint32_t)u;
            const float a = node < n_g ? h[node] : 0.0f;
            if (node < n_g) h[node] = 0.0f;
            v[u] = a * g.weight_factor;
            if (node == 0 || node == n_g - 1) v[u] *= 2.0f;
            any |= a != 0.0f;
        }
        if (any) red_add4(dens_out, k, n_g, v, vec);
    }
}

}  // namespace cudapic
