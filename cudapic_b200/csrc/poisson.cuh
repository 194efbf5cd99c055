// poisson.cuh -- the one-CTA scan-based Poisson solve and field (the body
// of the driver's solve kernels, kernels_poisson.cu, also run by the last
// CTA of the in-place step's scatter pass, kernels_inplace.cu).
//
// Reference: solve_poisson_scan_f32, Rust-CUDA/src/main.rs:408-494.  The
// Dirichlet problem pot[i-1] - 2 pot[i] + pot[i+1] = f_i has unit
// tridiagonal coefficients, so the Thomas recurrences collapse to
//     G_i = sum_{j<=i} j f_j,   r_i = -G_i / ((i+1) i),   pot_i = i sum_{j=i}^{N-2} r_j,
// two inclusive prefix sums (C/eduPIC.cc:461-494 is the sequential Thomas
// form of the same system).
#pragma once
#include "common.cuh"

namespace cudapic {

constexpr int POIS_MAX_THREADS = 1024;
constexpr int POIS_MAX_PER_THREAD = 16;  // N_G <= 16384

template <typename T>
__device__ __forceinline__ T warp_incl_scan(T v, int lane) {
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        T n = __shfl_up_sync(0xffffffffu, v, o);
        if (lane >= o) v += n;
    }
    return v;
}

// Exclusive block scan of one value per thread; also returns the block total.
template <typename T>
__device__ __forceinline__ T block_excl_scan(T v, T *wsum, T &total) {
    const int lane = threadIdx.x & 31;
    const int warp = threadIdx.x >> 5;
    const int nwarps = blockDim.x >> 5;
    T incl = warp_incl_scan(v, lane);
    if (lane == 31) wsum[warp] = incl;
    __syncthreads();
    if (warp == 0) {
        T w = lane < nwarps ? wsum[lane] : T(0);
        w = warp_incl_scan(w, lane);
        if (lane < nwarps) wsum[lane] = w;
    }
    __syncthreads();
    T excl = incl - v + (warp > 0 ? wsum[warp - 1] : T(0));
    total = wsum[nwarps - 1];
    __syncthreads();
    return excl;
}

// The solve of one discharge by one CTA (after grid_dep_wait), shared by
// poisson_kernel, the batched solve and the scatter pass of the in-place
// electron step, whose last CTA solves the next step's field
// (kernels_inplace.cu).  The densities are read through L2 (__ldcg): in the
// scatter pass other CTAs of the same launch have just added to them.
// T: arithmetic type of the scans (double or float); PT: nodes per thread.
template <typename T, int PT>
__device__ __forceinline__ void poisson_body(const float *__restrict__ e_density, const float *__restrict__ i_density,
                                             float *__restrict__ pot_out, float *__restrict__ efield_out,
                                             float pot0_arg, const float *__restrict__ pot0_table,
                                             uint32_t *__restrict__ step_counter, const cudapic_grid &g,
                                             float *__restrict__ zero_a, float *__restrict__ zero_b) {
    constexpr int per_thread = PT;
    extern __shared__ unsigned char smem_raw[];
    T *pot_s = reinterpret_cast<T *>(smem_raw);        // n_g
    __shared__ T wsum[32];
    __shared__ T r_total_s;
    __shared__ float pot0_s;

    const int n = (int)g.n_g;
    const int tid = threadIdx.x;
    for (int k = tid; k < n; k += blockDim.x) {  // next-step accumulators of the driver
        if (zero_a) zero_a[k] = 0.0f;
        if (zero_b) zero_b[k] = 0.0f;
    }
    if (tid == 0) {
        float p0 = pot0_arg;
        if (pot0_table) {
            uint32_t t = *step_counter;
            p0 = pot0_table[t % g.n_t];
            *step_counter = t + 1;
        }
        pot0_s = p0;
    }
    __syncthreads();
    const T pot0 = (T)pot0_s;

    // node-dependent constants in the arithmetic type of the solve
    const T e_charge = sizeof(T) == 8 ? (T)1.60217662e-19 : (T)g.e_charge;
    const T alpha = sizeof(T) == 8 ? (T)(-g.dx * g.dx / 8.85418781e-12) : (T)g.alpha;

    const int first = tid * per_thread;
    T rho[PT];
    T G[PT];
    T local = 0;
#pragma unroll
    for (int j = 0; j < PT; ++j) {
        if (j < per_thread) {
            const int i = first + j;
            T rh = 0, gi = 0;
            if (i < n) {
                const float di = __ldcg(i_density + i), de = __ldcg(e_density + i);
                if (sizeof(T) == 8)
                    rh = e_charge * ((T)di - (T)de);
                else
                    rh = e_charge * (T)(di - de);
                if (i != 0) {
                    T fi = alpha * rh - (i == 1 ? pot0 : T(0));
                    gi = (T)i * fi;
                }
            }
            rho[j] = rh;
            local += gi;
            G[j] = local;
        }
    }
    T tot;
    T off = block_excl_scan<T>(local, wsum, tot);

    T r[PT];
    T R[PT];
    local = 0;
#pragma unroll
    for (int j = 0; j < PT; ++j) {
        if (j < per_thread) {
            const int i = first + j;
            T ri = 0;
            if (i != 0 && i < n - 1) {
                T hi = -(G[j] + off) / ((T)i + T(1));
                ri = hi / (T)i;
            }
            r[j] = ri;
            local += ri;
            R[j] = local;
        }
    }
    off = block_excl_scan<T>(local, wsum, tot);
#pragma unroll
    for (int j = 0; j < PT; ++j) {
        if (j < per_thread && first + j == n - 2) r_total_s = R[j] + off;
    }
    __syncthreads();
    const T r_total = r_total_s;
#pragma unroll
    for (int j = 0; j < PT; ++j) {
        if (j < per_thread) {
            const int i = first + j;
            if (i < n) {
                T p;
                if (i == 0) p = pot0;
                else if (i < n - 1) p = (T)i * (r_total - (R[j] + off) + r[j]);
                else p = T(0);
                pot_s[i] = p;
            }
        }
    }
    __syncthreads();
    const T inv_dx = sizeof(T) == 8 ? (T)(1.0 / g.dx) : (T)g.inv_dx;
    const T half_inv_dx = sizeof(T) == 8 ? (T)(0.5 / g.dx) : (T)g.half_inv_dx;
    const T half_dx_over_eps = sizeof(T) == 8 ? (T)(g.dx / (2.0 * 8.85418781e-12)) : (T)g.half_dx_over_eps;
#pragma unroll
    for (int j = 0; j < PT; ++j) {
        if (j < per_thread) {
            const int i = first + j;
            if (i < n) {
                T pk = pot_s[i];
                T e;
                if (i == 0) e = (pk - pot_s[1]) * inv_dx - rho[j] * half_dx_over_eps;
                else if (i == n - 1) e = (pot_s[n - 2] - pk) * inv_dx + rho[j] * half_dx_over_eps;
                else e = (pot_s[i - 1] - pot_s[i + 1]) * half_inv_dx;
                pot_out[i] = (float)pk;
                efield_out[i] = (float)e;
            }
        }
    }
}

}  // namespace cudapic
