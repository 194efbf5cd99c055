// kernels_poisson.cu -- single-CTA scan-based Poisson solve and field.
//
// Reference: solve_poisson_scan_f32, Rust-CUDA/src/main.rs:408-494 (one
// thread per node, N_G <= 416, f32 block scans) and solve_poisson_dps_flexible,
// :496-564.  The Dirichlet problem pot[i-1] - 2 pot[i] + pot[i+1] = f_i has
// unit tridiagonal coefficients, so the Thomas recurrences collapse to
//     G_i = sum_{j<=i} j f_j,   r_i = -G_i / ((i+1) i),   pot_i = i sum_{j=i}^{N-2} r_j,
// i.e. two inclusive prefix sums (C/eduPIC.cc:461-494 is the sequential
// Thomas form of the same system).
//
// B200 design: one CTA of up to 1024 threads, each thread owning
// ceil(N_G / blockDim) consecutive nodes (N_G up to 16384), warp-shuffle
// scans plus one shared-memory pass over the warp totals.  The sums run in
// FP64 by default: in f32 the cancellation in R_total - R_i grows with N_G
// (relative L2 error ~4e-3 at N_G = 4096 against the FP64 Thomas solve),
// in FP64 it is at the f32 output rounding.  CUDAPIC_FLAG_POISSON_F32_SCAN
// selects the reference's f32 arithmetic.  Latency-bound: a few us.
//
// The driver variant reads pot0 from a device table indexed by a device
// step counter (so that one captured CUDA graph serves every RF phase) and
// advances the counter.
#include "batch_internal.h"
#include "common.cuh"
#include "internal.h"
#include "poisson.cuh"

namespace cudapic {

template <typename T, int PT>
__global__ void __launch_bounds__(POIS_MAX_THREADS)
    poisson_kernel(const float *__restrict__ e_density, const float *__restrict__ i_density,
                   float *__restrict__ pot_out, float *__restrict__ efield_out, float pot0_arg,
                   const float *__restrict__ pot0_table, uint32_t *__restrict__ step_counter,
                   const cudapic_grid g, float *__restrict__ zero_a, float *__restrict__ zero_b) {
    grid_dep_wait();
    poisson_body<T, PT>(e_density, i_density, pot_out, efield_out, pot0_arg, pot0_table, step_counter, g, zero_a,
                        zero_b);
}

// solve_poisson_dps_flexible: the same closed form with runtime n, dx and
// both Dirichlet values (used by the reference's Hakim convergence test,
// Rust-CUDA/src/main.rs:1895-1981).  FP64 sums.
template <int PT>
__global__ void __launch_bounds__(POIS_MAX_THREADS)
    poisson_flexible_kernel(const float *__restrict__ source, float *__restrict__ pot_out, int n,
                            double psi_left, double psi_right, double dx) {
    constexpr int per_thread = PT;
    __shared__ double wsum[32];
    __shared__ double r_total_s;
    const int tid = threadIdx.x;
    const int first = tid * per_thread;
    double G[PT];
    double local = 0;
#pragma unroll
    for (int j = 0; j < PT; ++j) {
        if (j < per_thread) {
            const int i = first + j;
            double gi = 0;
            if (i != 0 && i < n) {
                double fi = dx * dx * (double)source[i];
                if (i == 1) fi -= psi_left;
                if (i == n - 2) fi -= psi_right;
                gi = (double)i * fi;
            }
            local += gi;
            G[j] = local;
        }
    }
    double tot;
    double off = block_excl_scan<double>(local, wsum, tot);
    double r[PT], R[PT];
    local = 0;
#pragma unroll
    for (int j = 0; j < PT; ++j) {
        if (j < per_thread) {
            const int i = first + j;
            double ri = 0;
            if (i != 0 && i < n - 1) ri = (-(G[j] + off) / ((double)i + 1.0)) / (double)i;
            r[j] = ri;
            local += ri;
            R[j] = local;
        }
    }
    off = block_excl_scan<double>(local, wsum, tot);
#pragma unroll
    for (int j = 0; j < PT; ++j)
        if (j < per_thread && first + j == n - 2) r_total_s = R[j] + off;
    __syncthreads();
    const double r_total = r_total_s;
#pragma unroll
    for (int j = 0; j < PT; ++j) {
        if (j < per_thread) {
            const int i = first + j;
            if (i < n) {
                double p;
                if (i == 0) p = psi_left;
                else if (i < n - 1) p = (double)i * (r_total - (R[j] + off) + r[j]);
                else p = psi_right;
                pot_out[i] = (float)p;
            }
        }
    }
}

// Threads and nodes per thread (a power of two) for n nodes.
void poisson_shape(uint32_t n_g, int &threads, int &per_thread) {
    per_thread = 1;
    while ((uint32_t)per_thread * POIS_MAX_THREADS < n_g) per_thread *= 2;
    threads = (int)((((n_g + per_thread - 1) / per_thread) + 31) / 32 * 32);
}

template <typename T, int PT>
int launch_poisson_t(const float *e_density, const float *i_density, float *pot, float *efield, float pot0,
                     const float *pot0_table, uint32_t *step_counter, const cudapic_grid &g, int threads,
                     cudaStream_t stream, float *zero_a, float *zero_b) {
    size_t smem = (size_t)g.n_g * sizeof(T);
    auto kern = poisson_kernel<T, PT>;
    if (smem > 48 * 1024)
        CUDAPIC_CHECK(check_cuda(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem),
                                 "cudaFuncSetAttribute(poisson)"));
    return launch_kernel("solve_poisson_scan", kern, dim3(1), dim3(threads), smem, stream, e_density, i_density, pot,
                         efield, pot0, pot0_table, step_counter, g, zero_a, zero_b);
}

template <typename T>
int launch_poisson_pt(const float *e_density, const float *i_density, float *pot, float *efield, float pot0,
                      const float *pot0_table, uint32_t *step_counter, const cudapic_grid &g,
                      cudaStream_t stream, float *zero_a, float *zero_b) {
    int threads, pt;
    poisson_shape(g.n_g, threads, pt);
    switch (pt) {
    case 1: return launch_poisson_t<T, 1>(e_density, i_density, pot, efield, pot0, pot0_table, step_counter, g, threads, stream, zero_a, zero_b);
    case 2: return launch_poisson_t<T, 2>(e_density, i_density, pot, efield, pot0, pot0_table, step_counter, g, threads, stream, zero_a, zero_b);
    case 4: return launch_poisson_t<T, 4>(e_density, i_density, pot, efield, pot0, pot0_table, step_counter, g, threads, stream, zero_a, zero_b);
    case 8: return launch_poisson_t<T, 8>(e_density, i_density, pot, efield, pot0, pot0_table, step_counter, g, threads, stream, zero_a, zero_b);
    default: return launch_poisson_t<T, 16>(e_density, i_density, pot, efield, pot0, pot0_table, step_counter, g, threads, stream, zero_a, zero_b);
    }
}

// Adjoint of the solve and field (the sensitivity path, FP64 sums): from the
// field adjoint eb, the potential adjoint pb (the transposed differences),
// lam = T^-1 pb with the same two-scan closed form (T = tridiag(1, -2, 1) is
// symmetric), the density adjoints neb = -e rho_bar and
// nib_acc = (reset_acc ? 0 : nib_acc) + e rho_bar (rho_bar = alpha lam inside,
// the one-sided corrections at the electrodes), and
// vbar += cosv (pb_0 - lam_1), pot0 = V cosv entering f_1 with a minus sign.
// One CTA; eb is cleared for the next step.
template <int PT>
__global__ void __launch_bounds__(POIS_MAX_THREADS)
    poisson_adjoint_kernel(double *__restrict__ eb, double *__restrict__ neb, double *__restrict__ nib_acc,
                           int reset_acc, double cosv, double *__restrict__ vbar, const cudapic_grid g) {
    extern __shared__ unsigned char smem_raw[];
    double *eb_s = reinterpret_cast<double *>(smem_raw);  // n
    __shared__ double wsum[32];
    __shared__ double r_total_s, lam1_s;
    const int n = (int)g.n_g;
    const int tid = threadIdx.x;
    for (int k = tid; k < n; k += blockDim.x) {
        eb_s[k] = eb[k];
        eb[k] = 0.0;
    }
    __syncthreads();
    const double inv_dx = 1.0 / g.dx, half_inv_dx = 0.5 / g.dx;
    const double hdx_eps = g.dx / (2.0 * 8.85418781e-12);
    const double alpha = -g.dx * g.dx / 8.85418781e-12;
    const double e_charge = 1.60217662e-19;
    const int first = tid * PT;
    double G[PT], r[PT], R[PT];
    double local = 0.0;
#pragma unroll
    for (int j = 0; j < PT; ++j) {
        const int i = first + j;
        double gi = 0.0;
        if (i >= 1 && i <= n - 2) {
            double p = 0.0;
            if (i == 1) p -= eb_s[0] * inv_dx;
            if (i == n - 2) p += eb_s[n - 1] * inv_dx;
            if (i + 1 <= n - 2) p += eb_s[i + 1] * half_inv_dx;
            if (i - 1 >= 1) p -= eb_s[i - 1] * half_inv_dx;
            gi = (double)i * p;
        }
        local += gi;
        G[j] = local;
    }
    double tot;
    double off = block_excl_scan<double>(local, wsum, tot);
    local = 0.0;
#pragma unroll
    for (int j = 0; j < PT; ++j) {
        const int i = first + j;
        double ri = 0.0;
        if (i >= 1 && i <= n - 2) ri = (-(G[j] + off) / ((double)i + 1.0)) / (double)i;
        r[j] = ri;
        local += ri;
        R[j] = local;
    }
    off = block_excl_scan<double>(local, wsum, tot);
#pragma unroll
    for (int j = 0; j < PT; ++j)
        if (first + j == n - 2) r_total_s = R[j] + off;
    __syncthreads();
    const double r_total = r_total_s;
#pragma unroll
    for (int j = 0; j < PT; ++j) {
        const int i = first + j;
        if (i >= n) continue;
        double rb;
        if (i == 0) {
            rb = -eb_s[0] * hdx_eps;
        } else if (i == n - 1) {
            rb = eb_s[n - 1] * hdx_eps;
        } else {
            const double lam = (double)i * (r_total - (R[j] + off) + r[j]);
            if (i == 1) lam1_s = lam;
            rb = alpha * lam;
        }
        neb[i] = -e_charge * rb;
        nib_acc[i] = (reset_acc ? 0.0 : nib_acc[i]) + e_charge * rb;
    }
    __syncthreads();
    if (tid == 0) {
        const double pb0 = eb_s[0] * inv_dx + (n > 2 ? eb_s[1] * half_inv_dx : 0.0);
        *vbar += cosv * (pb0 - lam1_s);
    }
}

template <int PT>
int launch_poisson_adjoint_t(double *eb, double *neb, double *nib_acc, int reset_acc, double cosv, double *vbar,
                             const cudapic_grid &g, int threads, cudaStream_t stream) {
    const size_t smem = (size_t)g.n_g * sizeof(double);
    auto kern = poisson_adjoint_kernel<PT>;
    if (smem > 48 * 1024)
        CUDAPIC_CHECK(check_cuda(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem),
                                 "cudaFuncSetAttribute(poisson_adjoint)"));
    return launch_kernel("poisson_adjoint", kern, dim3(1), dim3(threads), smem, stream, eb, neb, nib_acc, reset_acc,
                         cosv, vbar, g);
}

int launch_poisson_adjoint(double *eb, double *neb, double *nib_acc, int reset_acc, double cosv, double *vbar,
                           const cudapic_grid &g, cudaStream_t stream) {
    if (g.n_g < 3 || g.n_g > (uint32_t)(POIS_MAX_THREADS * POIS_MAX_PER_THREAD))
        return fail(CUDAPIC_ERR_ARG, "poisson_adjoint: n_g outside 3..16384");
    int threads, pt;
    poisson_shape(g.n_g, threads, pt);
    switch (pt) {
    case 1: return launch_poisson_adjoint_t<1>(eb, neb, nib_acc, reset_acc, cosv, vbar, g, threads, stream);
    case 2: return launch_poisson_adjoint_t<2>(eb, neb, nib_acc, reset_acc, cosv, vbar, g, threads, stream);
    case 4: return launch_poisson_adjoint_t<4>(eb, neb, nib_acc, reset_acc, cosv, vbar, g, threads, stream);
    case 8: return launch_poisson_adjoint_t<8>(eb, neb, nib_acc, reset_acc, cosv, vbar, g, threads, stream);
    default: return launch_poisson_adjoint_t<16>(eb, neb, nib_acc, reset_acc, cosv, vbar, g, threads, stream);
    }
}

// The solve and field in FP64 in and out (the all-FP64 twin, fp64.cu):
// dens_e / dens_i are the CIC node sums before the boundary doubling;
// pot0 = pot0_table[*step % n_t], *step advanced.  With measurement
// (non-null sums): cumul_e += n_e, cumul_i += n_i (ion steps), pot_sum += pot.
template <int PT>
__global__ void __launch_bounds__(POIS_MAX_THREADS)
    poisson_f64_kernel(const double *__restrict__ dens_e, const double *__restrict__ dens_i, double *__restrict__ pot_out,
                       double *__restrict__ efield_out, const double *__restrict__ pot0_table,
                       uint32_t *__restrict__ step, int ion_step, double *__restrict__ cumul_e,
                       double *__restrict__ cumul_i, double *__restrict__ pot_sum, const cudapic_grid g) {
    extern __shared__ unsigned char smem_raw[];
    double *pot_s = reinterpret_cast<double *>(smem_raw);  // n
    __shared__ double wsum[32];
    __shared__ double r_total_s, pot0_s;
    const int n = (int)g.n_g;
    const int tid = threadIdx.x;
    if (tid == 0) {
        const uint32_t t = *step;
        pot0_s = pot0_table[t % g.n_t];
        *step = t + 1;
    }
    __syncthreads();
    const double pot0 = pot0_s;
    const double e_charge = 1.60217662e-19;
    const double alpha = -g.dx * g.dx / 8.85418781e-12;
    const int first = tid * PT;
    double rho[PT], G[PT], r[PT], R[PT];
    double local = 0.0;
#pragma unroll
    for (int j = 0; j < PT; ++j) {
        const int i = first + j;
        double rh = 0.0, gi = 0.0;
        if (i < n) {
            const double b = (i == 0 || i == n - 1) ? 2.0 : 1.0;
            const double ne = dens_e[i] * b, ni = dens_i[i] * b;
            if (cumul_e) cumul_e[i] += ne;
            if (cumul_i && ion_step) cumul_i[i] += ni;
            rh = e_charge * (ni - ne);
            if (i != 0) gi = (double)i * (alpha * rh - (i == 1 ? pot0 : 0.0));
        }
        rho[j] = rh;
        local += gi;
        G[j] = local;
    }
    double tot;
    double off = block_excl_scan<double>(local, wsum, tot);
    local = 0.0;
#pragma unroll
    for (int j = 0; j < PT; ++j) {
        const int i = first + j;
        double ri = 0.0;
        if (i != 0 && i < n - 1) ri = (-(G[j] + off) / ((double)i + 1.0)) / (double)i;
        r[j] = ri;
        local += ri;
        R[j] = local;
    }
    off = block_excl_scan<double>(local, wsum, tot);
#pragma unroll
    for (int j = 0; j < PT; ++j)
        if (first + j == n - 2) r_total_s = R[j] + off;
    __syncthreads();
    const double r_total = r_total_s;
#pragma unroll
    for (int j = 0; j < PT; ++j) {
        const int i = first + j;
        if (i < n) pot_s[i] = i == 0 ? pot0 : (i < n - 1 ? (double)i * (r_total - (R[j] + off) + r[j]) : 0.0);
    }
    __syncthreads();
    const double inv_dx = 1.0 / g.dx, half_inv_dx = 0.5 / g.dx, hdx_eps = g.dx / (2.0 * 8.85418781e-12);
#pragma unroll
    for (int j = 0; j < PT; ++j) {
        const int i = first + j;
        if (i >= n) continue;
        const double pk = pot_s[i];
        double e;
        if (i == 0) e = (pk - pot_s[1]) * inv_dx - rho[j] * hdx_eps;
        else if (i == n - 1) e = (pot_s[n - 2] - pk) * inv_dx + rho[j] * hdx_eps;
        else e = (pot_s[i - 1] - pot_s[i + 1]) * half_inv_dx;
        pot_out[i] = pk;
        efield_out[i] = e;
        if (pot_sum) pot_sum[i] += pk;
    }
}

template <int PT>
int launch_poisson_f64_t(const double *dens_e, const double *dens_i, double *pot, double *efield,
                         const double *pot0_table, uint32_t *step, int ion_step, double *cumul_e, double *cumul_i,
                         double *pot_sum, const cudapic_grid &g, int threads, cudaStream_t stream) {
    const size_t smem = (size_t)g.n_g * sizeof(double);
    auto kern = poisson_f64_kernel<PT>;
    if (smem > 48 * 1024)
        CUDAPIC_CHECK(check_cuda(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem),
                                 "cudaFuncSetAttribute(poisson_f64)"));
    return launch_kernel("poisson_f64", kern, dim3(1), dim3(threads), smem, stream, dens_e, dens_i, pot, efield,
                         pot0_table, step, ion_step, cumul_e, cumul_i, pot_sum, g);
}

int launch_poisson_f64(const double *dens_e, const double *dens_i, double *pot, double *efield,
                       const double *pot0_table, uint32_t *step, int ion_step, double *cumul_e, double *cumul_i,
                       double *pot_sum, const cudapic_grid &g, cudaStream_t stream) {
    if (g.n_g < 3 || g.n_g > (uint32_t)(POIS_MAX_THREADS * POIS_MAX_PER_THREAD))
        return fail(CUDAPIC_ERR_ARG, "poisson_f64: n_g outside 3..16384");
    int threads, pt;
    poisson_shape(g.n_g, threads, pt);
    switch (pt) {
    case 1: return launch_poisson_f64_t<1>(dens_e, dens_i, pot, efield, pot0_table, step, ion_step, cumul_e, cumul_i, pot_sum, g, threads, stream);
    case 2: return launch_poisson_f64_t<2>(dens_e, dens_i, pot, efield, pot0_table, step, ion_step, cumul_e, cumul_i, pot_sum, g, threads, stream);
    case 4: return launch_poisson_f64_t<4>(dens_e, dens_i, pot, efield, pot0_table, step, ion_step, cumul_e, cumul_i, pot_sum, g, threads, stream);
    case 8: return launch_poisson_f64_t<8>(dens_e, dens_i, pot, efield, pot0_table, step, ion_step, cumul_e, cumul_i, pot_sum, g, threads, stream);
    default: return launch_poisson_f64_t<16>(dens_e, dens_i, pot, efield, pot0_table, step, ion_step, cumul_e, cumul_i, pot_sum, g, threads, stream);
    }
}

int launch_poisson(const float *e_density, const float *i_density, float *pot, float *efield, float pot0,
                   const float *pot0_table, uint32_t *step_counter, const cudapic_grid &g,
                   cudaStream_t stream, float *zero_a, float *zero_b) {
    if (g.n_g > (uint32_t)(POIS_MAX_THREADS * POIS_MAX_PER_THREAD))
        return fail(CUDAPIC_ERR_ARG, "solve_poisson: n_g > 16384");
    if (g.flags & CUDAPIC_FLAG_POISSON_F32_SCAN)
        return launch_poisson_pt<float>(e_density, i_density, pot, efield, pot0, pot0_table, step_counter, g, stream, zero_a, zero_b);
    return launch_poisson_pt<double>(e_density, i_density, pot, efield, pot0, pot0_table, step_counter, g, stream, zero_a, zero_b);
}

// Batched solve: CTA d solves discharge d of the batch (the driver variant
// above, with the discharge's own step counter and RF table), writes its
// clamped particle counts for the batched particle kernels and, when
// measuring, adds the densities it read to the time averages
// (accumulate_density, Rust-CUDA/src/main.rs:1294-1299) and, with XT
// diagnostics, the step's grid quantities to their XT column.
template <typename T, int PT>
__global__ void __launch_bounds__(POIS_MAX_THREADS)
    batch_poisson_kernel(const BatchDisc *__restrict__ desc, uint32_t *__restrict__ counts, uint32_t D, int e_read,
                         int i_read, int ion_step, int measure) {
    __shared__ cudapic_grid s_g;
    const BatchDisc &dd = desc[blockIdx.x];
    if (threadIdx.x == 0) s_g = dd.g;
    __syncthreads();
    grid_dep_wait();
    uint32_t *ctr = dd.counters;
    if (threadIdx.x == 0) {
        counts[blockIdx.x] = load_count(ctr + 0, s_g.capacity, s_g.dev_err);
        counts[D + blockIdx.x] = load_count(ctr + 1, s_g.capacity, s_g.dev_err);
    }
    const float *e_dens = dd.e_dens[e_read];
    const float *i_dens = dd.i_dens[i_read];
    if (measure) {
        for (uint32_t k = threadIdx.x; k < s_g.n_g; k += blockDim.x) {
            dd.cumul_e[k] += (double)e_dens[k];
            if (ion_step) dd.cumul_i[k] += (double)i_dens[k];
        }
    }
    poisson_body<T, PT>(e_dens, i_dens, dd.pot, dd.efield, 0.0f, dd.pot0_table, ctr + 3, s_g, dd.e_dens[e_read ^ 1],
                        ion_step ? dd.i_dens[i_read ^ 1] : nullptr);
    if (measure && dd.xt) {  // XT grid quantities of the step (C/eduPIC.cc:705-715)
        __syncthreads();
        const uint32_t t = (*(volatile const uint32_t *)(ctr + 3) + s_g.n_t - 1u) % s_g.n_t;
        const uint32_t col = t / XT_BIN;
        const size_t plane = (size_t)s_g.n_g * dd.n_xt;
        for (uint32_t k = threadIdx.x; k < s_g.n_g; k += blockDim.x) {
            const size_t at = (size_t)k * dd.n_xt + col;
            dd.xt[XT_POT * plane + at] += (double)dd.pot[k];
            dd.xt[XT_EFIELD * plane + at] += (double)dd.efield[k];
            dd.xt[XT_NE * plane + at] += (double)e_dens[k];
            dd.xt[XT_NI * plane + at] += (double)i_dens[k];
        }
    }
}

template <typename T, int PT>
int launch_batch_poisson_t(const BatchDisc *desc, uint32_t *counts, uint32_t D, uint32_t max_n_g, int threads,
                           int e_read, int i_read, int ion_step, int measure, cudaStream_t stream) {
    const size_t smem = (size_t)max_n_g * sizeof(T);
    auto kern = batch_poisson_kernel<T, PT>;
    if (smem > 48 * 1024)
        CUDAPIC_CHECK(check_cuda(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem),
                                 "cudaFuncSetAttribute(batch poisson)"));
    return launch_kernel("batch_solve_poisson", kern, dim3(D), dim3(threads), smem, stream, desc, counts, D, e_read,
                         i_read, ion_step, measure);
}

template <typename T>
int launch_batch_poisson_pt(const BatchDisc *desc, uint32_t *counts, uint32_t D, uint32_t max_n_g, int e_read,
                            int i_read, int ion_step, int measure, cudaStream_t stream) {
    int threads, pt;
    poisson_shape(max_n_g, threads, pt);
    switch (pt) {
    case 1: return launch_batch_poisson_t<T, 1>(desc, counts, D, max_n_g, threads, e_read, i_read, ion_step, measure, stream);
    case 2: return launch_batch_poisson_t<T, 2>(desc, counts, D, max_n_g, threads, e_read, i_read, ion_step, measure, stream);
    case 4: return launch_batch_poisson_t<T, 4>(desc, counts, D, max_n_g, threads, e_read, i_read, ion_step, measure, stream);
    case 8: return launch_batch_poisson_t<T, 8>(desc, counts, D, max_n_g, threads, e_read, i_read, ion_step, measure, stream);
    default: return launch_batch_poisson_t<T, 16>(desc, counts, D, max_n_g, threads, e_read, i_read, ion_step, measure, stream);
    }
}

int launch_batch_poisson(const BatchDisc *desc, uint32_t *counts, uint32_t D, uint32_t max_n_g, uint32_t flags,
                         int e_read, int i_read, int ion_step, int measure, cudaStream_t stream) {
    if (max_n_g > (uint32_t)(POIS_MAX_THREADS * POIS_MAX_PER_THREAD))
        return fail(CUDAPIC_ERR_ARG, "batch: n_g > 16384");
    if (flags & CUDAPIC_FLAG_POISSON_F32_SCAN)
        return launch_batch_poisson_pt<float>(desc, counts, D, max_n_g, e_read, i_read, ion_step, measure, stream);
    return launch_batch_poisson_pt<double>(desc, counts, D, max_n_g, e_read, i_read, ion_step, measure, stream);
}

}  // namespace cudapic

using namespace cudapic;

extern "C" int cudapic_solve_poisson_scan_f32(const float *e_density, const float *i_density, float *pot,
                                              float *efield, float pot0, const cudapic_grid *grid,
                                              cudapic_stream_t stream) {
    CUDAPIC_CHECK(validate_grid(grid));
    CUDAPIC_REQUIRE(e_density && i_density && pot && efield, "solve_poisson_scan_f32: null pointer");
    return launch_poisson(e_density, i_density, pot, efield, pot0, nullptr, nullptr, *grid,
                          (cudaStream_t)stream);
}

extern "C" int cudapic_solve_poisson_dps_flexible(const float *source, float *pot, uint32_t n, float psi_left,
                                                  float psi_right, float dx, cudapic_stream_t stream) {
    CUDAPIC_REQUIRE(source && pot, "solve_poisson_dps_flexible: null pointer");
    CUDAPIC_REQUIRE(n >= 3 && n <= (uint32_t)(POIS_MAX_THREADS * POIS_MAX_PER_THREAD),
                    "solve_poisson_dps_flexible: n must be in [3, 16384]");
    int threads, pt;
    poisson_shape(n, threads, pt);
    cudaStream_t st = (cudaStream_t)stream;
    const double l = psi_left, r = psi_right, h = dx;
    switch (pt) {
    case 1: poisson_flexible_kernel<1><<<1, threads, 0, st>>>(source, pot, (int)n, l, r, h); break;
    case 2: poisson_flexible_kernel<2><<<1, threads, 0, st>>>(source, pot, (int)n, l, r, h); break;
    case 4: poisson_flexible_kernel<4><<<1, threads, 0, st>>>(source, pot, (int)n, l, r, h); break;
    case 8: poisson_flexible_kernel<8><<<1, threads, 0, st>>>(source, pot, (int)n, l, r, h); break;
    default: poisson_flexible_kernel<16><<<1, threads, 0, st>>>(source, pot, (int)n, l, r, h); break;
    }
    return check_launch("solve_poisson_dps_flexible");
}
