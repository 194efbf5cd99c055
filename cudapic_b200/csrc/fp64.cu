// fp64.cu -- an all-FP64 twin of a discharge for the precision study: the
// reference's step (Rust-CUDA/src/main.rs:1725-1808) with every particle
// coordinate, field, density, collision test and scattering in double
// (cudapic_fp64_* in include/cudapic.h).
//
// The launch sequence is the reference's: deposit (CIC, FP64 shared then
// global atomics), Poisson (FP64 in and out), compacting push (warp-aggregated
// slot claims), electron collisions with spawns, ion collisions, with the
// RNG stream of the slot a particle occupies (the reference's per-slot
// semantics).  Transcendentals are CUDA's double functions; the RNG draws
// and the cross-section tables are the reference's (23-bit uniforms, f32
// table entries widened to double).  Measurement: time sums of the node
// densities and potential, the EEPF of C/eduPIC.cc's central 10 % (the
// driver's definition: position after the step, the x velocity moved back
// half a kick), the <j E> power summed per electron at the push.  One ion
// cycle (N_SUB steps) is captured in a CUDA graph; the RF phase is a device
// step counter.  Not a hot path: plain grid-stride kernels.
#include <cuda_runtime.h>

#include <cmath>
#include <cstring>
#include <vector>

#include "common.cuh"
#include "internal.h"
#include "rng.cuh"
#include "state_impl.h"

namespace cudapic {

namespace {

constexpr int F64_THREADS = 256;
constexpr int F64_PER_SM = 4;
constexpr uint32_t F64_MAX_NG = 4096;

// counters block
enum : int { K_NE = 0, K_NI, K_ALIVE, K_STEP, K_ERR, K_ALIVE_I, K_COUNT };

struct D64 {
    uint32_t n_g, cap, n_t, n_sub;
    double dx, inv_dx, gap, dt_e, dt_i, fe, fi, wf, f1, f2, hme, hmu, nr, min_x, max_x, kick, me, qe;
};

struct P64 {
    double *x, *vx, *vy, *vz;
};

__device__ __forceinline__ double draw(Xoshiro128p &rs) { return (double)rs.uniform(); }

// Box-Muller as rng_next_three_normal (Rust-CUDA/src/main.rs:908-969), in double.
__device__ __forceinline__ void three_normal(Xoshiro128p &rs, double sigma, double &a, double &b, double &c) {
    const double u1 = fmax(draw(rs), 1e-9), u2 = fmax(draw(rs), 1e-9);
    const double u3 = fmax(draw(rs), 1e-9), u4 = fmax(draw(rs), 1e-9);
    const double r1 = sqrt(-2.0 * log(u1)), r2 = sqrt(-2.0 * log(u3));
    double s1, c1;
    sincos(6.283185307179586 * u2, &s1, &c1);
    a = r1 * c1 * sigma;
    b = r1 * s1 * sigma;
    c = r2 * cos(6.283185307179586 * u4) * sigma;
}

__device__ __forceinline__ uint32_t index_of(double energy) {
    double t = energy / 0.001 + 0.5;
    if (t > (double)(CS_RANGES - 1)) t = (double)(CS_RANGES - 1);
    return (uint32_t)t;
}

__device__ __forceinline__ int cell64(double pos, uint32_t n_g) {
    int p = (int)pos;
    if (!(pos >= 0.0)) p = 0;
    if (p > (int)n_g - 2) p = (int)n_g - 2;
    return p;
}

// Sines and cosines of the Euler angles of g from their algebraic forms.
__device__ __forceinline__ void euler64(double gx, double gy, double gz, double &st, double &ct, double &sp,
                                        double &cp) {
    const double r = sqrt(gy * gy + gz * gz);
    const double gn = sqrt(gx * gx + gy * gy + gz * gz);
    if (gx == 0.0) {
        st = 1.0;
        ct = 0.0;
    } else {
        st = r / gn;
        ct = gx / gn;
    }
    if (gy == 0.0) {
        sp = gz > 0.0 ? 1.0 : -1.0;
        cp = 0.0;
    } else {
        sp = gz / r;
        cp = gy / r;
    }
}

__device__ __forceinline__ void rot64(double g, double sc, double cc, double se, double ce, double st, double ct,
                                      double sp, double cp, double &ox, double &oy, double &oz) {
    ox = g * (ct * cc - st * sc * ce);
    oy = g * (st * cp * cc + ct * cp * sc * ce - sp * sc * se);
    oz = g * (st * sp * cc + ct * sp * sc * ce + cp * sc * se);
}

__device__ __forceinline__ bool claim(uint32_t *counter, uint32_t cap, uint32_t &slot) {
    slot = atomicAdd(counter, 1u);
    return slot < cap;
}

__device__ __forceinline__ double block_sum(double v, double *red) {
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    if (lane == 0) red[warp] = v;
    __syncthreads();
    double s = 0.0;
    if (threadIdx.x == 0)
        for (int w = 0; w < (int)(blockDim.x >> 5); ++w) s += red[w];
    return s;
}

// CIC weights (Rust-CUDA/src/main.rs:356-406) summed in FP64; boundary nodes
// are doubled by the Poisson kernel.
__global__ void __launch_bounds__(F64_THREADS)
    f64_deposit_kernel(const double *__restrict__ x, const uint32_t *__restrict__ n_ptr, double *__restrict__ dens,
                       const D64 k) {
    extern __shared__ double h[];
    for (uint32_t j = threadIdx.x; j < k.n_g; j += blockDim.x) h[j] = 0.0;
    __syncthreads();
    const uint32_t n = min(*n_ptr, k.cap);
    for (uint32_t p = blockIdx.x * blockDim.x + threadIdx.x; p < n; p += gridDim.x * blockDim.x) {
        const double pos = x[p] * k.inv_dx;
        const int c = cell64(pos, k.n_g);
        const double rem = pos - (double)c;
        atomicAdd(&h[c], (1.0 - rem) * k.wf);
        atomicAdd(&h[c + 1], rem * k.wf);
    }
    __syncthreads();
    for (uint32_t j = threadIdx.x; j < k.n_g; j += blockDim.x)
        if (h[j] != 0.0) atomicAdd(&dens[j], h[j]);
}

// move_and_compact (Rust-CUDA/src/main.rs:566-678) in FP64: survivors to the
// other side at warp-claimed slots; power (may be null) += sum of the
// electrons' (v + f E/2) E.
__global__ void __launch_bounds__(F64_THREADS)
    f64_push_kernel(P64 s, P64 d, uint32_t *__restrict__ alive, const uint32_t *__restrict__ n_ptr,
                    const double *__restrict__ E, double f, double dt, double *__restrict__ power, const D64 k) {
    __shared__ double red[F64_THREADS / 32];
    const uint32_t n = min(*n_ptr, k.cap);
    const int lane = threadIdx.x & 31;
    double acc = 0.0;
    const uint32_t stride = gridDim.x * blockDim.x;
    const uint32_t rounds = (n + stride - 1) / stride;  // whole-warp iterations for the ballot
    for (uint32_t r = 0; r < rounds; ++r) {
        const uint32_t p = r * stride + blockIdx.x * blockDim.x + threadIdx.x;
        const bool valid = p < n;
        double x1 = 0.0, v1 = 0.0, vy = 0.0, vz = 0.0;
        bool keep = false;
        if (valid) {
            const double x = s.x[p], v = s.vx[p];
            const double pos = x * k.inv_dx;
            const int c = cell64(pos, k.n_g);
            const double c2 = pos - (double)c;
            const double ex = (1.0 - c2) * E[c] + c2 * E[c + 1];
            if (power) acc += (v + 0.5 * f * ex) * ex;
            v1 = v + f * ex;
            x1 = x + v1 * dt;
            keep = x1 >= 0.0 && x1 <= k.gap;
            vy = s.vy[p];
            vz = s.vz[p];
        }
        const unsigned m = __ballot_sync(0xffffffffu, keep);
        uint32_t base = 0;
        if (lane == 0 && m) base = atomicAdd(alive, (uint32_t)__popc(m));
        base = __shfl_sync(0xffffffffu, base, 0);
        if (keep) {
            const uint32_t slot = base + __popc(m & lanemask_lt());
            if (slot < k.cap) {
                d.x[slot] = x1;
                d.vx[slot] = v1;
                d.vy[slot] = vy;
                d.vz[slot] = vz;
            }
        }
    }
    if (power) {
        const double sm = block_sum(acc, red);
        if (threadIdx.x == 0 && sm != 0.0) atomicAdd(power, sm);
    }
}

// dst = min(src, cap); src = dst or 0 (the reference's counter copies).
__global__ void f64_count_kernel(uint32_t *__restrict__ cnt, int dst, int src, int reset_to_dst, uint32_t cap,
                                 uint32_t err_bit) {
    if (threadIdx.x == 0) {
        uint32_t v = cnt[src];
        if (v > cap) {
            atomicOr(&cnt[K_ERR], err_bit);
            v = cap;
        }
        cnt[dst] = v;
        cnt[src] = reset_to_dst ? v : 0u;
    }
}

// check_collisions_e + collision_e (Rust-CUDA/src/main.rs:971-1165) in FP64.
__global__ void __launch_bounds__(F64_THREADS)
    f64_collide_e_kernel(P64 e, uint32_t *__restrict__ rng0, uint32_t *__restrict__ rng1, uint32_t *__restrict__ rng2,
                         uint32_t *__restrict__ rng3, uint32_t *__restrict__ cnt, P64 ion,
                         const float *__restrict__ sig, const float *__restrict__ cs, const D64 k) {
    const uint32_t n = min(cnt[K_NE], k.cap);
    for (uint32_t p = blockIdx.x * blockDim.x + threadIdx.x; p < n; p += gridDim.x * blockDim.x) {
        Xoshiro128p rs{rng0[p], rng1[p], rng2[p], rng3[p]};
        const double vx = e.vx[p], vy = e.vy[p], vz = e.vz[p];
        const double v2 = vx * vx + vy * vy + vz * vz;
        const uint32_t idx = index_of(k.hme * v2);
        const double nu = (double)__ldg(sig + idx) * sqrt(v2);
        const double u = draw(rs);
        if (u < 1.0 - exp(-nu * k.dt_e)) {
            const double t0 = (double)__ldg(cs + idx);
            const double t1 = t0 + (double)__ldg(cs + CS_RANGES + idx);
            const double t2 = t1 + (double)__ldg(cs + 2 * CS_RANGES + idx);
            double gm = sqrt(v2);
            double st, ct, sp, cp;
            euler64(vx, vy, vz, st, ct, sp, cp);
            const double rnd = draw(rs);
            double chi_s, chi_c, se, ce;
            if (rnd < t0 / t2 || rnd < t1 / t2) {
                if (!(rnd < t0 / t2)) {  // excitation, 11.5 eV
                    const double en = fabs(0.5 * k.me * gm * gm - 11.5 * k.qe);
                    gm = sqrt(2.0 * en / k.me);
                }
                chi_c = 1.0 - 2.0 * draw(rs);
                chi_s = sqrt(fmax(0.0, (1.0 - chi_c) * (1.0 + chi_c)));
                sincos(6.283185307179586 * draw(rs), &se, &ce);
            } else {  // ionization, 15.8 eV, energy sharing 10 tan(u atan(E / 20 eV)) eV
                const double en = fabs(0.5 * k.me * gm * gm - 15.8 * k.qe);
                const double e_new = 10.0 * tan(draw(rs) * atan(en / k.qe / 20.0)) * k.qe;
                const double e_orig = fabs(en - e_new);
                gm = sqrt(2.0 * e_orig / k.me);
                const double g_new = sqrt(2.0 * e_new / k.me);
                sincos(6.283185307179586 * draw(rs), &se, &ce);
                const double c2 = sqrt(e_new / en), s2 = sqrt(fmax(0.0, (1.0 - c2) * (1.0 + c2)));
                double nx, ny, nz;
                rot64(g_new, s2, c2, -se, -ce, st, ct, sp, cp, nx, ny, nz);  // eta + pi
                uint32_t slot;
                if (claim(&cnt[K_ALIVE], k.cap, slot)) {
                    e.x[slot] = e.x[p];
                    e.vx[slot] = k.f1 * vx + k.f2 * nx;
                    e.vy[slot] = k.f1 * vy + k.f2 * ny;
                    e.vz[slot] = k.f1 * vz + k.f2 * nz;
                } else {
                    atomicOr(&cnt[K_ERR], CUDAPIC_DEVERR_SPAWN_E);
                }
                double a, b, c;
                three_normal(rs, k.nr, a, b, c);
                if (claim(&cnt[K_NI], k.cap, slot)) {
                    ion.x[slot] = e.x[p];
                    ion.vx[slot] = a;
                    ion.vy[slot] = b;
                    ion.vz[slot] = c;
                } else {
                    atomicOr(&cnt[K_ERR], CUDAPIC_DEVERR_SPAWN_I);
                }
                chi_c = sqrt(e_orig / en);
                chi_s = sqrt(fmax(0.0, (1.0 - chi_c) * (1.0 + chi_c)));
            }
            double nx, ny, nz;
            rot64(gm, chi_s, chi_c, se, ce, st, ct, sp, cp, nx, ny, nz);
            e.vx[p] = k.f1 * vx + k.f2 * nx;
            e.vy[p] = k.f1 * vy + k.f2 * ny;
            e.vz[p] = k.f1 * vz + k.f2 * nz;
        }
        rng0[p] = rs.s0;
        rng1[p] = rs.s1;
        rng2[p] = rs.s2;
        rng3[p] = rs.s3;
    }
}

// check_collisions_i + collision_i (Rust-CUDA/src/main.rs:1167-1292) in FP64.
__global__ void __launch_bounds__(F64_THREADS)
    f64_collide_i_kernel(P64 ion, uint32_t *__restrict__ r0, uint32_t *__restrict__ r1, uint32_t *__restrict__ r2,
                         uint32_t *__restrict__ r3, const uint32_t *__restrict__ cnt, const float *__restrict__ sig,
                         const float *__restrict__ cs, const D64 k) {
    const uint32_t n = min(cnt[K_NI], k.cap);
    for (uint32_t p = blockIdx.x * blockDim.x + threadIdx.x; p < n; p += gridDim.x * blockDim.x) {
        Xoshiro128p rs{r0[p], r1[p], r2[p], r3[p]};
        double ax, ay, az;
        three_normal(rs, k.nr, ax, ay, az);
        const double vx = ion.vx[p], vy = ion.vy[p], vz = ion.vz[p];
        const double gx = vx - ax, gy = vy - ay, gz = vz - az;
        const double g2 = gx * gx + gy * gy + gz * gz;
        const uint32_t idx = index_of(k.hmu * g2);
        const double nu = (double)__ldg(sig + idx) * sqrt(g2);
        const double u = draw(rs);
        if (u < 1.0 - exp(-nu * k.dt_i)) {
            const double t0 = (double)__ldg(cs + 3 * CS_RANGES + idx);
            const double t1 = t0 + (double)__ldg(cs + 4 * CS_RANGES + idx);
            double st, ct, sp, cp;
            euler64(gx, gy, gz, st, ct, sp, cp);
            double sc = 0.0, cc = -1.0;  // backscatter, chi = pi
            if (draw(rs) < t0 / t1) {    // isotropic
                cc = 1.0 - 2.0 * draw(rs);
                sc = sqrt(fmax(0.0, (1.0 - cc) * (1.0 + cc)));
            }
            double se, ce;
            sincos(6.283185307179586 * draw(rs), &se, &ce);
            double nx, ny, nz;
            rot64(sqrt(g2), sc, cc, se, ce, st, ct, sp, cp, nx, ny, nz);
            ion.vx[p] = 0.5 * (vx + ax) + 0.5 * nx;
            ion.vy[p] = 0.5 * (vy + ay) + 0.5 * ny;
            ion.vz[p] = 0.5 * (vz + az) + 0.5 * nz;
        }
        r0[p] = rs.s0;
        r1[p] = rs.s1;
        r2[p] = rs.s2;
        r3[p] = rs.s3;
    }
}

// EEPF of the central 10 % after the step (accumulate_eepf's definition).
__global__ void __launch_bounds__(F64_THREADS)
    f64_eepf_kernel(P64 e, const uint32_t *__restrict__ cnt, const double *__restrict__ E, uint32_t *__restrict__ eepf,
                    const D64 k) {
    __shared__ uint32_t h[N_EEPF];
    for (uint32_t j = threadIdx.x; j < N_EEPF; j += blockDim.x) h[j] = 0u;
    __syncthreads();
    const uint32_t n = min(cnt[K_NE], k.cap);
    for (uint32_t p = blockIdx.x * blockDim.x + threadIdx.x; p < n; p += gridDim.x * blockDim.x) {
        const double x = e.x[p];
        if (x <= k.min_x || x >= k.max_x) continue;
        const double pos = x * k.inv_dx;
        const int c = cell64(pos, k.n_g);
        const double c2 = pos - (double)c;
        const double ex = (1.0 - c2) * E[c] + c2 * E[c + 1];
        const double mvx = e.vx[p] - 0.5 * ex * k.kick;
        const double en = k.hme * (mvx * mvx + e.vy[p] * e.vy[p] + e.vz[p] * e.vz[p]);
        const double bin = en / 0.05;
        if (bin < (double)N_EEPF) atomicAdd(&h[(uint32_t)bin], 1u);
    }
    __syncthreads();
    for (uint32_t j = threadIdx.x; j < N_EEPF; j += blockDim.x)
        if (h[j]) atomicAdd(&eepf[j], h[j]);
}

}  // namespace

}  // namespace cudapic

using namespace cudapic;

struct cudapic_fp64 {
    cudapic_state *st = nullptr;
    int device = 0;
    cudaStream_t stream = nullptr;
    D64 k{};
    cudapic_grid g{};
    P64 p[2][2]{};       // [species][side]
    int side[2] = {0, 0};
    uint32_t *rng[2][4] = {};
    uint32_t *cnt = nullptr;
    double *dens_e = nullptr, *dens_i = nullptr, *pot = nullptr, *efield = nullptr, *pot0 = nullptr;
    double *cumul_e = nullptr, *cumul_i = nullptr, *pot_sum = nullptr, *power = nullptr;
    uint32_t *eepf = nullptr;
    bool measure = false;
    uint64_t t = 0, measured = 0, ion_measured = 0;
    cudaGraphExec_t graph[2] = {nullptr, nullptr};
    int graph_side[2][2] = {{-1, -1}, {-1, -1}};
    std::vector<void *> allocs;
};

namespace {

template <typename T>
int f64_alloc(cudapic_fp64 *d, T **p, size_t count) {
    void *v = nullptr;
    const cudaError_t e = cudaMalloc(&v, std::max<size_t>(count * sizeof(T), 16));
    if (e != cudaSuccess) return check_cuda(e, "fp64 allocation");
    d->allocs.push_back(v);
    *p = static_cast<T *>(v);
    return CUDAPIC_OK;
}

unsigned f64_grid(uint32_t cap) { return persistent_grid(F64_PER_SM, (cap + F64_THREADS - 1) / F64_THREADS); }

// One reference step (Rust-CUDA/src/main.rs:1728-1807) in FP64, on d->stream.
int f64_step(cudapic_fp64 *d, bool ion_step) {
    cudaStream_t st = d->stream;
    const D64 &k = d->k;
    const unsigned gd = f64_grid(k.cap);
    const int se = d->side[0], si = d->side[1];
    const size_t hsm = sizeof(double) * k.n_g;
    CUDAPIC_CHECK(check_cuda(cudaMemsetAsync(d->dens_e, 0, hsm, st), "fp64 zero density"));
    CUDAPIC_CHECK(launch_kernel("f64_deposit", f64_deposit_kernel, gd, F64_THREADS, hsm, st, d->p[0][se].x,
                                d->cnt + K_NE, d->dens_e, k));
    if (ion_step) {
        CUDAPIC_CHECK(check_cuda(cudaMemsetAsync(d->dens_i, 0, hsm, st), "fp64 zero ion density"));
        CUDAPIC_CHECK(launch_kernel("f64_deposit", f64_deposit_kernel, gd, F64_THREADS, hsm, st, d->p[1][si].x,
                                    d->cnt + K_NI, d->dens_i, k));
    }
    CUDAPIC_CHECK(launch_poisson_f64(d->dens_e, d->dens_i, d->pot, d->efield, d->pot0, d->cnt + K_STEP, ion_step ? 1 : 0,
                                     d->measure ? d->cumul_e : nullptr, d->measure ? d->cumul_i : nullptr,
                                     d->measure ? d->pot_sum : nullptr, d->g, st));
    CUDAPIC_CHECK(launch_kernel("f64_push", f64_push_kernel, gd, F64_THREADS, 0, st, d->p[0][se], d->p[0][se ^ 1],
                                d->cnt + K_ALIVE, d->cnt + K_NE, (const double *)d->efield, k.fe, k.dt_e,
                                d->measure ? d->power : nullptr, k));
    d->side[0] ^= 1;
    // n_e = alive; alive = n_e (the spawn counter starts at the survivors)
    CUDAPIC_CHECK(launch_kernel("f64_count", f64_count_kernel, 1, 32, 0, st, d->cnt, K_NE, K_ALIVE, 1, k.cap,
                                CUDAPIC_DEVERR_SPAWN_E));
    if (ion_step) {
        CUDAPIC_CHECK(launch_kernel("f64_push", f64_push_kernel, gd, F64_THREADS, 0, st, d->p[1][si], d->p[1][si ^ 1],
                                    d->cnt + K_ALIVE_I, d->cnt + K_NI, (const double *)d->efield, k.fi, k.dt_i,
                                    (double *)nullptr, k));
        d->side[1] ^= 1;
        CUDAPIC_CHECK(launch_kernel("f64_count", f64_count_kernel, 1, 32, 0, st, d->cnt, K_NI, K_ALIVE_I, 0, k.cap,
                                    CUDAPIC_DEVERR_SPAWN_I));
    }
    const int ne = d->side[0], ni = d->side[1];
    CUDAPIC_CHECK(launch_kernel("f64_collide_e", f64_collide_e_kernel, gd, F64_THREADS, 0, st, d->p[0][ne],
                                d->rng[0][0], d->rng[0][1], d->rng[0][2], d->rng[0][3], d->cnt, d->p[1][ni],
                                (const float *)d->st->sigma_tot_e, (const float *)d->st->cs, k));
    // n_e = alive (survivors + spawns); alive = 0
    CUDAPIC_CHECK(launch_kernel("f64_count", f64_count_kernel, 1, 32, 0, st, d->cnt, K_NE, K_ALIVE, 0, k.cap,
                                CUDAPIC_DEVERR_SPAWN_E));
    if (ion_step)
        CUDAPIC_CHECK(launch_kernel("f64_collide_i", f64_collide_i_kernel, gd, F64_THREADS, 0, st, d->p[1][ni],
                                    d->rng[1][0], d->rng[1][1], d->rng[1][2], d->rng[1][3], (const uint32_t *)d->cnt,
                                    (const float *)d->st->sigma_tot_i, (const float *)d->st->cs, k));
    if (d->measure)
        CUDAPIC_CHECK(launch_kernel("f64_eepf", f64_eepf_kernel, gd, F64_THREADS, 0, st, d->p[0][ne],
                                    (const uint32_t *)d->cnt, (const double *)d->efield, d->eepf, k));
    return CUDAPIC_OK;
}

}  // namespace

extern "C" int cudapic_fp64_create(cudapic_state *st, cudapic_fp64 **out) {
    if (!st || !out) return fail(CUDAPIC_ERR_ARG, "fp64_create: null pointer");
    *out = nullptr;
    const cudapic_params &pp = st->params;
    if (pp.n_g > F64_MAX_NG) return fail(CUDAPIC_ERR_ARG, "fp64_create: n_g > 4096");
    uint64_t steps = 0;
    CUDAPIC_CHECK(cudapic_state_steps_done(st, &steps));
    if (steps % pp.n_sub) return fail(CUDAPIC_ERR_STATE, "fp64_create: the state is inside an ion cycle");
    DeviceGuard dg(st->device);
    auto *d = new cudapic_fp64();
    d->st = st;
    d->device = st->device;
    d->stream = st->stream;
    d->g = st->grid;
    d->g.dev_err = nullptr;
    d->g.work = nullptr;
    D64 &k = d->k;
    const double e = 1.60217662e-19, me = 9.10938356e-31, mi = 6.63352090e-26, kb = 1.38064852e-23;
    const double dt_e = 1.0 / pp.frequency / (double)pp.n_t;
    k.n_g = pp.n_g;
    k.cap = pp.capacity;
    k.n_t = pp.n_t;
    k.n_sub = pp.n_sub;
    k.dx = pp.gap / (double)(pp.n_g - 1);
    k.inv_dx = 1.0 / k.dx;
    k.gap = pp.gap;
    k.dt_e = dt_e;
    k.dt_i = (double)pp.n_sub * dt_e;
    k.fe = -e * dt_e / me;
    k.fi = e * k.dt_i / mi;
    k.wf = pp.weight / (pp.electrode_area * k.dx);
    k.f1 = me / (me + mi);
    k.f2 = mi / (me + mi);
    k.hme = 0.5 * me / e;
    k.hmu = 0.5 * (mi / 2.0) / e;
    k.nr = std::sqrt(kb * pp.temperature / mi);
    k.min_x = 0.45 * pp.gap;
    k.max_x = 0.55 * pp.gap;
    k.kick = dt_e * e / me;
    k.me = me;
    k.qe = e;
    d->t = steps;
    const size_t cap = k.cap, n_g = k.n_g;
    int rc = CUDAPIC_OK;
    auto bail = [&](int r) {
        cudapic_fp64_destroy(d);
        return r;
    };
    for (int sp = 0; sp < 2; ++sp)
        for (int sd = 0; sd < 2; ++sd)
            if ((rc = f64_alloc(d, &d->p[sp][sd].x, cap)) || (rc = f64_alloc(d, &d->p[sp][sd].vx, cap)) ||
                (rc = f64_alloc(d, &d->p[sp][sd].vy, cap)) || (rc = f64_alloc(d, &d->p[sp][sd].vz, cap)))
                return bail(rc);
    for (int sp = 0; sp < 2; ++sp)
        for (int c = 0; c < 4; ++c)
            if ((rc = f64_alloc(d, &d->rng[sp][c], cap))) return bail(rc);
    if ((rc = f64_alloc(d, &d->cnt, K_COUNT + 4)) || (rc = f64_alloc(d, &d->dens_e, n_g)) ||
        (rc = f64_alloc(d, &d->dens_i, n_g)) || (rc = f64_alloc(d, &d->pot, n_g)) ||
        (rc = f64_alloc(d, &d->efield, n_g)) || (rc = f64_alloc(d, &d->pot0, pp.n_t)) ||
        (rc = f64_alloc(d, &d->cumul_e, n_g)) || (rc = f64_alloc(d, &d->cumul_i, n_g)) ||
        (rc = f64_alloc(d, &d->pot_sum, n_g)) || (rc = f64_alloc(d, &d->power, 1)) ||
        (rc = f64_alloc(d, &d->eepf, N_EEPF)))
        return bail(rc);
    // particles (widened from the state's f32) and RNG planes
    uint32_t ne = 0, ni = 0;
    if ((rc = cudapic_state_counts(st, &ne, &ni))) return bail(rc);
    cudapic_buffers b;
    if ((rc = cudapic_state_buffers(st, &b))) return bail(rc);
    const uint32_t n[2] = {ne, ni};
    std::vector<float> hf(cap);
    std::vector<double> hd(cap);
    for (int sp = 0; sp < 2; ++sp) {
        const float *src[4] = {b.x[sp], b.vx[sp], b.vy[sp], b.vz[sp]};
        double *dst[4] = {d->p[sp][0].x, d->p[sp][0].vx, d->p[sp][0].vy, d->p[sp][0].vz};
        for (int c = 0; c < 4; ++c) {
            if (n[sp]) {
                if ((rc = check_cuda(cudaMemcpyAsync(hf.data(), src[c], sizeof(float) * n[sp], cudaMemcpyDeviceToHost,
                                                     d->stream), "fp64 read")) ||
                    (rc = check_cuda(cudaStreamSynchronize(d->stream), "fp64 read sync")))
                    return bail(rc);
                for (uint32_t j = 0; j < n[sp]; ++j) hd[j] = (double)hf[j];
                if ((rc = check_cuda(cudaMemcpyAsync(dst[c], hd.data(), sizeof(double) * n[sp], cudaMemcpyHostToDevice,
                                                     d->stream), "fp64 write")) ||
                    (rc = check_cuda(cudaStreamSynchronize(d->stream), "fp64 write sync")))
                    return bail(rc);
            }
            if ((rc = check_cuda(cudaMemcpyAsync(d->rng[sp][c], b.rng[sp][c], sizeof(uint32_t) * cap,
                                                 cudaMemcpyDeviceToDevice, d->stream), "fp64 rng")))
                return bail(rc);
        }
    }
    std::vector<double> table(pp.n_t);
    for (uint32_t t = 0; t < pp.n_t; ++t)
        table[t] = pp.voltage * std::cos(((double)t / (double)pp.n_t) * (2.0 * 3.141592653589793));
    uint32_t c0[K_COUNT + 4] = {};
    c0[K_NE] = ne;
    c0[K_NI] = ni;
    c0[K_STEP] = (uint32_t)(steps % pp.n_t);
    if ((rc = check_cuda(cudaMemcpyAsync(d->pot0, table.data(), sizeof(double) * pp.n_t, cudaMemcpyHostToDevice,
                                         d->stream), "fp64 rf table")) ||
        (rc = check_cuda(cudaMemcpyAsync(d->cnt, c0, sizeof(c0), cudaMemcpyHostToDevice, d->stream), "fp64 counters")) ||
        (rc = check_cuda(cudaStreamSynchronize(d->stream), "fp64 create sync")))
        return bail(rc);
    if ((rc = cudapic_fp64_set_measure(d, 0))) return bail(rc);
    *out = d;
    return CUDAPIC_OK;
}

extern "C" int cudapic_fp64_set_measure(cudapic_fp64 *d, int on) {
    if (!d) return fail(CUDAPIC_ERR_ARG, "fp64_set_measure: null pointer");
    DeviceGuard dg(d->device);
    cudaStream_t st = d->stream;
    const size_t n_g = d->k.n_g;
    CUDAPIC_CHECK(check_cuda(cudaMemsetAsync(d->cumul_e, 0, sizeof(double) * n_g, st), "fp64 measure"));
    CUDAPIC_CHECK(check_cuda(cudaMemsetAsync(d->cumul_i, 0, sizeof(double) * n_g, st), "fp64 measure"));
    CUDAPIC_CHECK(check_cuda(cudaMemsetAsync(d->pot_sum, 0, sizeof(double) * n_g, st), "fp64 measure"));
    CUDAPIC_CHECK(check_cuda(cudaMemsetAsync(d->power, 0, sizeof(double), st), "fp64 measure"));
    CUDAPIC_CHECK(check_cuda(cudaMemsetAsync(d->eepf, 0, sizeof(uint32_t) * N_EEPF, st), "fp64 measure"));
    d->measure = on != 0;
    d->measured = 0;
    d->ion_measured = 0;
    return CUDAPIC_OK;
}

extern "C" int cudapic_fp64_run_steps(cudapic_fp64 *d, uint64_t n_steps) {
    if (!d) return fail(CUDAPIC_ERR_ARG, "fp64_run_steps: null pointer");
    DeviceGuard dg(d->device);
    const uint32_t n_sub = d->k.n_sub;
    const int m = d->measure ? 1 : 0;
    while (n_steps) {
        const bool ion_step = d->t % n_sub == 0;
        if (ion_step && n_steps >= n_sub) {
            // one ion cycle from a CUDA graph (captured for the current sides)
            if (!d->graph[m] || d->graph_side[m][0] != d->side[0] || d->graph_side[m][1] != d->side[1]) {
                if (d->graph[m]) cudaGraphExecDestroy(d->graph[m]);
                d->graph[m] = nullptr;
                const int s0 = d->side[0], s1 = d->side[1];
                cudaGraph_t gr;
                CUDAPIC_CHECK(check_cuda(cudaStreamBeginCapture(d->stream, cudaStreamCaptureModeThreadLocal), "fp64 capture"));
                int rc = CUDAPIC_OK;
                for (uint32_t j = 0; j < n_sub && rc == CUDAPIC_OK; ++j) rc = f64_step(d, j == 0);
                const cudaError_t ce = cudaStreamEndCapture(d->stream, &gr);
                d->side[0] = s0;  // the capture only recorded the steps
                d->side[1] = s1;
                if (rc != CUDAPIC_OK) return rc;
                CUDAPIC_CHECK(check_cuda(ce, "fp64 end capture"));
                const cudaError_t ie = cudaGraphInstantiate(&d->graph[m], gr, 0);
                cudaGraphDestroy(gr);
                CUDAPIC_CHECK(check_cuda(ie, "fp64 instantiate"));
                d->graph_side[m][0] = s0;
                d->graph_side[m][1] = s1;
            }
            CUDAPIC_CHECK(check_cuda(cudaGraphLaunch(d->graph[m], d->stream), "fp64 graph launch"));
            // n_sub steps flip the electron side n_sub times, the ion side once
            if (n_sub & 1u) d->side[0] ^= 1;
            d->side[1] ^= 1;
            d->t += n_sub;
            if (d->measure) {
                d->measured += n_sub;
                d->ion_measured += 1;
            }
            n_steps -= n_sub;
        } else {
            CUDAPIC_CHECK(f64_step(d, ion_step));
            d->t += 1;
            if (d->measure) {
                d->measured += 1;
                d->ion_measured += ion_step ? 1 : 0;
            }
            n_steps -= 1;
        }
    }
    return CUDAPIC_OK;
}

extern "C" int cudapic_fp64_measurements(cudapic_fp64 *d, double *cumul_e, double *cumul_i, double *pot_sum,
                                         uint32_t *eepf, double *power_sum, uint64_t steps[2], uint32_t counts[2],
                                         uint32_t *dev_err) {
    if (!d) return fail(CUDAPIC_ERR_ARG, "fp64_measurements: null pointer");
    DeviceGuard dg(d->device);
    cudaStream_t st = d->stream;
    const size_t n_g = d->k.n_g;
    if (cumul_e) CUDAPIC_CHECK(check_cuda(cudaMemcpyAsync(cumul_e, d->cumul_e, 8 * n_g, cudaMemcpyDeviceToHost, st), "fp64 read"));
    if (cumul_i) CUDAPIC_CHECK(check_cuda(cudaMemcpyAsync(cumul_i, d->cumul_i, 8 * n_g, cudaMemcpyDeviceToHost, st), "fp64 read"));
    if (pot_sum) CUDAPIC_CHECK(check_cuda(cudaMemcpyAsync(pot_sum, d->pot_sum, 8 * n_g, cudaMemcpyDeviceToHost, st), "fp64 read"));
    if (eepf) CUDAPIC_CHECK(check_cuda(cudaMemcpyAsync(eepf, d->eepf, 4 * N_EEPF, cudaMemcpyDeviceToHost, st), "fp64 read"));
    if (power_sum) CUDAPIC_CHECK(check_cuda(cudaMemcpyAsync(power_sum, d->power, 8, cudaMemcpyDeviceToHost, st), "fp64 read"));
    uint32_t c[K_COUNT];
    CUDAPIC_CHECK(check_cuda(cudaMemcpyAsync(c, d->cnt, sizeof(c), cudaMemcpyDeviceToHost, st), "fp64 read"));
    CUDAPIC_CHECK(check_cuda(cudaStreamSynchronize(st), "fp64 read sync"));
    if (steps) {
        steps[0] = d->measured;
        steps[1] = d->ion_measured;
    }
    if (counts) {
        counts[0] = c[K_NE];
        counts[1] = c[K_NI];
    }
    if (dev_err) *dev_err = c[K_ERR];
    return CUDAPIC_OK;
}

extern "C" int cudapic_fp64_destroy(cudapic_fp64 *d) {
    if (!d) return CUDAPIC_OK;
    DeviceGuard dg(d->device);
    if (d->stream) cudaStreamSynchronize(d->stream);
    for (int m = 0; m < 2; ++m)
        if (d->graph[m]) cudaGraphExecDestroy(d->graph[m]);
    for (void *p : d->allocs) cudaFree(p);
    delete d;
    return CUDAPIC_OK;
}
