// sensitivity.cu -- voltage sensitivities of time-averaged observables of one
// discharge by a pathwise adjoint, with collision events and random draws
// frozen: forward run with checkpoints, segment-wise recompute with a tape,
// reverse sweep (cudapic_sens_* in include/cudapic.h).
//
// Model: the slot form of the reference step (Rust-CUDA/src/main.rs:1725-1808):
// the same kernels in the same order -- densities, Poisson, electron push,
// ion push every N_SUB-th step, electron collisions with their spawns, ion
// collisions -- with particles kept in their slots.  An absorbed particle is
// marked dead (x = -1) instead of being compacted away, and the spawns of a
// step take the next free slots in the slot order of their parents (a chunk
// count, a scan, a ranked write), so each particle keeps one RNG stream for
// its whole life and a run is a deterministic function of the initial state
// and the voltage: recompute from a checkpoint reproduces the trajectory bit
// for bit.  Deposits are exact integer sums (2^-20 fixed point), the Poisson
// sums FP64, scattering uses the algebraic sines and cosines.
//
// Observables (time averages over the window of K steps):
//   J_P  <j E> electron power averaged over the gap [W m^-3] (C/eduPIC.cc:
//        593-614, 1011-1026, per particle): -e (W/A) / L / K * sum over steps
//        and electrons of (v + f E(x)/2) E(x);
//   J_G  ion flux to the grounded electrode [m^-2 s^-1]: the CIC flux density
//        n v at node N_G-1 (boundary node doubled, as the density), a smooth
//        estimate of the counted flux of C/eduPIC.cc:651-658.
//
// Adjoint kernels: push (field gather -> its adjoint scatters into the field
// adjoint, FP64 shared-memory sums), collisions (Jacobians by forward-mode
// tangents of the same scattering arithmetic, applied transposed), spawns
// (a child's adjoint flows back to its parent), the symmetric Poisson solve
// (the same two-scan closed form, in kernels_poisson.cu), deposit (a gather).
// Particle adjoints in f32, the field, density and voltage adjoints in FP64.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <vector>

#include "common.cuh"
#include "detmath.cuh"
#include "internal.h"
#include "mcc.cuh"
#include "state_impl.h"

namespace cudapic {

namespace {

constexpr int SENS_THREADS = 256;
constexpr int SENS_PER_SM = 4;
constexpr uint32_t SENS_CHUNK = 1024;      // spawn-order chunk (one CTA of the spawn write)
constexpr uint32_t NO_SPAWN = 0xFFFFFFFFu;
constexpr uint32_t SPAWN_NOREC = 0xFFFFFFFEu;
constexpr uint32_t NO_SLOT = 0xFFFFFFFFu;
constexpr uint32_t SENS_DEP_Q = 20;
constexpr uint32_t SENS_MAX_NG = 4096;

// counters block
enum : int { C_NE = 0, C_NI, C_REC_E, C_REC_I, C_ERR, C_N0E, C_N0I, C_PAD, C_COUNT };

struct SensRecE {
    uint32_t p, ev, ce, ci;
    float v[3];
    float a, eta;   // a: cos chi draw 1 - 2u (ev 1, 2) or the energy-sharing draw u (ev 3)
};

struct SensRecI {
    uint32_t p, ev;
    float v[3], t[3];  // pre-collision velocity, target atom velocity
    float c, eta;      // c: cos chi draw (ev 4)
};

struct Planes {
    float *x, *vx, *vy, *vz;
    uint32_t *r[4];
};

// ---------------------------------------------------------------- tangents
// Forward-mode derivative in three directions (d/dvx, d/dvy, d/dvz).
struct D3 {
    float v, d0, d1, d2;
};
__device__ __forceinline__ D3 dc(float c) { return {c, 0.0f, 0.0f, 0.0f}; }
__device__ __forceinline__ D3 operator+(D3 a, D3 b) { return {a.v + b.v, a.d0 + b.d0, a.d1 + b.d1, a.d2 + b.d2}; }
__device__ __forceinline__ D3 operator-(D3 a, D3 b) { return {a.v - b.v, a.d0 - b.d0, a.d1 - b.d1, a.d2 - b.d2}; }
__device__ __forceinline__ D3 operator-(D3 a) { return {-a.v, -a.d0, -a.d1, -a.d2}; }
__device__ __forceinline__ D3 operator*(D3 a, D3 b) {
    return {a.v * b.v, a.d0 * b.v + a.v * b.d0, a.d1 * b.v + a.v * b.d1, a.d2 * b.v + a.v * b.d2};
}
__device__ __forceinline__ D3 operator*(float a, D3 b) { return {a * b.v, a * b.d0, a * b.d1, a * b.d2}; }
__device__ __forceinline__ D3 operator*(D3 a, float b) { return {a.v * b, a.d0 * b, a.d1 * b, a.d2 * b}; }
__device__ __forceinline__ D3 operator/(D3 a, D3 b) {
    const float q = a.v / b.v;
    return {q, (a.d0 - q * b.d0) / b.v, (a.d1 - q * b.d1) / b.v, (a.d2 - q * b.d2) / b.v};
}
__device__ __forceinline__ D3 operator/(D3 a, float b) { return {a.v / b, a.d0 / b, a.d1 / b, a.d2 / b}; }
__device__ __forceinline__ D3 operator-(float a, D3 b) { return {a - b.v, -b.d0, -b.d1, -b.d2}; }
__device__ __forceinline__ D3 operator+(float a, D3 b) { return {a + b.v, b.d0, b.d1, b.d2}; }
__device__ __forceinline__ D3 operator+(D3 a, float b) { return {a.v + b, a.d0, a.d1, a.d2}; }
__device__ __forceinline__ D3 operator-(D3 a, float b) { return {a.v - b, a.d0, a.d1, a.d2}; }
__device__ __forceinline__ float val(float a) { return a; }
__device__ __forceinline__ float val(const D3 &a) { return a.v; }
__device__ __forceinline__ float tsqrt(float a) { return sqrtf(a); }
__device__ __forceinline__ D3 tsqrt(D3 a) {
    const float s = sqrtf(a.v);
    const float k = s > 0.0f ? 0.5f / s : 0.0f;
    return {s, a.d0 * k, a.d1 * k, a.d2 * k};
}
__device__ __forceinline__ float tfabs(float a) { return fabsf(a); }
__device__ __forceinline__ D3 tfabs(D3 a) { return a.v < 0.0f ? -a : a; }
__device__ __forceinline__ float ttan(float a) { return dm::tanf_det(a); }
__device__ __forceinline__ D3 ttan(D3 a) {
    const float t = dm::tanf_det(a.v);
    const float k = 1.0f + t * t;
    return {t, a.d0 * k, a.d1 * k, a.d2 * k};
}
__device__ __forceinline__ float tatan(float a) { return dm::atanf_det(a); }
__device__ __forceinline__ D3 tatan(D3 a) {
    const float k = 1.0f / (1.0f + a.v * a.v);
    return {dm::atanf_det(a.v), a.d0 * k, a.d1 * k, a.d2 * k};
}
template <typename T> __device__ __forceinline__ T tconst(float c);
template <> __device__ __forceinline__ float tconst<float>(float c) { return c; }
template <> __device__ __forceinline__ D3 tconst<D3>(float c) { return dc(c); }

// --------------------------------------------------------------- scattering
struct ScatK {
    float f1, f2;
};

template <typename T>
__device__ __forceinline__ void euler_alg_t(T gx, T gy, T gz, T &st, T &ct, T &sp, T &cp) {
    const T r2 = gy * gy + gz * gz;
    const T r = tsqrt(r2);
    if (val(gx) == 0.0f) {
        st = tconst<T>(1.0f);
        ct = tconst<T>(0.0f);
    } else {
        const T gn = tsqrt(gx * gx + r2);
        st = r / gn;
        ct = gx / gn;
    }
    if (val(gy) == 0.0f) {
        sp = tconst<T>(val(gz) > 0.0f ? 1.0f : -1.0f);
        cp = tconst<T>(0.0f);
    } else {
        sp = gz / r;
        cp = gy / r;
    }
}

template <typename T>
__device__ __forceinline__ void sincos_acos_t(T c, T &s, T &co) {
    const T t = (1.0f - c) * (1.0f + c);
    s = val(t) > 0.0f ? tsqrt(t) : tconst<T>(0.0f);
    co = c;
}

template <typename T>
__device__ __forceinline__ void rot_t(T g, T sc, T cc, float se, float ce, T st, T ct, T sp, T cp, T &ox, T &oy,
                                      T &oz) {
    ox = g * (ct * cc - st * sc * ce);
    oy = g * (st * cp * cc + ct * cp * sc * ce - sp * sc * se);
    oz = g * (st * sp * cc + ct * sp * sc * ce + cp * sc * se);
}

// collision_e (Rust-CUDA/src/main.rs:1035-1165) with the algebraic sines and
// cosines and the draws given (ev 1 elastic / 2 excitation: a = 1 - 2u is
// cos chi; ev 3 ionization: a = the energy-sharing draw u; eta = 2 pi u):
// out = the scattered velocity, child (ev 3) = the new electron.  T = float
// is the forward arithmetic, T = D3 its tangents.
template <typename T>
__device__ void scatter_e_t(const ScatK &k, const T v[3], int ev, float a, float eta, T out[3], T child[3]) {
    const float exc_j = 11.5f * E_CHARGE_F;
    const float ion_j = 15.8f * E_CHARGE_F;
    const T gx = v[0], gy = v[1], gz = v[2];
    T gm = tsqrt(gx * gx + gy * gy + gz * gz);
    const T wx = k.f1 * gx, wy = k.f1 * gy, wz = k.f1 * gz;
    T st, ct, sp, cp;
    euler_alg_t(gx, gy, gz, st, ct, sp, cp);
    T chi_s, chi_c;
    float se, ce;
    if (ev == 1) {
        sincos_acos_t(tconst<T>(a), chi_s, chi_c);
    } else if (ev == 2) {
        T en = 0.5f * E_MASS_F * gm * gm;
        en = tfabs(en - exc_j);
        gm = tsqrt(2.0f * en / E_MASS_F);
        sincos_acos_t(tconst<T>(a), chi_s, chi_c);
    } else {
        T en = 0.5f * E_MASS_F * gm * gm;
        en = tfabs(en - ion_j);
        const T e_new = 10.0f * ttan(a * tatan(en / E_CHARGE_F / 20.0f)) * E_CHARGE_F;
        const T e_orig = tfabs(en - e_new);
        gm = tsqrt(2.0f * e_orig / E_MASS_F);
        const T g_new = tsqrt(2.0f * e_new / E_MASS_F);
        T sc2, cc2, nx, ny, nz;
        sincos_acos_t(tsqrt(e_new / en), sc2, cc2);
        dm::sincosf_det(eta, &se, &ce);
        rot_t(g_new, sc2, cc2, -se, -ce, st, ct, sp, cp, nx, ny, nz);
        child[0] = wx + k.f2 * nx;
        child[1] = wy + k.f2 * ny;
        child[2] = wz + k.f2 * nz;
        sincos_acos_t(tsqrt(e_orig / en), chi_s, chi_c);
    }
    if (ev != 3) dm::sincosf_det(eta, &se, &ce);
    T nx, ny, nz;
    rot_t(gm, chi_s, chi_c, se, ce, st, ct, sp, cp, nx, ny, nz);
    out[0] = wx + k.f2 * nx;
    out[1] = wy + k.f2 * ny;
    out[2] = wz + k.f2 * nz;
}

// collision_i (Rust-CUDA/src/main.rs:1221-1292) with the algebraic sines and
// cosines: ev 4 isotropic (c = cos chi), ev 5 backscatter (chi = pi exactly).
template <typename T>
__device__ void scatter_i_t(const T v[3], const float t[3], int ev, float c, float eta, T out[3]) {
    const T gx = v[0] - t[0], gy = v[1] - t[1], gz = v[2] - t[2];
    const T gg = tsqrt(gx * gx + gy * gy + gz * gz);
    const T wx = 0.5f * (v[0] + t[0]), wy = 0.5f * (v[1] + t[1]), wz = 0.5f * (v[2] + t[2]);
    T st, ct, sp, cp, sc, cc;
    euler_alg_t(gx, gy, gz, st, ct, sp, cp);
    if (ev == 4) {
        sincos_acos_t(tconst<T>(c), sc, cc);
    } else {
        sc = tconst<T>(0.0f);
        cc = tconst<T>(-1.0f);
    }
    float se, ce;
    dm::sincosf_det(eta, &se, &ce);
    T nx, ny, nz;
    rot_t(gg, sc, cc, se, ce, st, ct, sp, cp, nx, ny, nz);
    out[0] = wx + 0.5f * nx;
    out[1] = wy + 0.5f * ny;
    out[2] = wz + 0.5f * nz;
}

__device__ __forceinline__ D3 seed(float v, int k) {
    return {v, k == 0 ? 1.0f : 0.0f, k == 1 ? 1.0f : 0.0f, k == 2 ? 1.0f : 0.0f};
}

// w^T J: the adjoint of the inputs given the adjoint w of the outputs.
__device__ __forceinline__ void apply_jt(const D3 out[3], const float w[3], float r[3]) {
    r[0] = out[0].d0 * w[0] + out[1].d0 * w[1] + out[2].d0 * w[2];
    r[1] = out[0].d1 * w[0] + out[1].d1 * w[1] + out[2].d1 * w[2];
    r[2] = out[0].d2 * w[0] + out[1].d2 * w[1] + out[2].d2 * w[2];
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

// ------------------------------------------------------------------ forward
__global__ void __launch_bounds__(SENS_THREADS)
    sens_deposit_kernel(const float *__restrict__ x, const uint32_t *__restrict__ n_ptr,
                        unsigned long long *__restrict__ hist, const cudapic_grid g) {
    extern __shared__ unsigned long long h[];
    for (uint32_t k = threadIdx.x; k < g.n_g; k += blockDim.x) h[k] = 0ull;
    __syncthreads();
    const uint32_t n = min(*n_ptr, g.capacity);
    for (uint32_t p = blockIdx.x * blockDim.x + threadIdx.x; p < n; p += gridDim.x * blockDim.x) {
        const float xv = x[p];
        if (!(xv >= 0.0f)) continue;
        const float pos = xv * g.inv_dx;
        const int c = cell_of(pos, g.n_g);
        const float rem = pos - (float)c;
        const uint32_t r = min(__float2uint_rn(rem * (float)(1u << SENS_DEP_Q)), 1u << SENS_DEP_Q);
        atomicAdd(&h[c], (unsigned long long)((1u << SENS_DEP_Q) - r));
        atomicAdd(&h[c + 1], (unsigned long long)r);
    }
    __syncthreads();
    for (uint32_t k = threadIdx.x; k < g.n_g; k += blockDim.x)
        if (h[k]) atomicAdd(&hist[k], h[k]);
}

// Node sums -> f32 densities (boundary nodes doubled); clears the sums.
__global__ void sens_density_kernel(unsigned long long *__restrict__ hist_e, unsigned long long *__restrict__ hist_i,
                                    float *__restrict__ dens_e, float *__restrict__ dens_i, int ions,
                                    const cudapic_grid g) {
    const double w = g.weight_factor_d * (1.0 / (double)(1u << SENS_DEP_Q));
    for (int s = 0; s < (ions ? 2 : 1); ++s) {
        unsigned long long *h = s ? hist_i : hist_e;
        float *d = s ? dens_i : dens_e;
        for (uint32_t k = threadIdx.x; k < g.n_g; k += blockDim.x) {
            float f = (float)((double)h[k] * w);
            if (k == 0 || k == g.n_g - 1) f *= 2.0f;
            d[k] = f;
            h[k] = 0ull;
        }
    }
}

// Push of the live slots in place (Rust-CUDA/src/main.rs:596-620); a particle
// leaving [0, L] is marked dead.  obs (may be null) += the observable sum of
// the species; tx / tv (may be null): the tape of x and v before the push.
__global__ void __launch_bounds__(SENS_THREADS)
    sens_push_kernel(float *__restrict__ x, float *__restrict__ vx, const uint32_t *__restrict__ n_ptr,
                     const float *__restrict__ E, float f, float dt, int ions, double *__restrict__ obs,
                     float *__restrict__ tx, float *__restrict__ tv, const cudapic_grid g) {
    __shared__ double red[SENS_THREADS / 32];
    const uint32_t n = min(*n_ptr, g.capacity);
    double acc = 0.0;
    for (uint32_t p = blockIdx.x * blockDim.x + threadIdx.x; p < n; p += gridDim.x * blockDim.x) {
        const float xv = x[p], v = vx[p];
        if (tx) {
            tx[p] = xv;
            tv[p] = v;
        }
        if (!(xv >= 0.0f)) continue;
        const float pos = xv * g.inv_dx;
        const int c = cell_of(pos, g.n_g);
        const float c2 = pos - (float)c;
        const float ex = (1.0f - c2) * E[c] + c2 * E[c + 1];
        if (!ions) acc += ((double)v + 0.5 * (double)f * (double)ex) * (double)ex;
        else if (c == (int)g.n_g - 2) acc += (double)v * (double)c2;
        const float v1 = v + f * ex;
        const float x1 = xv + v1 * dt;
        vx[p] = v1;
        x[p] = (x1 >= 0.0f && x1 <= g.gap) ? x1 : -1.0f;
    }
    if (obs) {
        const double s = block_sum(acc, red);
        if (threadIdx.x == 0 && s != 0.0) atomicAdd(obs, s);
    }
}

// check_collisions_e (Rust-CUDA/src/main.rs:971-1033) over the slots live
// before this step's spawns; an ionizing slot leaves its spawn request
// (children's velocities, record index) for the ranked spawn write.
__global__ void __launch_bounds__(SENS_THREADS)
    sens_collide_e_kernel(Planes e, uint32_t *__restrict__ cnt, const float *__restrict__ sig_e,
                          const float *__restrict__ cs, SensRecE *__restrict__ rec, uint32_t rec_cap,
                          uint32_t *__restrict__ spawn_rec, float *__restrict__ spawn_v,
                          uint32_t *__restrict__ chunk_count, const cudapic_grid g) {
    const uint32_t n = min(cnt[C_NE], g.capacity);
    const uint32_t cap = g.capacity;
    const ScatK k{g.f1, g.f2};
    for (uint32_t p = blockIdx.x * blockDim.x + threadIdx.x; p < n; p += gridDim.x * blockDim.x) {
        if (!(e.x[p] >= 0.0f)) continue;
        Xoshiro128p rs{e.r[0][p], e.r[1][p], e.r[2][p], e.r[3][p]};
        const float v[3] = {e.vx[p], e.vy[p], e.vz[p]};
        const Test ts = test_electron(v[0], v[1], v[2], rs, GlobalTable{sig_e}, g);
        if (ts.collide) {
            const uint32_t idx = ts.idx;
            const float t0 = __ldg(cs + idx);
            const float t1 = t0 + __ldg(cs + CS_RANGES + idx);
            const float t2 = t1 + __ldg(cs + 2 * CS_RANGES + idx);
            const float rnd = rs.uniform();
            int ev;
            float a;
            if (rnd < t0 / t2) {
                ev = 1;
                a = 1.0f - 2.0f * rs.uniform();
            } else if (rnd < t1 / t2) {
                ev = 2;
                a = 1.0f - 2.0f * rs.uniform();
            } else {
                ev = 3;
                a = rs.uniform();
            }
            const float eta = TWO_PI_F * rs.uniform();
            float out[3], child[3];
            scatter_e_t<float>(k, v, ev, a, eta, out, child);
            uint32_t ri = SPAWN_NOREC;
            if (rec) {
                ri = atomicAdd(&cnt[C_REC_E], 1u);
                if (ri < rec_cap) {
                    SensRecE r;
                    r.p = p;
                    r.ev = (uint32_t)ev;
                    r.ce = NO_SLOT;
                    r.ci = NO_SLOT;
                    r.v[0] = v[0];
                    r.v[1] = v[1];
                    r.v[2] = v[2];
                    r.a = a;
                    r.eta = eta;
                    rec[ri] = r;
                } else {
                    set_dev_err(&cnt[C_ERR], CUDAPIC_DEVERR_RECORDS);
                    ri = SPAWN_NOREC;
                }
            }
            if (ev == 3) {
                float ia, ib, ic;
                rs.three_normal(g.normal_range, ia, ib, ic);
                spawn_v[0 * (size_t)cap + p] = child[0];
                spawn_v[1 * (size_t)cap + p] = child[1];
                spawn_v[2 * (size_t)cap + p] = child[2];
                spawn_v[3 * (size_t)cap + p] = ia;
                spawn_v[4 * (size_t)cap + p] = ib;
                spawn_v[5 * (size_t)cap + p] = ic;
                spawn_rec[p] = ri;
                atomicAdd(&chunk_count[p / SENS_CHUNK], 1u);
            }
            e.vx[p] = out[0];
            e.vy[p] = out[1];
            e.vz[p] = out[2];
        }
        e.r[0][p] = rs.s0;
        e.r[1][p] = rs.s1;
        e.r[2][p] = rs.s2;
        e.r[3][p] = rs.s3;
    }
}

__device__ __forceinline__ uint32_t block_excl_scan_u32(uint32_t v, uint32_t *wsum, uint32_t &total) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
    uint32_t incl = v;
    for (int o = 1; o < 32; o <<= 1) {
        const uint32_t t = __shfl_up_sync(0xffffffffu, incl, o);
        if (lane >= o) incl += t;
    }
    if (lane == 31) wsum[warp] = incl;
    __syncthreads();
    if (warp == 0) {
        uint32_t w = lane < nw ? wsum[lane] : 0u;
        for (int o = 1; o < 32; o <<= 1) {
            const uint32_t t = __shfl_up_sync(0xffffffffu, w, o);
            if (lane >= o) w += t;
        }
        if (lane < nw) wsum[lane] = w;
    }
    __syncthreads();
    const uint32_t excl = incl - v + (warp > 0 ? wsum[warp - 1] : 0u);
    total = wsum[nw - 1];
    __syncthreads();
    return excl;
}

// One CTA: exclusive scan of the spawn counts of the chunks in slot order;
// advances both counts (capped at the capacity, flagging dropped spawns).
__global__ void __launch_bounds__(1024)
    sens_spawn_scan_kernel(uint32_t *__restrict__ cnt, uint32_t *__restrict__ chunk_count,
                           uint32_t *__restrict__ chunk_off, uint32_t cap) {
    __shared__ uint32_t wsum[32];
    const uint32_t n0e = min(cnt[C_NE], cap), n0i = min(cnt[C_NI], cap);
    const uint32_t nch = (n0e + SENS_CHUNK - 1) / SENS_CHUNK;
    uint32_t running = 0;
    for (uint32_t base = 0; base < nch; base += blockDim.x) {
        const uint32_t i = base + threadIdx.x;
        const uint32_t v = i < nch ? chunk_count[i] : 0u;
        uint32_t total;
        const uint32_t ex = block_excl_scan_u32(v, wsum, total);
        if (i < nch) {
            chunk_off[i] = running + ex;
            chunk_count[i] = 0u;
        }
        running += total;
    }
    if (threadIdx.x == 0) {
        chunk_off[nch] = running;
        cnt[C_N0E] = n0e;
        cnt[C_N0I] = n0i;
        const uint64_t ne = (uint64_t)n0e + running, ni = (uint64_t)n0i + running;
        if (ne > cap) set_dev_err(&cnt[C_ERR], CUDAPIC_DEVERR_SPAWN_E);
        if (ni > cap) set_dev_err(&cnt[C_ERR], CUDAPIC_DEVERR_SPAWN_I);
        cnt[C_NE] = ne > cap ? cap : (uint32_t)ne;
        cnt[C_NI] = ni > cap ? cap : (uint32_t)ni;
    }
}

// One CTA of SENS_CHUNK threads per chunk with spawns: children at
// n0 + chunk offset + rank of the parent among the chunk's spawning slots.
__global__ void __launch_bounds__(SENS_CHUNK)
    sens_spawn_write_kernel(Planes e, Planes ion, const uint32_t *__restrict__ cnt,
                            const uint32_t *__restrict__ chunk_off, uint32_t *__restrict__ spawn_rec,
                            const float *__restrict__ spawn_v, SensRecE *__restrict__ rec, uint32_t cap) {
    __shared__ uint32_t wsum[32];
    const uint32_t n0e = cnt[C_N0E], n0i = cnt[C_N0I];
    const uint32_t nch = (n0e + SENS_CHUNK - 1) / SENS_CHUNK;
    for (uint32_t c = blockIdx.x; c < nch; c += gridDim.x) {
        if (chunk_off[c + 1] == chunk_off[c]) continue;  // uniform in the block
        const uint32_t p = c * SENS_CHUNK + threadIdx.x;
        const uint32_t fl = p < n0e ? spawn_rec[p] : NO_SPAWN;
        const uint32_t flag = fl != NO_SPAWN ? 1u : 0u;
        uint32_t total;
        const uint32_t rank = block_excl_scan_u32(flag, wsum, total);
        if (flag) {
            const uint32_t k = chunk_off[c] + rank;
            const uint32_t se = n0e + k, si = n0i + k;
            const float xp = e.x[p];
            uint32_t ce = NO_SLOT, ci = NO_SLOT;
            if (se < cap) {
                e.x[se] = xp;
                e.vx[se] = spawn_v[0 * (size_t)cap + p];
                e.vy[se] = spawn_v[1 * (size_t)cap + p];
                e.vz[se] = spawn_v[2 * (size_t)cap + p];
                ce = se;
            }
            if (si < cap) {
                ion.x[si] = xp;
                ion.vx[si] = spawn_v[3 * (size_t)cap + p];
                ion.vy[si] = spawn_v[4 * (size_t)cap + p];
                ion.vz[si] = spawn_v[5 * (size_t)cap + p];
                ci = si;
            }
            if (rec && fl != SPAWN_NOREC) {
                rec[fl].ce = ce;
                rec[fl].ci = ci;
            }
            spawn_rec[p] = NO_SPAWN;
        }
    }
}

// check_collisions_i (Rust-CUDA/src/main.rs:1167-1219) over the live ions,
// this step's spawns included.
__global__ void __launch_bounds__(SENS_THREADS)
    sens_collide_i_kernel(Planes ion, uint32_t *__restrict__ cnt, const float *__restrict__ sig_i,
                          const float *__restrict__ cs, SensRecI *__restrict__ rec, uint32_t rec_cap,
                          const cudapic_grid g) {
    const uint32_t n = min(cnt[C_NI], g.capacity);
    for (uint32_t p = blockIdx.x * blockDim.x + threadIdx.x; p < n; p += gridDim.x * blockDim.x) {
        if (!(ion.x[p] >= 0.0f)) continue;
        Xoshiro128p rs{ion.r[0][p], ion.r[1][p], ion.r[2][p], ion.r[3][p]};
        const float v[3] = {ion.vx[p], ion.vy[p], ion.vz[p]};
        const IonTest ts = test_ion(v[0], v[1], v[2], rs, GlobalTable{sig_i}, g);
        if (ts.collide) {
            const uint32_t idx = ts.idx;
            const float t0 = __ldg(cs + 3 * CS_RANGES + idx);
            const float t1 = t0 + __ldg(cs + 4 * CS_RANGES + idx);
            const float rnd = rs.uniform();
            int ev;
            float c = 0.0f;
            if (rnd < t0 / t1) {
                ev = 4;
                c = 1.0f - 2.0f * rs.uniform();
            } else {
                ev = 5;
            }
            const float eta = TWO_PI_F * rs.uniform();
            const float t[3] = {ts.vxa, ts.vya, ts.vza};
            float out[3];
            scatter_i_t<float>(v, t, ev, c, eta, out);
            ion.vx[p] = out[0];
            ion.vy[p] = out[1];
            ion.vz[p] = out[2];
            if (rec) {
                const uint32_t ri = atomicAdd(&cnt[C_REC_I], 1u);
                if (ri < rec_cap) {
                    SensRecI r;
                    r.p = p;
                    r.ev = (uint32_t)ev;
                    for (int j = 0; j < 3; ++j) {
                        r.v[j] = v[j];
                        r.t[j] = t[j];
                    }
                    r.c = c;
                    r.eta = eta;
                    rec[ri] = r;
                } else {
                    set_dev_err(&cnt[C_ERR], CUDAPIC_DEVERR_RECORDS);
                }
            }
        }
        ion.r[0][p] = rs.s0;
        ion.r[1][p] = rs.s1;
        ion.r[2][p] = rs.s2;
        ion.r[3][p] = rs.s3;
    }
}

__global__ void sens_fill_kernel(float *__restrict__ p, uint32_t n, float v) {
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) p[i] = v;
}

// Tape mark of a step: slot counts and record counters at its start.
__global__ void sens_mark_kernel(const uint32_t *__restrict__ cnt, uint32_t *__restrict__ mark) {
    if (threadIdx.x < 4) mark[threadIdx.x] = cnt[threadIdx.x];
}

// ------------------------------------------------------------------ adjoint
__global__ void __launch_bounds__(SENS_THREADS)
    sens_adj_collide_i_kernel(const SensRecI *__restrict__ rec, const uint32_t *__restrict__ mark0,
                              const uint32_t *__restrict__ mark1, uint32_t rec_cap, float *__restrict__ vbx,
                              float *__restrict__ vby, float *__restrict__ vbz) {
    // an overflowed tape (flagged by the forward kernel) is read only up to its capacity
    const uint32_t b = min(mark0[C_REC_I], rec_cap), e = min(mark1[C_REC_I], rec_cap);
    for (uint32_t j = b + blockIdx.x * blockDim.x + threadIdx.x; j < e; j += gridDim.x * blockDim.x) {
        const SensRecI r = rec[j];
        D3 v[3], out[3];
        for (int q = 0; q < 3; ++q) v[q] = seed(r.v[q], q);
        scatter_i_t<D3>(v, r.t, (int)r.ev, r.c, r.eta, out);
        const float w[3] = {vbx[r.p], vby[r.p], vbz[r.p]};
        float nv[3];
        apply_jt(out, w, nv);
        vbx[r.p] = nv[0];
        vby[r.p] = nv[1];
        vbz[r.p] = nv[2];
    }
}

struct AdjPlanes {
    float *x, *vx, *vy, *vz;
};

__global__ void __launch_bounds__(SENS_THREADS)
    sens_adj_collide_e_kernel(const SensRecE *__restrict__ rec, const uint32_t *__restrict__ mark0,
                              const uint32_t *__restrict__ mark1, uint32_t rec_cap, AdjPlanes e, AdjPlanes ion,
                              const cudapic_grid g) {
    const uint32_t b = min(mark0[C_REC_E], rec_cap), en = min(mark1[C_REC_E], rec_cap);
    const ScatK k{g.f1, g.f2};
    for (uint32_t j = b + blockIdx.x * blockDim.x + threadIdx.x; j < en; j += gridDim.x * blockDim.x) {
        const SensRecE r = rec[j];
        D3 v[3], out[3], child[3];
        for (int q = 0; q < 3; ++q) v[q] = seed(r.v[q], q);
        scatter_e_t<D3>(k, v, (int)r.ev, r.a, r.eta, out, child);
        const uint32_t p = r.p;
        const float w[3] = {e.vx[p], e.vy[p], e.vz[p]};
        float nv[3];
        apply_jt(out, w, nv);
        float xb = e.x[p];
        if (r.ev == 3 && r.ce != NO_SLOT) {
            const uint32_t s = r.ce;
            const float wc[3] = {e.vx[s], e.vy[s], e.vz[s]};
            float nc[3];
            apply_jt(child, wc, nc);
            for (int q = 0; q < 3; ++q) nv[q] += nc[q];
            xb += e.x[s];
            e.x[s] = e.vx[s] = e.vy[s] = e.vz[s] = 0.0f;
        }
        if (r.ev == 3 && r.ci != NO_SLOT) {
            const uint32_t s = r.ci;
            xb += ion.x[s];
            ion.x[s] = ion.vx[s] = ion.vy[s] = ion.vz[s] = 0.0f;
        }
        e.x[p] = xb;
        e.vx[p] = nv[0];
        e.vy[p] = nv[1];
        e.vz[p] = nv[2];
    }
}

// Adjoint of the push (and of the species' observable term, weight wo) of
// the slots live at the step's start; the field adjoint is summed in FP64.
__global__ void __launch_bounds__(SENS_THREADS)
    sens_adj_push_kernel(const float *__restrict__ tx, const float *__restrict__ tv, const uint32_t *__restrict__ n_ptr,
                         const float *__restrict__ E, float f, float dt, int ions, float wo, float *__restrict__ xb,
                         float *__restrict__ vb, double *__restrict__ eb, const cudapic_grid g) {
    extern __shared__ double ebs[];
    for (uint32_t k = threadIdx.x; k < g.n_g; k += blockDim.x) ebs[k] = 0.0;
    __syncthreads();
    const uint32_t n = min(*n_ptr, g.capacity);
    const float inv_dx = g.inv_dx;
    for (uint32_t p = blockIdx.x * blockDim.x + threadIdx.x; p < n; p += gridDim.x * blockDim.x) {
        const float x = tx[p];
        if (!(x >= 0.0f)) continue;
        const float v = tv[p];
        const float pos = x * inv_dx;
        const int c = cell_of(pos, g.n_g);
        const float c2 = pos - (float)c;
        const float e0 = E[c], e1 = E[c + 1];
        const float ex = (1.0f - c2) * e0 + c2 * e1;
        const float dex = (e1 - e0) * inv_dx;
        const float a = xb[p], b = vb[p];
        const float bt = b + dt * a;
        float nx = a, nv = bt, eg = bt * f;
        if (!ions) {
            nv += wo * ex;
            eg += wo * (v + f * ex);
        } else if (c == (int)g.n_g - 2) {
            nv += wo * c2;
            nx += wo * v * inv_dx;
        }
        nx += eg * dex;
        atomicAdd(&ebs[c], (double)eg * (double)(1.0f - c2));
        atomicAdd(&ebs[c + 1], (double)eg * (double)c2);
        xb[p] = nx;
        vb[p] = nv;
    }
    __syncthreads();
    for (uint32_t k = threadIdx.x; k < g.n_g; k += blockDim.x)
        if (ebs[k] != 0.0) atomicAdd(&eb[k], ebs[k]);
}

// Deposit adjoint: x adjoint += d/dx sum_k db[k] n_k(x) (CIC, boundary nodes doubled).
__global__ void __launch_bounds__(SENS_THREADS)
    sens_adj_gather_kernel(const float *__restrict__ tx, const uint32_t *__restrict__ n_ptr,
                           const double *__restrict__ db, float *__restrict__ xb, const cudapic_grid g) {
    const uint32_t n = min(*n_ptr, g.capacity);
    const double k = g.weight_factor_d / g.dx;
    for (uint32_t p = blockIdx.x * blockDim.x + threadIdx.x; p < n; p += gridDim.x * blockDim.x) {
        const float x = tx[p];
        if (!(x >= 0.0f)) continue;
        const int c = cell_of(x * g.inv_dx, g.n_g);
        const double b0 = c == 0 ? 2.0 : 1.0, b1 = (c + 1 == (int)g.n_g - 1) ? 2.0 : 1.0;
        xb[p] += (float)(k * (b1 * db[c + 1] - b0 * db[c]));
    }
}

}  // namespace

}  // namespace cudapic

using namespace cudapic;

struct cudapic_sens {
    cudapic_state *st = nullptr;
    int device = 0;
    cudaStream_t stream = nullptr;
    cudapic_grid g{};
    uint32_t cap = 0, K = 0, S = 0, H = 0, n_seg = 0, n_g = 0, n_sub = 0, n_t = 0;
    uint32_t rec_cap_e = 0, rec_cap_i = 0;
    uint32_t n_init[2] = {0, 0};
    double voltage = 0.0;
    bool have_forward = false;
    Planes cur[2]{}, init[2]{};
    uint32_t *cnt = nullptr;
    unsigned long long *hist = nullptr;  // [2][n_g]
    float *dens = nullptr, *efield = nullptr, *pot = nullptr;
    double *obs = nullptr;               // [2] raw sums
    uint32_t *spawn_rec = nullptr, *chunk_count = nullptr, *chunk_off = nullptr;
    float *spawn_v = nullptr;
    float *ckpt = nullptr;               // [n_seg][2][8][cap] (RNG planes stored bitwise)
    uint32_t *ckpt_cnt = nullptr;        // [n_seg][C_COUNT]
    float *tx_e = nullptr, *tv_e = nullptr, *tx_i = nullptr, *tv_i = nullptr, *tE = nullptr;
    uint32_t *tmark = nullptr;           // [S + 1][4]
    SensRecE *rec_e = nullptr;
    SensRecI *rec_i = nullptr;
    float *adj = nullptr;                // [2][4][cap]
    double *eb = nullptr, *neb = nullptr, *nib_acc = nullptr, *vbar = nullptr;
    std::vector<void *> allocs;
    size_t bytes = 0;
};

namespace {

int sens_alloc(cudapic_sens *s, void **p, size_t bytes) {
    *p = nullptr;
    if (bytes == 0) bytes = 16;
    const cudaError_t e = cudaMalloc(p, bytes);
    if (e != cudaSuccess) return check_cuda(e, "sensitivity allocation");
    s->allocs.push_back(*p);
    s->bytes += bytes;
    return CUDAPIC_OK;
}

template <typename T>
int sens_alloc_t(cudapic_sens *s, T **p, size_t count) {
    void *v = nullptr;
    CUDAPIC_CHECK(sens_alloc(s, &v, count * sizeof(T)));
    *p = static_cast<T *>(v);
    return CUDAPIC_OK;
}

Planes planes_of(float *base, uint32_t cap) {
    Planes p;
    p.x = base;
    p.vx = base + (size_t)cap;
    p.vy = base + 2 * (size_t)cap;
    p.vz = base + 3 * (size_t)cap;
    for (int k = 0; k < 4; ++k) p.r[k] = reinterpret_cast<uint32_t *>(base + (4 + k) * (size_t)cap);
    return p;
}

AdjPlanes adj_of(const cudapic_sens *s, int sp) {
    float *b = s->adj + (size_t)sp * 4 * s->cap;
    return {b, b + s->cap, b + 2 * (size_t)s->cap, b + 3 * (size_t)s->cap};
}

unsigned grid_n(uint32_t units) { return persistent_grid(SENS_PER_SM, (units + SENS_THREADS - 1) / SENS_THREADS); }

bool ion_step(const cudapic_sens *s, uint32_t t) { return t % s->n_sub == 0; }

float pot0_at(const cudapic_sens *s, uint32_t t) {
    return (float)(s->voltage * std::cos(((double)(t % s->n_t) / (double)s->n_t) * (2.0 * 3.141592653589793)));
}

double cos_at(const cudapic_sens *s, uint32_t t) {
    return std::cos(((double)(t % s->n_t) / (double)s->n_t) * (2.0 * 3.141592653589793));
}

// Observable scales per unit of the raw sums: J_P, J_G.
void obs_scale(const cudapic_sens *s, double *cP, double *cG) {
    const double w_over_a = s->g.weight_factor_d * s->g.dx;
    uint32_t k_i = 0;
    for (uint32_t t = 0; t < s->K; ++t) k_i += ion_step(s, t);
    *cP = -1.60217662e-19 * w_over_a / (double)s->g.gap / (double)s->K;
    *cG = 2.0 * s->g.weight_factor_d / (double)(k_i ? k_i : 1);
}

// One forward step t; rec: record the tape at step j of the segment.
int fwd_step(cudapic_sens *s, uint32_t t, bool rec, uint32_t j) {
    cudaStream_t st = s->stream;
    const cudapic_grid &g = s->g;
    const bool ions = ion_step(s, t);
    const size_t cap = s->cap;
    if (rec) CUDAPIC_CHECK(launch_kernel("sens_mark", sens_mark_kernel, 1, 32, 0, st, s->cnt, s->tmark + 4 * j));
    const unsigned gd = grid_n(s->cap);
    const size_t hsm = sizeof(unsigned long long) * s->n_g;
    CUDAPIC_CHECK(launch_kernel("sens_deposit", sens_deposit_kernel, gd, SENS_THREADS, hsm, st, s->cur[0].x,
                                s->cnt + C_NE, s->hist, g));
    if (ions)
        CUDAPIC_CHECK(launch_kernel("sens_deposit", sens_deposit_kernel, gd, SENS_THREADS, hsm, st, s->cur[1].x,
                                    s->cnt + C_NI, s->hist + s->n_g, g));
    CUDAPIC_CHECK(launch_kernel("sens_density", sens_density_kernel, 1, 512, 0, st, s->hist, s->hist + s->n_g,
                                s->dens, s->dens + s->n_g, ions ? 1 : 0, g));
    CUDAPIC_CHECK(launch_poisson(s->dens, s->dens + s->n_g, s->pot, s->efield, pot0_at(s, t), nullptr, nullptr, g, st));
    if (rec)
        CUDAPIC_CHECK(check_cuda(cudaMemcpyAsync(s->tE + (size_t)j * s->n_g, s->efield, sizeof(float) * s->n_g,
                                                 cudaMemcpyDeviceToDevice, st), "sensitivity field tape"));
    CUDAPIC_CHECK(launch_kernel("sens_push", sens_push_kernel, gd, SENS_THREADS, 0, st, s->cur[0].x, s->cur[0].vx,
                                s->cnt + C_NE, s->efield, g.factor_e, g.dt_e, 0, rec ? nullptr : s->obs,
                                rec ? s->tx_e + j * cap : nullptr, rec ? s->tv_e + j * cap : nullptr, g));
    if (ions) {
        const size_t ji = j / s->n_sub;
        CUDAPIC_CHECK(launch_kernel("sens_push", sens_push_kernel, gd, SENS_THREADS, 0, st, s->cur[1].x, s->cur[1].vx,
                                    s->cnt + C_NI, s->efield, g.factor_i, g.dt_i, 1, rec ? nullptr : s->obs + 1,
                                    rec ? s->tx_i + ji * cap : nullptr, rec ? s->tv_i + ji * cap : nullptr, g));
    }
    CUDAPIC_CHECK(launch_kernel("sens_collide_e", sens_collide_e_kernel, gd, SENS_THREADS, 0, st, s->cur[0], s->cnt,
                                s->st->sigma_tot_e, s->st->cs, rec ? s->rec_e : nullptr, s->rec_cap_e, s->spawn_rec,
                                s->spawn_v, s->chunk_count, g));
    CUDAPIC_CHECK(launch_kernel("sens_spawn_scan", sens_spawn_scan_kernel, 1, 1024, 0, st, s->cnt, s->chunk_count,
                                s->chunk_off, s->cap));
    const unsigned nch = (s->cap + SENS_CHUNK - 1) / SENS_CHUNK;
    CUDAPIC_CHECK(launch_kernel("sens_spawn_write", sens_spawn_write_kernel, std::min<unsigned>(nch, 4096u),
                                SENS_CHUNK, 0, st, s->cur[0], s->cur[1], s->cnt, s->chunk_off, s->spawn_rec,
                                s->spawn_v, rec ? s->rec_e : nullptr, s->cap));
    if (ions)
        CUDAPIC_CHECK(launch_kernel("sens_collide_i", sens_collide_i_kernel, gd, SENS_THREADS, 0, st, s->cur[1], s->cnt,
                                    s->st->sigma_tot_i, s->st->cs, rec ? s->rec_i : nullptr, s->rec_cap_i, g));
    return CUDAPIC_OK;
}

int copy_planes(cudapic_sens *s, float *dst, const float *src) {
    return check_cuda(cudaMemcpyAsync(dst, src, sizeof(float) * 16 * (size_t)s->cap, cudaMemcpyDeviceToDevice,
                                      s->stream),
                      "sensitivity plane copy");
}

// Reverse step t (segment step j).
int adj_step(cudapic_sens *s, uint32_t t, uint32_t j, float wP, float wG) {
    cudaStream_t st = s->stream;
    const cudapic_grid &g = s->g;
    const bool ions = ion_step(s, t);
    const size_t cap = s->cap;
    const uint32_t *m0 = s->tmark + 4 * j, *m1 = s->tmark + 4 * (j + 1);
    const unsigned gd = grid_n(s->cap);
    AdjPlanes ae = adj_of(s, 0), ai = adj_of(s, 1);
    if (ions)
        CUDAPIC_CHECK(launch_kernel("sens_adj_collide_i", sens_adj_collide_i_kernel, gd, SENS_THREADS, 0, st, s->rec_i,
                                    m0, m1, s->rec_cap_i, ai.vx, ai.vy, ai.vz));
    CUDAPIC_CHECK(launch_kernel("sens_adj_collide_e", sens_adj_collide_e_kernel, gd, SENS_THREADS, 0, st, s->rec_e, m0,
                                m1, s->rec_cap_e, ae, ai, g));
    const float *E = s->tE + (size_t)j * s->n_g;
    const size_t esm = sizeof(double) * s->n_g;
    CUDAPIC_CHECK(launch_kernel("sens_adj_push", sens_adj_push_kernel, gd, SENS_THREADS, esm, st, s->tx_e + j * cap,
                                s->tv_e + j * cap, m0 + C_NE, E, g.factor_e, g.dt_e, 0, wP, ae.x, ae.vx, s->eb, g));
    const size_t ji = j / s->n_sub;
    if (ions)
        CUDAPIC_CHECK(launch_kernel("sens_adj_push", sens_adj_push_kernel, gd, SENS_THREADS, esm, st,
                                    s->tx_i + ji * cap, s->tv_i + ji * cap, m0 + C_NI, E, g.factor_i, g.dt_i, 1, wG,
                                    ai.x, ai.vx, s->eb, g));
    // the ion-density adjoint gathered at step t + 1 (an ion step) restarts
    CUDAPIC_CHECK(launch_poisson_adjoint(s->eb, s->neb, s->nib_acc, ion_step(s, t + 1) ? 1 : 0, cos_at(s, t), s->vbar,
                                         g, st));
    CUDAPIC_CHECK(launch_kernel("sens_adj_gather", sens_adj_gather_kernel, gd, SENS_THREADS, 0, st, s->tx_e + j * cap,
                                m0 + C_NE, (const double *)s->neb, ae.x, g));
    if (ions)
        CUDAPIC_CHECK(launch_kernel("sens_adj_gather", sens_adj_gather_kernel, gd, SENS_THREADS, 0, st,
                                    s->tx_i + ji * cap, m0 + C_NI, (const double *)s->nib_acc, ai.x, g));
    return CUDAPIC_OK;
}

int read_err(cudapic_sens *s, uint32_t *err) {
    CUDAPIC_CHECK(check_cuda(cudaMemcpyAsync(err, s->cnt + C_ERR, sizeof(uint32_t), cudaMemcpyDeviceToHost, s->stream),
                             "sensitivity error word"));
    return check_cuda(cudaStreamSynchronize(s->stream), "sensitivity sync");
}

}  // namespace

extern "C" int cudapic_sens_create(cudapic_state *st, uint32_t window_steps, uint32_t checkpoint_every,
                                   uint32_t horizon, cudapic_sens **out) {
    if (!st || !out) return fail(CUDAPIC_ERR_ARG, "sens_create: null pointer");
    *out = nullptr;
    const cudapic_params &p = st->params;
    if (window_steps == 0 || checkpoint_every == 0) return fail(CUDAPIC_ERR_ARG, "sens_create: empty window");
    if (checkpoint_every % p.n_sub || window_steps % checkpoint_every)
        return fail(CUDAPIC_ERR_ARG, "sens_create: the window must be whole checkpoint intervals of whole ion cycles");
    if (horizon % checkpoint_every) return fail(CUDAPIC_ERR_ARG, "sens_create: horizon must be whole checkpoint intervals");
    if (p.n_g > SENS_MAX_NG) return fail(CUDAPIC_ERR_ARG, "sens_create: n_g > 4096");
    if (p.flags & CUDAPIC_FLAG_POISSON_F32_SCAN) return fail(CUDAPIC_ERR_ARG, "sens_create: needs the FP64 Poisson sums");
    DeviceGuard dg(st->device);
    if (!dg.ok) return fail(CUDAPIC_ERR_CUDA, "sens_create: cannot select the state's device");
    auto *s = new cudapic_sens();
    s->st = st;
    s->device = st->device;
    s->stream = st->stream;
    s->g = st->grid;
    s->g.dev_err = nullptr;
    s->g.work = nullptr;
    s->cap = p.capacity;
    s->K = window_steps;
    s->S = checkpoint_every;
    s->H = horizon;
    s->n_seg = window_steps / checkpoint_every;
    s->n_g = p.n_g;
    s->n_sub = p.n_sub;
    s->n_t = p.n_t;
    const size_t cap = s->cap;
    s->rec_cap_e = (uint32_t)std::min<uint64_t>(0xFFFFFFF0ull, cap * s->S / 32 + 65536);
    s->rec_cap_i = (uint32_t)std::min<uint64_t>(0xFFFFFFF0ull, cap * (s->S / s->n_sub) / 8 + 65536);
    auto fail_free = [&](int rc) {
        cudapic_sens_destroy(s);
        return rc;
    };
    int rc = CUDAPIC_OK;
    float *init = nullptr, *cur = nullptr;
    if ((rc = sens_alloc_t(s, &init, 16 * cap)) || (rc = sens_alloc_t(s, &cur, 16 * cap)) ||
        (rc = sens_alloc_t(s, &s->cnt, C_COUNT)) || (rc = sens_alloc_t(s, &s->hist, 2 * (size_t)s->n_g)) ||
        (rc = sens_alloc_t(s, &s->dens, 2 * (size_t)s->n_g)) || (rc = sens_alloc_t(s, &s->efield, s->n_g)) ||
        (rc = sens_alloc_t(s, &s->pot, s->n_g)) || (rc = sens_alloc_t(s, &s->obs, 2)) ||
        (rc = sens_alloc_t(s, &s->spawn_rec, cap)) || (rc = sens_alloc_t(s, &s->spawn_v, 6 * cap)) ||
        (rc = sens_alloc_t(s, &s->chunk_count, cap / SENS_CHUNK + 2)) ||
        (rc = sens_alloc_t(s, &s->chunk_off, cap / SENS_CHUNK + 2)) ||
        (rc = sens_alloc_t(s, &s->ckpt, (size_t)s->n_seg * 16 * cap)) ||
        (rc = sens_alloc_t(s, &s->ckpt_cnt, (size_t)s->n_seg * C_COUNT)) ||
        (rc = sens_alloc_t(s, &s->tx_e, (size_t)s->S * cap)) || (rc = sens_alloc_t(s, &s->tv_e, (size_t)s->S * cap)) ||
        (rc = sens_alloc_t(s, &s->tx_i, (size_t)(s->S / s->n_sub) * cap)) ||
        (rc = sens_alloc_t(s, &s->tv_i, (size_t)(s->S / s->n_sub) * cap)) ||
        (rc = sens_alloc_t(s, &s->tE, (size_t)s->S * s->n_g)) ||
        (rc = sens_alloc_t(s, &s->tmark, 4 * ((size_t)s->S + 1))) ||
        (rc = sens_alloc_t(s, &s->rec_e, s->rec_cap_e)) || (rc = sens_alloc_t(s, &s->rec_i, s->rec_cap_i)) ||
        (rc = sens_alloc_t(s, &s->adj, 8 * cap)) || (rc = sens_alloc_t(s, &s->eb, s->n_g)) ||
        (rc = sens_alloc_t(s, &s->neb, s->n_g)) || (rc = sens_alloc_t(s, &s->nib_acc, s->n_g)) ||
        (rc = sens_alloc_t(s, &s->vbar, 1)))
        return fail_free(rc);
    for (int sp = 0; sp < 2; ++sp) {
        s->init[sp] = planes_of(init + (size_t)sp * 8 * cap, s->cap);
        s->cur[sp] = planes_of(cur + (size_t)sp * 8 * cap, s->cap);
    }
    // snapshot of the state's particles and RNG streams (the initial state of every run)
    uint32_t ne = 0, ni = 0;
    if ((rc = cudapic_state_counts(st, &ne, &ni))) return fail_free(rc);
    cudapic_buffers b;
    if ((rc = cudapic_state_buffers(st, &b))) return fail_free(rc);
    s->n_init[0] = ne;
    s->n_init[1] = ni;
    cudaStream_t sm = s->stream;
    for (int sp = 0; sp < 2; ++sp) {
        const Planes &d = s->init[sp];
        const float *src[4] = {b.x[sp], b.vx[sp], b.vy[sp], b.vz[sp]};
        float *dst[4] = {d.x, d.vx, d.vy, d.vz};
        for (int k = 0; k < 4; ++k) {
            if ((rc = check_cuda(cudaMemsetAsync(dst[k], 0, sizeof(float) * cap, sm), "sens init")))
                return fail_free(rc);
            // slots past the live count start dead (x = -1)
            if (k == 0 &&
                (rc = launch_kernel("sens_fill", sens_fill_kernel, grid_n(s->cap), SENS_THREADS, 0, sm, dst[0],
                                    s->cap, -1.0f)))
                return fail_free(rc);
            if (s->n_init[sp] &&
                (rc = check_cuda(cudaMemcpyAsync(dst[k], src[k], sizeof(float) * s->n_init[sp], cudaMemcpyDeviceToDevice,
                                                 sm), "sens init copy")))
                return fail_free(rc);
            if ((rc = check_cuda(cudaMemcpyAsync(d.r[k], b.rng[sp][k], sizeof(uint32_t) * cap, cudaMemcpyDeviceToDevice,
                                                 sm), "sens init rng")))
                return fail_free(rc);
        }
    }
    if ((rc = check_cuda(cudaMemsetAsync(s->spawn_rec, 0xFF, sizeof(uint32_t) * cap, sm), "sens spawn flags")) ||
        (rc = check_cuda(cudaMemsetAsync(s->chunk_count, 0, sizeof(uint32_t) * (cap / SENS_CHUNK + 2), sm), "sens chunks")) ||
        (rc = check_cuda(cudaMemsetAsync(s->hist, 0, sizeof(unsigned long long) * 2 * s->n_g, sm), "sens hist")) ||
        (rc = check_cuda(cudaStreamSynchronize(sm), "sens create sync")))
        return fail_free(rc);
    *out = s;
    return CUDAPIC_OK;
}

extern "C" int cudapic_sens_forward(cudapic_sens *s, double voltage, double obs[2]) {
    if (!s || !obs) return fail(CUDAPIC_ERR_ARG, "sens_forward: null pointer");
    DeviceGuard dg(s->device);
    s->voltage = voltage;
    s->have_forward = false;
    cudaStream_t st = s->stream;
    const size_t cap = s->cap;
    // start: the snapshot (dead slots beyond the live counts)
    CUDAPIC_CHECK(copy_planes(s, s->cur[0].x, s->init[0].x));
    uint32_t c0[C_COUNT] = {s->n_init[0], s->n_init[1], 0, 0, 0, 0, 0, 0};
    CUDAPIC_CHECK(check_cuda(cudaMemcpyAsync(s->cnt, c0, sizeof(c0), cudaMemcpyHostToDevice, st), "sens counters"));
    CUDAPIC_CHECK(check_cuda(cudaMemsetAsync(s->obs, 0, 2 * sizeof(double), st), "sens obs"));
    for (uint32_t t = 0; t < s->K; ++t) {
        if (t % s->S == 0) {
            const uint32_t k = t / s->S;
            CUDAPIC_CHECK(copy_planes(s, s->ckpt + (size_t)k * 16 * cap, s->cur[0].x));
            CUDAPIC_CHECK(check_cuda(cudaMemcpyAsync(s->ckpt_cnt + (size_t)k * C_COUNT, s->cnt, sizeof(uint32_t) * C_COUNT,
                                                     cudaMemcpyDeviceToDevice, st), "sens checkpoint counters"));
        }
        CUDAPIC_CHECK(fwd_step(s, t, false, 0));
    }
    double raw[2];
    CUDAPIC_CHECK(check_cuda(cudaMemcpyAsync(raw, s->obs, sizeof(raw), cudaMemcpyDeviceToHost, st), "sens obs read"));
    uint32_t err = 0;
    CUDAPIC_CHECK(read_err(s, &err));
    double cP, cG;
    obs_scale(s, &cP, &cG);
    obs[0] = cP * raw[0];
    obs[1] = cG * raw[1];
    s->have_forward = true;
    if (err) return fail(CUDAPIC_ERR_CAPACITY, "sens_forward: device error (spawns beyond the capacity)");
    return CUDAPIC_OK;
}

extern "C" int cudapic_sens_backward(cudapic_sens *s, double grad[2]) {
    if (!s || !grad) return fail(CUDAPIC_ERR_ARG, "sens_backward: null pointer");
    if (!s->have_forward) return fail(CUDAPIC_ERR_STATE, "sens_backward: no forward run");
    DeviceGuard dg(s->device);
    cudaStream_t st = s->stream;
    const size_t cap = s->cap;
    double cP, cG;
    obs_scale(s, &cP, &cG);
    for (int o = 0; o < 2; ++o) {
        const float wP = o == 0 ? (float)cP : 0.0f, wG = o == 1 ? (float)cG : 0.0f;
        CUDAPIC_CHECK(check_cuda(cudaMemsetAsync(s->adj, 0, sizeof(float) * 8 * cap, st), "sens adjoint"));
        CUDAPIC_CHECK(check_cuda(cudaMemsetAsync(s->eb, 0, sizeof(double) * s->n_g, st), "sens eb"));
        CUDAPIC_CHECK(check_cuda(cudaMemsetAsync(s->nib_acc, 0, sizeof(double) * s->n_g, st), "sens nib"));
        CUDAPIC_CHECK(check_cuda(cudaMemsetAsync(s->vbar, 0, sizeof(double), st), "sens vbar"));
        for (int64_t k = (int64_t)s->n_seg - 1; k >= 0; --k) {
            const uint32_t t0 = (uint32_t)k * s->S;
            if (s->H && (t0 + s->S) % s->H == 0)  // a horizon ends after this segment: the adjoint restarts
                CUDAPIC_CHECK(check_cuda(cudaMemsetAsync(s->adj, 0, sizeof(float) * 8 * cap, st), "sens horizon"));
            // recompute the segment from its checkpoint, recording the tape
            CUDAPIC_CHECK(copy_planes(s, s->cur[0].x, s->ckpt + (size_t)k * 16 * cap));
            CUDAPIC_CHECK(check_cuda(cudaMemcpyAsync(s->cnt, s->ckpt_cnt + (size_t)k * C_COUNT, sizeof(uint32_t) * C_COUNT,
                                                     cudaMemcpyDeviceToDevice, st), "sens restore counters"));
            CUDAPIC_CHECK(check_cuda(cudaMemsetAsync(s->cnt + C_REC_E, 0, 2 * sizeof(uint32_t), st), "sens records"));
            for (uint32_t j = 0; j < s->S; ++j) CUDAPIC_CHECK(fwd_step(s, t0 + j, true, j));
            CUDAPIC_CHECK(launch_kernel("sens_mark", sens_mark_kernel, 1, 32, 0, st, s->cnt, s->tmark + 4 * s->S));
            for (int64_t j = (int64_t)s->S - 1; j >= 0; --j)
                CUDAPIC_CHECK(adj_step(s, t0 + (uint32_t)j, (uint32_t)j, wP, wG));
        }
        CUDAPIC_CHECK(check_cuda(cudaMemcpyAsync(&grad[o], s->vbar, sizeof(double), cudaMemcpyDeviceToHost, st),
                                 "sens gradient read"));
        uint32_t err = 0;
        CUDAPIC_CHECK(read_err(s, &err));
        if (err & CUDAPIC_DEVERR_RECORDS) return fail(CUDAPIC_ERR_CAPACITY, "sens_backward: collision records overflowed");
        if (err) return fail(CUDAPIC_ERR_CAPACITY, "sens_backward: device error (spawns beyond the capacity)");
    }
    return CUDAPIC_OK;
}

extern "C" int cudapic_sens_info(cudapic_sens *s, uint32_t counts[2], uint32_t *dev_err, uint64_t *device_bytes) {
    if (!s) return fail(CUDAPIC_ERR_ARG, "sens_info: null pointer");
    DeviceGuard dg(s->device);
    uint32_t c[C_COUNT];
    CUDAPIC_CHECK(check_cuda(cudaMemcpyAsync(c, s->cnt, sizeof(c), cudaMemcpyDeviceToHost, s->stream), "sens info"));
    CUDAPIC_CHECK(check_cuda(cudaStreamSynchronize(s->stream), "sens info sync"));
    if (counts) {
        counts[0] = c[C_NE];
        counts[1] = c[C_NI];
    }
    if (dev_err) *dev_err = c[C_ERR];
    if (device_bytes) *device_bytes = s->bytes;
    return CUDAPIC_OK;
}

extern "C" int cudapic_sens_download(cudapic_sens *s, int species, float *x, float *vx, float *vy, float *vz,
                                     uint32_t *rng, uint32_t capacity) {
    if (!s || species < 0 || species > 1 || !x || !vx || !vy || !vz)
        return fail(CUDAPIC_ERR_ARG, "sens_download: bad arguments");
    if (capacity < s->cap) return fail(CUDAPIC_ERR_ARG, "sens_download: host buffers smaller than the capacity");
    DeviceGuard dg(s->device);
    const Planes &p = s->cur[species];
    float *dst[4] = {x, vx, vy, vz};
    const float *src[4] = {p.x, p.vx, p.vy, p.vz};
    for (int k = 0; k < 4; ++k)
        CUDAPIC_CHECK(check_cuda(cudaMemcpyAsync(dst[k], src[k], sizeof(float) * s->cap, cudaMemcpyDeviceToHost, s->stream),
                                 "sens download"));
    if (rng)
        for (int k = 0; k < 4; ++k)
            CUDAPIC_CHECK(check_cuda(cudaMemcpyAsync(rng + (size_t)k * s->cap, p.r[k], sizeof(uint32_t) * s->cap,
                                                     cudaMemcpyDeviceToHost, s->stream), "sens download rng"));
    return check_cuda(cudaStreamSynchronize(s->stream), "sens download sync");
}

extern "C" int cudapic_sens_destroy(cudapic_sens *s) {
    if (!s) return CUDAPIC_OK;
    DeviceGuard dg(s->device);
    if (s->stream) cudaStreamSynchronize(s->stream);
    for (void *p : s->allocs) cudaFree(p);
    delete s;
    return CUDAPIC_OK;
}
