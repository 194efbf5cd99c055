// kernels_mcc.cu -- Monte-Carlo collisions of electrons and ions.
//
// Reference: check_collisions_e / collision_e, Rust-CUDA/src/main.rs:971-1165,
// check_collisions_i / collision_i, :1167-1292.  Per electron: energy index
// min(int(E/1 meV + 0.5), 1e6-1), nu = sigma_tot(E) |v|, collide iff
// u < 1 - exp(-nu dt); the type (elastic / excitation / ionization) from
// the cumulative cross-section ratios; Euler-angle rotation of the relative
// velocity; ionization spawns an electron and an ion.  Per ion: a Maxwellian
// target atom (Box-Muller), relative energy, isotropic or backward
// scattering.  The RNG draw order of the reference is kept exactly.
//
// B200 design: HBM-bound streaming (28 B read + 16 B RNG written per
// particle, velocities written only by colliders, ~1-5 % per step):
//  * persistent grid-stride loop, one particle per thread and iteration,
//    coalesced SoA loads; the RNG state is held in registers for all draws;
//  * sigma_tot gathers through the read-only path (__ldg: L1 / 126 MB L2
//    resident 4 MB table); the per-process tables only for colliders;
//  * ionization spawns claim slots with one warp-aggregated atomicAdd per
//    counter (coalesced group of the ionizing lanes), bounded by capacity:
//    a spawn that does not fit is dropped and flagged, never written
//    out of bounds (the reference writes unbounded, :1132-1149);
//  * transcendentals from detmath.cuh (bit-reproducible, see there).
#include <cooperative_groups.h>

#include "common.cuh"
#include "detmath.cuh"
#include "internal.h"
#include "rng.cuh"

namespace cg = cooperative_groups;

namespace cudapic {

constexpr int MCC_THREADS = 256;

__device__ __forceinline__ uint32_t energy_index(float energy) {
    float t = fminf(energy / DE_CS_F + 0.5f, (float)(CS_RANGES - 1));
    return (uint32_t)t;
}

struct Euler {
    float st, ct, sp, cp;
};

// Euler angles of (gx, gy, gz), Rust-CUDA/src/main.rs:1066-1090.
__device__ __forceinline__ Euler euler_angles(float gx, float gy, float gz) {
    float theta, phi;
    if (gx == 0.0f) theta = 0.5f * PI_F;
    else theta = dm::atan2f_det(sqrtf(gy * gy + gz * gz), gx);
    if (gy == 0.0f) phi = (gz > 0.0f) ? 0.5f * PI_F : -0.5f * PI_F;
    else phi = dm::atan2f_det(gz, gy);
    Euler e;
    dm::sincosf_det(theta, &e.st, &e.ct);
    dm::sincosf_det(phi, &e.sp, &e.cp);
    return e;
}

// Scattered relative velocity, Rust-CUDA/src/main.rs:1152-1158.
__device__ __forceinline__ void rotate(float g, float sc, float cc, float se, float ce, const Euler &a, float &gx,
                                       float &gy, float &gz) {
    gx = g * (a.ct * cc - a.st * sc * ce);
    gy = g * (a.st * a.cp * cc + a.ct * a.cp * sc * ce - a.sp * sc * se);
    gz = g * (a.st * a.sp * cc + a.ct * a.sp * sc * ce + a.cp * sc * se);
}

// Claims one slot of `counter` for every lane of the calling coalesced
// group with a single atomicAdd; never hands out a slot >= capacity.
__device__ __forceinline__ bool claim_slot(uint32_t *counter, uint32_t capacity, uint32_t &slot) {
    cg::coalesced_group grp = cg::coalesced_threads();
    uint32_t base = 0, granted = 0;
    if (grp.thread_rank() == 0) {
        const uint32_t cnt = grp.size();
        const uint32_t old = atomicAdd(counter, cnt);
        granted = old >= capacity ? 0u : min(cnt, capacity - old);
        if (granted < cnt) atomicSub(counter, cnt - granted);
        base = old;
    }
    base = grp.shfl(base, 0);
    granted = grp.shfl(granted, 0);
    slot = base + grp.thread_rank();
    return grp.thread_rank() < granted;
}

template <bool EVENTS>
__global__ void __launch_bounds__(MCC_THREADS)
    check_collisions_e_kernel(const float *__restrict__ sigma_tot_e, const float *__restrict__ cs,
                              const uint32_t *__restrict__ active_e, float *__restrict__ x,
                              float *__restrict__ vx, float *__restrict__ vy, float *__restrict__ vz,
                              uint32_t *__restrict__ rng0, uint32_t *__restrict__ rng1,
                              uint32_t *__restrict__ rng2, uint32_t *__restrict__ rng3,
                              float *__restrict__ ix, float *__restrict__ ivx, float *__restrict__ ivy,
                              float *__restrict__ ivz, uint32_t *__restrict__ alive_e,
                              uint32_t *__restrict__ alive_i, uint8_t *__restrict__ events,
                              const cudapic_grid g) {
    const uint32_t n = load_count(active_e, g.capacity, g.dev_err);
    const uint32_t stride = gridDim.x * MCC_THREADS;
    const float exc_j = 11.5f * E_CHARGE_F;
    const float ion_j = 15.8f * E_CHARGE_F;
    for (uint32_t i = blockIdx.x * MCC_THREADS + threadIdx.x; i < n; i += stride) {
        Xoshiro128p rs{rng0[i], rng1[i], rng2[i], rng3[i]};
        const float vxi = vx[i], vyi = vy[i], vzi = vz[i];
        const float v2 = vxi * vxi + vyi * vyi + vzi * vzi;
        const float energy = g.half_me_over_e * v2;
        const uint32_t idx = energy_index(energy);
        const float velocity = sqrtf(v2);
        const float nu = __ldg(sigma_tot_e + idx) * velocity;
        const float rand_val = rs.uniform();
        const float p_coll = 1.0f - dm::expf_det(-nu * g.dt_e);
        uint8_t ev = 0;
        if (rand_val < p_coll) {
            float gx = vxi, gy = vyi, gz = vzi;
            float gm = sqrtf(gx * gx + gy * gy + gz * gz);
            const float wx = g.f1 * vxi, wy = g.f1 * vyi, wz = g.f1 * vzi;
            const float t0 = __ldg(cs + idx);
            const float t1 = t0 + __ldg(cs + CS_RANGES + idx);
            const float t2 = t1 + __ldg(cs + 2 * CS_RANGES + idx);
            const Euler eu = euler_angles(gx, gy, gz);
            float chi_s, chi_c, eta;
            const float rnd = rs.uniform();
            if (rnd < t0 / t2) {
                ev = 1;  // elastic
                const float chi = dm::acosf_det(1.0f - 2.0f * rs.uniform());
                eta = TWO_PI_F * rs.uniform();
                dm::sincosf_det(chi, &chi_s, &chi_c);
            } else if (rnd < t1 / t2) {
                ev = 2;  // excitation
                float en = 0.5f * E_MASS_F * gm * gm;
                en = fabsf(en - exc_j);
                gm = sqrtf(2.0f * en / E_MASS_F);
                const float chi = dm::acosf_det(1.0f - 2.0f * rs.uniform());
                eta = TWO_PI_F * rs.uniform();
                dm::sincosf_det(chi, &chi_s, &chi_c);
            } else {
                ev = 3;  // ionization
                float en = 0.5f * E_MASS_F * gm * gm;
                en = fabsf(en - ion_j);
                const float e_new = 10.0f * dm::tanf_det(rs.uniform() * dm::atanf_det(en / E_CHARGE_F / 20.0f)) *
                                    E_CHARGE_F;
                const float e_orig = fabsf(en - e_new);
                gm = sqrtf(2.0f * e_orig / E_MASS_F);
                const float g_new = sqrtf(2.0f * e_new / E_MASS_F);
                const float chi = dm::acosf_det(sqrtf(e_orig / en));
                const float chi_new = dm::acosf_det(sqrtf(e_new / en));
                eta = TWO_PI_F * rs.uniform();
                const float eta_new = eta + PI_F;
                float sc2, cc2, se2, ce2;
                dm::sincosf_det(chi_new, &sc2, &cc2);
                dm::sincosf_det(eta_new, &se2, &ce2);
                float ngx, ngy, ngz;
                rotate(g_new, sc2, cc2, se2, ce2, eu, ngx, ngy, ngz);
                const float xi = x[i];
                uint32_t slot;
                if (claim_slot(alive_e, g.capacity, slot)) {
                    x[slot] = xi;
                    vx[slot] = wx + g.f2 * ngx;
                    vy[slot] = wy + g.f2 * ngy;
                    vz[slot] = wz + g.f2 * ngz;
                } else {
                    set_dev_err(g.dev_err, CUDAPIC_DEVERR_SPAWN_E);
                }
                float a, b, c;
                rs.three_normal(g.normal_range, a, b, c);
                if (claim_slot(alive_i, g.capacity, slot)) {
                    ix[slot] = xi;
                    ivx[slot] = a;
                    ivy[slot] = b;
                    ivz[slot] = c;
                } else {
                    set_dev_err(g.dev_err, CUDAPIC_DEVERR_SPAWN_I);
                }
                dm::sincosf_det(chi, &chi_s, &chi_c);
            }
            float se, ce;
            dm::sincosf_det(eta, &se, &ce);
            float ngx, ngy, ngz;
            rotate(gm, chi_s, chi_c, se, ce, eu, ngx, ngy, ngz);
            vx[i] = wx + g.f2 * ngx;
            vy[i] = wy + g.f2 * ngy;
            vz[i] = wz + g.f2 * ngz;
        }
        rng0[i] = rs.s0;
        rng1[i] = rs.s1;
        rng2[i] = rs.s2;
        rng3[i] = rs.s3;
        if (EVENTS) events[i] = ev;
    }
}

template <bool EVENTS>
__global__ void __launch_bounds__(MCC_THREADS)
    check_collisions_i_kernel(const float *__restrict__ sigma_tot_i, const float *__restrict__ cs,
                              const uint32_t *__restrict__ active_i, float *__restrict__ vx,
                              float *__restrict__ vy, float *__restrict__ vz, uint32_t *__restrict__ rng0,
                              uint32_t *__restrict__ rng1, uint32_t *__restrict__ rng2,
                              uint32_t *__restrict__ rng3, uint8_t *__restrict__ events, const cudapic_grid g) {
    const uint32_t n = load_count(active_i, g.capacity, g.dev_err);
    const uint32_t stride = gridDim.x * MCC_THREADS;
    for (uint32_t i = blockIdx.x * MCC_THREADS + threadIdx.x; i < n; i += stride) {
        Xoshiro128p rs{rng0[i], rng1[i], rng2[i], rng3[i]};
        float vxa, vya, vza;
        rs.three_normal(g.normal_range, vxa, vya, vza);
        const float vxi = vx[i], vyi = vy[i], vzi = vz[i];
        const float gx = vxi - vxa, gy = vyi - vya, gz = vzi - vza;
        const float g2 = gx * gx + gy * gy + gz * gz;
        const float energy = g.half_mu_over_e * g2;
        const uint32_t idx = energy_index(energy);
        const float gmag = sqrtf(g2);
        const float nu = __ldg(sigma_tot_i + idx) * gmag;
        const float rand_val = rs.uniform();
        const float p_coll = 1.0f - dm::expf_det(-nu * g.dt_i);
        uint8_t ev = 0;
        if (rand_val < p_coll) {
            const float t0 = __ldg(cs + 3 * CS_RANGES + idx);
            const float t1 = t0 + __ldg(cs + 4 * CS_RANGES + idx);
            const float gg = sqrtf(gx * gx + gy * gy + gz * gz);
            const float wx = 0.5f * (vxi + vxa), wy = 0.5f * (vyi + vya), wz = 0.5f * (vzi + vza);
            const Euler eu = euler_angles(gx, gy, gz);
            const float rnd = rs.uniform();
            float chi;
            if (rnd < t0 / t1) {
                ev = 4;
                chi = dm::acosf_det(1.0f - 2.0f * rs.uniform());
            } else {
                ev = 5;
                chi = PI_F;
            }
            const float eta = TWO_PI_F * rs.uniform();
            float sc, cc, se, ce;
            dm::sincosf_det(chi, &sc, &cc);
            dm::sincosf_det(eta, &se, &ce);
            float ngx, ngy, ngz;
            rotate(gg, sc, cc, se, ce, eu, ngx, ngy, ngz);
            vx[i] = wx + 0.5f * ngx;
            vy[i] = wy + 0.5f * ngy;
            vz[i] = wz + 0.5f * ngz;
        }
        rng0[i] = rs.s0;
        rng1[i] = rs.s1;
        rng2[i] = rs.s2;
        rng3[i] = rs.s3;
        if (EVENTS) events[i] = ev;
    }
}

// accumulate_eepf, Rust-CUDA/src/main.rs:1301-1339: per-block shared
// histogram, one global atomic per non-empty bin and block.
__global__ void __launch_bounds__(256)
    accumulate_eepf_kernel(const float *__restrict__ x, const float *__restrict__ vx, const float *__restrict__ vy,
                           const float *__restrict__ vz, const float *__restrict__ efield,
                           const uint32_t *__restrict__ active_e, uint32_t *__restrict__ eepf,
                           const cudapic_grid g) {
    __shared__ uint32_t h[N_EEPF];
    for (uint32_t k = threadIdx.x; k < N_EEPF; k += blockDim.x) h[k] = 0;
    __syncthreads();
    const uint32_t n = load_count(active_e, g.capacity, g.dev_err);
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const float xi = x[i];
        if (xi <= g.min_x || xi >= g.max_x) continue;
        const float pos = xi * g.inv_dx;
        const int p = cell_of(pos, g.n_g);
        const float c2 = pos - (float)p;
        const float e_x = (1.0f - c2) * __ldg(efield + p) + c2 * __ldg(efield + p + 1);
        const float mvx = vx[i] - 0.5f * e_x * g.eepf_half_kick;
        const float vyi = vy[i], vzi = vz[i];
        const float v2 = mvx * mvx + vyi * vyi + vzi * vzi;
        const float energy = g.half_me_over_e * v2;
        const float binf = energy / DE_EEPF_F;
        if (binf < (float)N_EEPF) atomicAdd(&h[(uint32_t)binf], 1u);
    }
    __syncthreads();
    for (uint32_t k = threadIdx.x; k < N_EEPF; k += blockDim.x)
        if (h[k]) atomicAdd(&eepf[k], h[k]);
}

int mcc_grid(uint32_t capacity, const void *kernel) {
    int per_sm = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, MCC_THREADS, 0) != cudaSuccess) per_sm = 4;
    per_sm = std::max(per_sm, 1);
    const uint64_t need = ((uint64_t)capacity + MCC_THREADS - 1) / MCC_THREADS;
    return (int)std::max<uint64_t>(1, std::min<uint64_t>((uint64_t)sm_count() * per_sm, need));
}

int launch_collisions_e(const float *total_cs_e, const float *cs, const uint32_t *active_e, float *x, float *vx,
                        float *vy, float *vz, uint32_t *rng0, uint32_t *rng1, uint32_t *rng2, uint32_t *rng3,
                        float *i_x, float *i_vx, float *i_vy, float *i_vz, uint32_t *alive_e, uint32_t *alive_i,
                        uint8_t *events, const cudapic_grid &g, cudaStream_t stream) {
    if (events) {
        auto k = check_collisions_e_kernel<true>;
        k<<<mcc_grid(g.capacity, (const void *)k), MCC_THREADS, 0, stream>>>(
            total_cs_e, cs, active_e, x, vx, vy, vz, rng0, rng1, rng2, rng3, i_x, i_vx, i_vy, i_vz, alive_e,
            alive_i, events, g);
    } else {
        auto k = check_collisions_e_kernel<false>;
        k<<<mcc_grid(g.capacity, (const void *)k), MCC_THREADS, 0, stream>>>(
            total_cs_e, cs, active_e, x, vx, vy, vz, rng0, rng1, rng2, rng3, i_x, i_vx, i_vy, i_vz, alive_e,
            alive_i, nullptr, g);
    }
    return check_launch("check_collisions_e");
}

int launch_collisions_i(const float *total_cs_i, const float *cs, const uint32_t *active_i, float *vx, float *vy,
                        float *vz, uint32_t *rng0, uint32_t *rng1, uint32_t *rng2, uint32_t *rng3, uint8_t *events,
                        const cudapic_grid &g, cudaStream_t stream) {
    if (events) {
        auto k = check_collisions_i_kernel<true>;
        k<<<mcc_grid(g.capacity, (const void *)k), MCC_THREADS, 0, stream>>>(total_cs_i, cs, active_i, vx, vy, vz,
                                                                               rng0, rng1, rng2, rng3, events, g);
    } else {
        auto k = check_collisions_i_kernel<false>;
        k<<<mcc_grid(g.capacity, (const void *)k), MCC_THREADS, 0, stream>>>(total_cs_i, cs, active_i, vx, vy, vz,
                                                                               rng0, rng1, rng2, rng3, nullptr, g);
    }
    return check_launch("check_collisions_i");
}

int launch_eepf(const float *x, const float *vx, const float *vy, const float *vz, const float *efield,
                const uint32_t *active_e, uint32_t *eepf, const cudapic_grid &g, cudaStream_t stream) {
    const uint64_t need = ((uint64_t)g.capacity + 255) / 256;
    const unsigned grid = (unsigned)std::max<uint64_t>(1, std::min<uint64_t>((uint64_t)sm_count() * 2, need));
    accumulate_eepf_kernel<<<grid, 256, 0, stream>>>(x, vx, vy, vz, efield, active_e, eepf, g);
    return check_launch("accumulate_eepf");
}

}  // namespace cudapic

using namespace cudapic;

#define CUDAPIC_E_ARGS_NONNULL                                                                              \
    (total_cs_e && cs && active_e && x && vx && vy && vz && rng0 && rng1 && rng2 && rng3 && i_x && i_vx && \
     i_vy && i_vz && alive_e && alive_i)

extern "C" int cudapic_check_collisions_e(const float *total_cs_e, const float *cs, const uint32_t *active_e,
                                          float *x, float *vx, float *vy, float *vz, uint32_t *rng0,
                                          uint32_t *rng1, uint32_t *rng2, uint32_t *rng3, float *i_x, float *i_vx,
                                          float *i_vy, float *i_vz, uint32_t *alive_e, uint32_t *alive_i,
                                          const cudapic_grid *grid, cudapic_stream_t stream) {
    CUDAPIC_CHECK(validate_grid(grid));
    CUDAPIC_REQUIRE(CUDAPIC_E_ARGS_NONNULL, "check_collisions_e: null pointer");
    return launch_collisions_e(total_cs_e, cs, active_e, x, vx, vy, vz, rng0, rng1, rng2, rng3, i_x, i_vx, i_vy,
                               i_vz, alive_e, alive_i, nullptr, *grid, (cudaStream_t)stream);
}

extern "C" int cudapic_check_collisions_e_events(const float *total_cs_e, const float *cs,
                                                 const uint32_t *active_e, float *x, float *vx, float *vy,
                                                 float *vz, uint32_t *rng0, uint32_t *rng1, uint32_t *rng2,
                                                 uint32_t *rng3, float *i_x, float *i_vx, float *i_vy,
                                                 float *i_vz, uint32_t *alive_e, uint32_t *alive_i,
                                                 uint8_t *events, const cudapic_grid *grid,
                                                 cudapic_stream_t stream) {
    CUDAPIC_CHECK(validate_grid(grid));
    CUDAPIC_REQUIRE(CUDAPIC_E_ARGS_NONNULL && events, "check_collisions_e_events: null pointer");
    return launch_collisions_e(total_cs_e, cs, active_e, x, vx, vy, vz, rng0, rng1, rng2, rng3, i_x, i_vx, i_vy,
                               i_vz, alive_e, alive_i, events, *grid, (cudaStream_t)stream);
}

extern "C" int cudapic_check_collisions_i(const float *total_cs_i, const float *cs, const uint32_t *active_i,
                                          float *vx, float *vy, float *vz, uint32_t *rng0, uint32_t *rng1,
                                          uint32_t *rng2, uint32_t *rng3, const cudapic_grid *grid,
                                          cudapic_stream_t stream) {
    CUDAPIC_CHECK(validate_grid(grid));
    CUDAPIC_REQUIRE(total_cs_i && cs && active_i && vx && vy && vz && rng0 && rng1 && rng2 && rng3,
                    "check_collisions_i: null pointer");
    return launch_collisions_i(total_cs_i, cs, active_i, vx, vy, vz, rng0, rng1, rng2, rng3, nullptr, *grid,
                               (cudaStream_t)stream);
}

extern "C" int cudapic_check_collisions_i_events(const float *total_cs_i, const float *cs,
                                                 const uint32_t *active_i, float *vx, float *vy, float *vz,
                                                 uint32_t *rng0, uint32_t *rng1, uint32_t *rng2, uint32_t *rng3,
                                                 uint8_t *events, const cudapic_grid *grid,
                                                 cudapic_stream_t stream) {
    CUDAPIC_CHECK(validate_grid(grid));
    CUDAPIC_REQUIRE(total_cs_i && cs && active_i && vx && vy && vz && rng0 && rng1 && rng2 && rng3 && events,
                    "check_collisions_i_events: null pointer");
    return launch_collisions_i(total_cs_i, cs, active_i, vx, vy, vz, rng0, rng1, rng2, rng3, events, *grid,
                               (cudaStream_t)stream);
}

extern "C" int cudapic_accumulate_eepf(const float *x, const float *vx, const float *vy, const float *vz,
                                       const float *efield, const uint32_t *active_e, uint32_t *eepf,
                                       const cudapic_grid *grid, cudapic_stream_t stream) {
    CUDAPIC_CHECK(validate_grid(grid));
    CUDAPIC_REQUIRE(x && vx && vy && vz && efield && active_e && eepf, "accumulate_eepf: null pointer");
    return launch_eepf(x, vx, vy, vz, efield, active_e, eepf, *grid, (cudaStream_t)stream);
}
