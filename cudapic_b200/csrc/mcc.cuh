// mcc.cuh -- Monte-Carlo collision physics shared by the collision kernels
// (kernels_mcc.cu) and the fused electron step (kernels_step.cu).
//
// Reference: check_collisions_e / collision_e, Rust-CUDA/src/main.rs:971-1165,
// check_collisions_i / collision_i, :1167-1292.  The RNG draw order of the
// reference is kept exactly; transcendentals come from detmath.cuh.
#pragma once
#include <cooperative_groups.h>

#include "common.cuh"
#include "detmath.cuh"
#include "rng.cuh"

namespace cudapic {

namespace cg = cooperative_groups;

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

// The same angles' sines and cosines from their exact algebraic forms,
// without the angles: sin theta = r / |g|, cos theta = gx / |g| with
// r = sqrt(gy^2 + gz^2), and sin phi = gz / r, cos phi = gy / r (the special
// cases gx = 0 and gy = 0 as above, with cos(+-pi/2) = 0 exactly).  Equal to
// euler_angles up to the rounding of the transcendentals it skips.
__device__ __forceinline__ Euler euler_angles_alg(float gx, float gy, float gz) {
    Euler e;
    const float r2 = gy * gy + gz * gz;
    const float r = sqrtf(r2);
    if (gx == 0.0f) {
        e.st = 1.0f;
        e.ct = 0.0f;
    } else {
        const float gn = sqrtf(gx * gx + r2);
        e.st = r / gn;
        e.ct = gx / gn;
    }
    if (gy == 0.0f) {
        e.sp = (gz > 0.0f) ? 1.0f : -1.0f;
        e.cp = 0.0f;
    } else {
        e.sp = gz / r;
        e.cp = gy / r;
    }
    return e;
}

// sin and cos of acos(c), c in [-1, 1]: sqrt((1 - c)(1 + c)) and c.
__device__ __forceinline__ void sincos_of_acos(float c, float *s, float *co) {
    *s = sqrtf(fmaxf(0.0f, (1.0f - c) * (1.0f + c)));
    *co = c;
}

// Scattered relative velocity, Rust-CUDA/src/main.rs:1152-1158.
__device__ __forceinline__ void rotate(float g, float sc, float cc, float se, float ce, const Euler &a, float &gx,
                                       float &gy, float &gz) {
    gx = g * (a.ct * cc - a.st * sc * ce);
    gy = g * (a.st * a.cp * cc + a.ct * a.cp * sc * ce - a.sp * sc * se);
    gz = g * (a.st * a.sp * cc + a.ct * a.sp * sc * ce + a.cp * sc * se);
}

// Claims one slot of `counter` for every lane that reaches it together
// with the same counter, one atomicAdd per such group (lanes of a warp that
// scatter for different discharges of a batch form separate groups; within
// a group, lanes take consecutive slots in lane order); never hands out a
// slot >= capacity (the same capacity for every lane of a group).
__device__ __forceinline__ bool claim_slot(uint32_t *counter, uint32_t capacity, uint32_t &slot) {
    const unsigned active = __activemask();
    const unsigned peers = __match_any_sync(active, reinterpret_cast<unsigned long long>(counter));
    const int leader = __ffs(peers) - 1;
    const uint32_t rank = __popc(peers & lanemask_lt());
    uint32_t base = 0, granted = 0;
    if ((int)(threadIdx.x & 31u) == leader) {
        const uint32_t cnt = __popc(peers);
        const uint32_t old = atomicAdd(counter, cnt);
        granted = old >= capacity ? 0u : min(cnt, capacity - old);
        if (granted < cnt) atomicSub(counter, cnt - granted);
        base = old;
    }
    base = __shfl_sync(peers, base, leader);
    granted = __shfl_sync(peers, granted, leader);
    slot = base + rank;
    return rank < granted;
}

// Collision decision u < p with p = 1 - exp(-a), a = nu dt (the reference
// evaluates exp(-nu * dt) with -nu * dt == -(nu * dt) exactly,
// Rust-CUDA/src/main.rs:1011, 1196).  Since 1 - e^-a <= a, exp_det is
// within 2 ulp and 1 - y is exact for y >= 1/2, the computed p never
// exceeds a + 3.1e-7: any u >= fl(a + 5e-7) is a certain "no collision",
// decided without evaluating exp (about 99 % of draws at the reference
// conditions).  The decision is bit-identical to the full test.
__device__ __forceinline__ bool collision_draw(float u, float a) {
    if (u >= a + 5e-7f) return false;
    const float p_coll = 1.0f - dm::expf_det(-a);
    return u < p_coll;
}

// Outcome of the collision test of one particle.
struct Test {
    uint32_t idx;
    bool collide;
};

// sigma_tot lookups: straight from the global table (read-only path), or
// from a shared-memory copy of its first `resident` entries.
struct GlobalTable {
    const float *__restrict__ t;
    __device__ __forceinline__ float operator()(uint32_t idx) const { return __ldg(t + idx); }
};
struct ResidentTable {
    const float *__restrict__ t;   // global table
    const float *s;                // shared copy of t[0 .. resident)
    uint32_t resident;
    __device__ __forceinline__ float operator()(uint32_t idx) const {
        return idx < resident ? s[idx] : __ldg(t + idx);
    }
};

// Electron collision test, Rust-CUDA/src/main.rs:992-1012 (one draw).
template <typename Table>
__device__ __forceinline__ Test test_electron(float vxi, float vyi, float vzi, Xoshiro128p &rs,
                                              const Table &sigma_tot_e, const cudapic_grid &g) {
    const float v2 = vxi * vxi + vyi * vyi + vzi * vzi;
    const float energy = g.half_me_over_e * v2;
    Test t;
    t.idx = energy_index(energy);
    const float velocity = sqrtf(v2);
    const float nu = sigma_tot_e(t.idx) * velocity;
    const float rand_val = rs.uniform();
    t.collide = collision_draw(rand_val, nu * g.dt_e);
    return t;
}

// CIC deposit of one particle straight into a global density (boundary
// nodes doubled per contribution, equal to doubling the node sum).
__device__ __forceinline__ void deposit_global(float *dens, float xv, const cudapic_grid &g) {
    const float pos = xv * g.inv_dx;
    const int p = cell_of(pos, g.n_g);
    const float rem = pos - (float)p;
    float c1 = (1.0f - rem) * g.weight_factor;
    float c2 = rem * g.weight_factor;
    if (p == 0) c1 *= 2.0f;
    if (p + 1 == (int)g.n_g - 1) c2 *= 2.0f;
    atomicAdd(&dens[p], c1);
    atomicAdd(&dens[p + 1], c2);
}

// collision_e, Rust-CUDA/src/main.rs:1035-1165: scatters electron i (state
// rs already past the test draw), writes its velocity and any spawns;
// returns the event (1 elastic, 2 excitation, 3 ionization).  dep_e / dep_i
// (may be null): next-step densities that also receive the spawned
// electron / ion.  Slots (i and the spawns' claimed slots) are relative to
// element `off` of the planes (a discharge of a batch's pool; 0 otherwise).
// ALG: the sines and cosines of the Euler angles, of the scattering angles
// chi = acos(c) and of eta + pi from their algebraic forms (euler_angles_alg,
// sincos_of_acos, sin(eta + pi) = -sin eta) instead of evaluating the
// angles: the same draws and events, velocities equal up to the rounding of
// the skipped transcendentals, a fraction of the arithmetic.
// XPRE: the caller passes the electron's position as xpre (loaded ahead,
// alongside its other loads); else an ionization loads x[off + i] itself.
template <bool ALG, bool XPRE>
__device__ __forceinline__ uint32_t collide_electron_body(uint32_t off, uint32_t i, uint32_t idx, float vxi,
                                                          float vyi, float vzi, Xoshiro128p &rs,
                                                          const float *__restrict__ cs, float *x, float *vx,
                                                          float *vy, float *vz, float *ix, float *ivx, float *ivy,
                                                          float *ivz, uint32_t *alive_e, uint32_t *alive_i,
                                                          const cudapic_grid &g, float *dep_e, float *dep_i,
                                                          float xpre) {
    const float exc_j = 11.5f * E_CHARGE_F;
    const float ion_j = 15.8f * E_CHARGE_F;
    float gx = vxi, gy = vyi, gz = vzi;
    float gm = sqrtf(gx * gx + gy * gy + gz * gz);
    const float wx = g.f1 * vxi, wy = g.f1 * vyi, wz = g.f1 * vzi;
    const float t0 = __ldg(cs + idx);
    const float t1 = t0 + __ldg(cs + CS_RANGES + idx);
    const float t2 = t1 + __ldg(cs + 2 * CS_RANGES + idx);
    const Euler eu = ALG ? euler_angles_alg(gx, gy, gz) : euler_angles(gx, gy, gz);
    float chi_s, chi_c, eta, se, ce;
    uint32_t ev;
    const float rnd = rs.uniform();
    if (rnd < t0 / t2) {
        ev = 1;  // elastic
        const float c = 1.0f - 2.0f * rs.uniform();
        eta = TWO_PI_F * rs.uniform();
        if (ALG) sincos_of_acos(c, &chi_s, &chi_c);
        else dm::sincosf_det(dm::acosf_det(c), &chi_s, &chi_c);
    } else if (rnd < t1 / t2) {
        ev = 2;  // excitation
        float en = 0.5f * E_MASS_F * gm * gm;
        en = fabsf(en - exc_j);
        gm = sqrtf(2.0f * en / E_MASS_F);
        const float c = 1.0f - 2.0f * rs.uniform();
        eta = TWO_PI_F * rs.uniform();
        if (ALG) sincos_of_acos(c, &chi_s, &chi_c);
        else dm::sincosf_det(dm::acosf_det(c), &chi_s, &chi_c);
    } else {
        ev = 3;  // ionization
        float en = 0.5f * E_MASS_F * gm * gm;
        en = fabsf(en - ion_j);
        const float e_new =
            10.0f * dm::tanf_det(rs.uniform() * dm::atanf_det(en / E_CHARGE_F / 20.0f)) * E_CHARGE_F;
        const float e_orig = fabsf(en - e_new);
        gm = sqrtf(2.0f * e_orig / E_MASS_F);
        const float g_new = sqrtf(2.0f * e_new / E_MASS_F);
        eta = TWO_PI_F * rs.uniform();
        float sc2, cc2, se2, ce2;
        if (ALG) {  // eta_new = eta + pi
            sincos_of_acos(sqrtf(e_new / en), &sc2, &cc2);
            dm::sincosf_det(eta, &se, &ce);
            se2 = -se;
            ce2 = -ce;
        } else {
            dm::sincosf_det(dm::acosf_det(sqrtf(e_new / en)), &sc2, &cc2);
            dm::sincosf_det(eta + PI_F, &se2, &ce2);
        }
        float ngx, ngy, ngz;
        rotate(g_new, sc2, cc2, se2, ce2, eu, ngx, ngy, ngz);
        const float xi = XPRE ? xpre : x[off + i];
        uint32_t slot;
        if (claim_slot(alive_e, g.capacity, slot)) {
            x[off + slot] = xi;
            vx[off + slot] = wx + g.f2 * ngx;
            vy[off + slot] = wy + g.f2 * ngy;
            vz[off + slot] = wz + g.f2 * ngz;
            if (dep_e) deposit_global(dep_e, xi, g);
        } else {
            set_dev_err(g.dev_err, CUDAPIC_DEVERR_SPAWN_E);
        }
        float a, b, c;
        rs.three_normal(g.normal_range, a, b, c);
        if (claim_slot(alive_i, g.capacity, slot)) {
            ix[off + slot] = xi;
            ivx[off + slot] = a;
            ivy[off + slot] = b;
            ivz[off + slot] = c;
            if (dep_i) deposit_global(dep_i, xi, g);
        } else {
            set_dev_err(g.dev_err, CUDAPIC_DEVERR_SPAWN_I);
        }
        if (ALG) sincos_of_acos(sqrtf(e_orig / en), &chi_s, &chi_c);
        else dm::sincosf_det(dm::acosf_det(sqrtf(e_orig / en)), &chi_s, &chi_c);
    }
    if (!ALG || ev != 3) dm::sincosf_det(eta, &se, &ce);
    float ngx, ngy, ngz;
    rotate(gm, chi_s, chi_c, se, ce, eu, ngx, ngy, ngz);
    vx[off + i] = wx + g.f2 * ngx;
    vy[off + i] = wy + g.f2 * ngy;
    vz[off + i] = wz + g.f2 * ngz;
    return ev;
}

// The body as one out-of-line function: the callers that run it inside a
// streaming loop keep its registers out of their own.
template <bool ALG>
static __device__ __noinline__ uint32_t collide_electron_t(uint32_t off, uint32_t i, uint32_t idx, float vxi,
                                                    float vyi, float vzi, Xoshiro128p &rs,
                                                    const float *__restrict__ cs, float *x, float *vx, float *vy,
                                                    float *vz, float *ix, float *ivx, float *ivy, float *ivz,
                                                    uint32_t *alive_e, uint32_t *alive_i, const cudapic_grid &g,
                                                    float *dep_e, float *dep_i) {
    return collide_electron_body<ALG, false>(off, i, idx, vxi, vyi, vzi, rs, cs, x, vx, vy, vz, ix, ivx, ivy, ivz,
                                             alive_e, alive_i, g, dep_e, dep_i, 0.0f);
}

// The reference formulation (the drop-in collision kernels).
static __device__ __forceinline__ uint32_t collide_electron(uint32_t off, uint32_t i, uint32_t idx, float vxi,
                                                            float vyi, float vzi, Xoshiro128p &rs,
                                                            const float *__restrict__ cs, float *x, float *vx,
                                                            float *vy, float *vz, float *ix, float *ivx, float *ivy,
                                                            float *ivz, uint32_t *alive_e, uint32_t *alive_i,
                                                            const cudapic_grid &g, float *dep_e, float *dep_i) {
    return collide_electron_t<false>(off, i, idx, vxi, vyi, vzi, rs, cs, x, vx, vy, vz, ix, ivx, ivy, ivz, alive_e,
                                     alive_i, g, dep_e, dep_i);
}

struct IonTest {
    uint32_t idx;
    float vxa, vya, vza;
    bool collide;
};

// Ion collision test with a Maxwellian target, Rust-CUDA/src/main.rs:1180-1197.
template <typename Table>
__device__ __forceinline__ IonTest test_ion(float vxi, float vyi, float vzi, Xoshiro128p &rs,
                                            const Table &sigma_tot_i, const cudapic_grid &g) {
    IonTest t;
    rs.three_normal(g.normal_range, t.vxa, t.vya, t.vza);
    const float gx = vxi - t.vxa, gy = vyi - t.vya, gz = vzi - t.vza;
    const float g2 = gx * gx + gy * gy + gz * gz;
    const float energy = g.half_mu_over_e * g2;
    t.idx = energy_index(energy);
    const float gmag = sqrtf(g2);
    const float nu = sigma_tot_i(t.idx) * gmag;
    const float rand_val = rs.uniform();
    t.collide = collision_draw(rand_val, nu * g.dt_i);
    return t;
}

// The ion test's outcome, first without the target atom (the same decision
// and the same five draws as test_ion, bit for bit).  Box-Muller's four draws
// are only advanced, and the test draw is compared with a bound on nu dt
// over every target the draws can give: with u >= 1e-9 each radius is at
// most sqrt(-2 ln 1e-9) = 6.438, so |v_atom| <= sqrt(rad1^2 + rad2^2) sigma
// <= 9.2 sigma, |g| <= |v| + 9.2 sigma and nu dt <= k (|v| + 9.2 sigma)
// with k >= max(sigma_tot_i) dt_i (rounded up by 1e-5 for the f32 products).
// A draw at or above that bound + 6e-7 cannot collide (collision_draw's
// bound: the computed p <= a + 3.1e-7): no transcendental is evaluated, for
// nearly every ion at the reference conditions.  Otherwise (or k = +inf,
// no bound) the full test runs again from the saved state.
template <typename Table>
__device__ __forceinline__ bool ion_collides(float vxi, float vyi, float vzi, Xoshiro128p &rs,
                                             const Table &sigma_tot_i, const cudapic_grid &g, float k) {
    if (k < INFINITY) {  // uniform across the launch: the drop-in entry passes +inf
        const Xoshiro128p r0 = rs;
        rs.next();
        rs.next();
        rs.next();
        rs.next();
        const float u = rs.uniform();
        const float vmag = sqrtf(vxi * vxi + vyi * vyi + vzi * vzi);
        if (u >= fmaf(k, vmag + 9.2f * g.normal_range, 6e-7f)) return false;
        rs = r0;
    }
    return test_ion(vxi, vyi, vzi, rs, sigma_tot_i, g).collide;
}

// collision_i, Rust-CUDA/src/main.rs:1221-1292; returns 4 isotropic, 5 backscatter.
static __device__ __noinline__ uint32_t collide_ion(uint32_t i, uint32_t idx, float vxi, float vyi, float vzi, float vxa,
                                             float vya, float vza, Xoshiro128p &rs, const float *__restrict__ cs,
                                             float *vx, float *vy, float *vz, const cudapic_grid &g) {
    const float gx = vxi - vxa, gy = vyi - vya, gz = vzi - vza;
    const float t0 = __ldg(cs + 3 * CS_RANGES + idx);
    const float t1 = t0 + __ldg(cs + 4 * CS_RANGES + idx);
    const float gg = sqrtf(gx * gx + gy * gy + gz * gz);
    const float wx = 0.5f * (vxi + vxa), wy = 0.5f * (vyi + vya), wz = 0.5f * (vzi + vza);
    const Euler eu = euler_angles(gx, gy, gz);
    const float rnd = rs.uniform();
    float chi;
    uint32_t ev;
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
    return ev;
}

}  // namespace cudapic
