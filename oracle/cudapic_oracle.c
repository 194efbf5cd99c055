/*
 * cudapic_oracle.c -- CPU restatement of the cudaPIC per-timestep cycle.
 *
 * TEST INFRASTRUCTURE ONLY (see cudapic_oracle.h): the checker of the CUDA
 * kernels, never part of the product path.  Compile with -ffp-contract=off.
 *
 * Reference citations are to the reference project tree:
 *   Rust-CUDA/src/main.rs   cudaPIC (cuda-oxide kernels and host driver)
 *   C/eduPIC.cc             eduPIC 1.0, the FP64 CPU code the GPU path ports
 */
#include <math.h>
#include <stdlib.h>
#include <string.h>
#include "cudapic_oracle.h"
#include "cudapic_oracle_mcc.h"

/* ------------------------------------------------------------------ */
/* parameters                                                          */
/* ------------------------------------------------------------------ */

/* Rust-CUDA/src/main.rs:40-50 and :79 (MAX_PARTICLES). */
void orc_params_default(orc_params *p) {
    p->n_g = 400;
    p->n_t = 4000;
    p->n_sub = 20;
    p->capacity = 120000;
    p->frequency = 13.56e6;
    p->voltage = 250.0;
    p->gap = 0.025;
    p->pressure = 10.0;
    p->temperature = 350.0;
    p->weight = 7.0e4;
    p->electrode_area = 1.0e-4;
}

/* Derived constants, Rust-CUDA/src/main.rs:53-59, 80-82, 92-109.  Every
 * `X as Real` of the reference is a double expression rounded to float. */
void orc_phys_from_params(const orc_params *p, orc_phys *o) {
    double period = 1.0 / p->frequency;
    double dt_e = period / (double)p->n_t;
    double dt_i = (double)p->n_sub * dt_e;
    double dx = p->gap / (double)(p->n_g - 1);
    double inv_dx = 1.0 / dx;
    o->n_g = p->n_g;
    o->capacity = p->capacity;
    o->inv_dx = (float)inv_dx;
    o->weight_factor = (float)(p->weight / (p->electrode_area * dx));
    o->gap = (float)p->gap;
    o->dt_e = (float)dt_e;
    o->dt_i = (float)dt_i;
    o->factor_e = (float)(dt_e / ORC_E_MASS * (-ORC_E_CHARGE));
    o->factor_i = (float)(dt_i / ORC_AR_MASS * ORC_E_CHARGE);
    o->e_charge = (float)ORC_E_CHARGE;
    o->alpha = (float)(-dx * dx / ORC_EPSILON0);
    o->half_dx_over_eps = (float)(dx / (2.0 * ORC_EPSILON0));
    o->half_inv_dx = (float)(0.5 * inv_dx);
    o->normal_range = (float)sqrt(ORC_K_BOLTZMANN * p->temperature / ORC_AR_MASS);
    o->f1 = (float)(ORC_E_MASS / (ORC_E_MASS + ORC_AR_MASS));
    o->f2 = (float)(ORC_AR_MASS / (ORC_E_MASS + ORC_AR_MASS));
    o->half_me_over_e = (float)(0.5 * ORC_E_MASS / ORC_E_CHARGE);
    o->half_mu_over_e = (float)(0.5 * (ORC_AR_MASS / 2.0) / ORC_E_CHARGE);
    o->min_x = (float)(0.45 * p->gap);
    o->max_x = (float)(0.55 * p->gap);
    o->eepf_half_kick = (float)(dt_e * ORC_E_CHARGE / ORC_E_MASS);
    o->dx = dx;
    o->weight_factor_d = p->weight / (p->electrode_area * dx);
    o->voltage = p->voltage;
    o->omega = 2.0 * ORC_PI * p->frequency;
    o->n_t = p->n_t;
    o->n_sub = p->n_sub;
    o->gas_density = p->pressure / (ORC_K_BOLTZMANN * p->temperature);
    o->dt_e_d = dt_e;
    o->dt_i_d = dt_i;
}

/* ------------------------------------------------------------------ */
/* RNG                                                                 */
/* ------------------------------------------------------------------ */

static inline uint32_t rotl32(uint32_t x, int k) { return (x << k) | (x >> (32 - k)); }

/* xoshiro128+ 1.0 step, Rust-CUDA/src/main.rs:864-881 (Vigna's
 * Rust-CUDA/xorshiro128c/xoshiro128p.c:39-54). */
uint32_t orc_xoshiro128p_next(uint32_t s[4]) {
    uint32_t result = s[0] + s[3];
    uint32_t t = s[1] << 9;
    s[2] ^= s[0];
    s[3] ^= s[1];
    s[1] ^= s[2];
    s[0] ^= s[3];
    s[2] ^= t;
    s[3] = rotl32(s[3], 11);
    return result;
}

void orc_xoshiro128p_stream(const uint32_t seed[4], uint32_t n, uint32_t *out) {
    uint32_t s[4] = {seed[0], seed[1], seed[2], seed[3]};
    for (uint32_t i = 0; i < n; ++i) out[i] = orc_xoshiro128p_next(s);
}

/* u32_to_real, Rust-CUDA/src/main.rs:883-885: 23 high bits as a float in [0,1). */
float orc_u32_to_real(uint32_t x) {
    uint32_t b = 0x3F800000u | (x >> 9);
    float f;
    memcpy(&f, &b, 4);
    return f - 1.0f;
}

/* jump(): advance by 2^64 steps, Rust-CUDA/src/main.rs:1452, 1473-1487. */
void orc_jump(uint32_t s[4]) {
    static const uint32_t JUMP[4] = {0x8764000bu, 0xf542d2d3u, 0x6fa035c3u, 0x77f2db5bu};
    uint32_t acc[4] = {0, 0, 0, 0};
    for (int w = 0; w < 4; ++w) {
        for (int b = 0; b < 32; ++b) {
            if (JUMP[w] & (1u << b)) {
                acc[0] ^= s[0];
                acc[1] ^= s[1];
                acc[2] ^= s[2];
                acc[3] ^= s[3];
            }
            orc_xoshiro128p_next(s);
        }
    }
    s[0] = acc[0]; s[1] = acc[1]; s[2] = acc[2]; s[3] = acc[3];
}

/* xoshiro128_seed_streams, Rust-CUDA/src/main.rs:1446-1496: stream k is the
 * master state after k jumps.  Returns -1 for the all-zero master state
 * (the reference asserts, :1447-1450). */
int orc_seed_streams(const uint32_t master[4], uint32_t n,
                     uint32_t *s0, uint32_t *s1, uint32_t *s2, uint32_t *s3) {
    if ((master[0] | master[1] | master[2] | master[3]) == 0) return -1;
    uint32_t s[4] = {master[0], master[1], master[2], master[3]};
    for (uint32_t k = 0; k < n; ++k) {
        s0[k] = s[0]; s1[k] = s[1]; s2[k] = s[2]; s3[k] = s[3];
        orc_jump(s);
    }
    return 0;
}

/* ------------------------------------------------------------------ */
/* cross sections, Rust-CUDA/src/main.rs:1378-1444                    */
/* ------------------------------------------------------------------ */

static double q_mom_e(double e) {
    return 1.0e-20 *
           (fabs(6.0 / pow(1.0 + e / 0.1 + pow(e / 0.6, 2.0), 3.3) -
                 1.1 * pow(e, 1.4) / (1.0 + pow(e / 15.0, 1.2)) /
                     sqrt(1.0 + pow(e / 5.5, 2.5) + pow(e / 60.0, 4.1))) +
            0.05 / pow(1.0 + e / 10.0, 2.0) + 0.01 * pow(e, 3.0) / (1.0 + pow(e / 12.0, 6.0)));
}

static double q_exc_e(double e) {
    if (e <= 11.5) return 0.0;
    return (0.034 * pow(e - 11.5, 1.1) * (1.0 + pow(e / 15.0, 2.8)) / (1.0 + pow(e / 23.0, 5.5)) +
            0.023 * (e - 11.5) / pow(1.0 + e / 80.0, 1.9)) *
           1.0e-20;
}

static double q_ion_e(double e) {
    if (e <= 15.8) return 0.0;
    return (970.0 * (e - 15.8) / pow(70.0 + e, 2.0) + 0.06 * pow(e - 15.8, 2.0) * exp(-e / 9.0)) *
           1.0e-20;
}

static double q_moi(double e_lab) { return 1.15e-18 * pow(e_lab, -0.1) * pow(1.0 + 0.015 / e_lab, 0.6); }
static double q_iso(double e_lab) {
    return 2.0e-19 * pow(e_lab, -0.5) / (1.0 + e_lab) + 3.0e-19 * e_lab / pow(1.0 + e_lab / 3.0, 2.0);
}
static double q_chx(double e_lab) { return 0.5 * (q_moi(e_lab) - q_iso(e_lab)); }

void orc_cross_sections(double gas_density, float *cs, float *sig_e, float *sig_i) {
    const uint32_t R = ORC_CS_RANGES;
    for (uint32_t i = 0; i < R; ++i) {
        double e = (i == 0) ? 0.001 : (double)i * 0.001;
        cs[0 * R + i] = (float)q_mom_e(e);
        cs[1 * R + i] = (float)q_exc_e(e);
        cs[2 * R + i] = (float)q_ion_e(e);
        cs[3 * R + i] = (float)q_iso(2.0 * e);
        cs[4 * R + i] = (float)q_chx(2.0 * e);
    }
    for (uint32_t i = 0; i < R; ++i) {
        double se = (double)cs[0 * R + i] + (double)cs[1 * R + i] + (double)cs[2 * R + i];
        double si = (double)cs[3 * R + i] + (double)cs[4 * R + i];
        sig_e[i] = (float)(se * gas_density);
        sig_i[i] = (float)(si * gas_density);
    }
}

/* ------------------------------------------------------------------ */
/* cell index with the bounds clamp of this project                    */
/* ------------------------------------------------------------------ */


/* ------------------------------------------------------------------ */
/* deposition                                                          */
/* ------------------------------------------------------------------ */

/* get_density, Rust-CUDA/src/main.rs:356-406: CIC weights
 * c1 = (1-rem) W, c2 = rem W into nodes p, p+1; boundary nodes doubled. */
void orc_get_density_f32(const float *x, uint32_t n, float *density, const orc_phys *ph) {
    uint32_t n_g = ph->n_g;
    for (uint32_t k = 0; k < n_g; ++k) density[k] = 0.0f;
    for (uint32_t i = 0; i < n; ++i) {
        float pos = x[i] * ph->inv_dx;
        int p = cell_of(pos, n_g);
        float rem = pos - (float)p;
        float c1 = (1.0f - rem) * ph->weight_factor;
        float c2 = rem * ph->weight_factor;
        density[p] += c1;
        density[p + 1] += c2;
    }
    density[0] *= 2.0f;
    density[n_g - 1] *= 2.0f;
}

/* FP64 deposit of eduPIC, C/eduPIC.cc:520-529 (positions are the f32 inputs). */
void orc_get_density_f64(const float *x, uint32_t n, double *density, const orc_phys *ph) {
    uint32_t n_g = ph->n_g;
    double inv_dx = 1.0 / ph->dx;
    double fw = ph->weight_factor_d;
    for (uint32_t k = 0; k < n_g; ++k) density[k] = 0.0;
    for (uint32_t i = 0; i < n; ++i) {
        double c0 = (double)x[i] * inv_dx;
        int p = (int)c0;
        if (p > (int)n_g - 2) p = (int)n_g - 2;
        if (p < 0) p = 0;
        density[p] += (p + 1 - c0) * fw;
        density[p + 1] += (c0 - p) * fw;
    }
    density[0] *= 2.0;
    density[n_g - 1] *= 2.0;
}

/* ------------------------------------------------------------------ */
/* Poisson                                                             */
/* ------------------------------------------------------------------ */

/* solve_Poisson of eduPIC, C/eduPIC.cc:461-494: Thomas algorithm for
 * pot[i-1] - 2 pot[i] + pot[i+1] = -DX^2 rho_i / eps0 with pot[0] = pot0,
 * pot[N_G-1] = 0, then central differences and one-sided electrode fields.
 * rho = e (n_i - n_e) is formed in double from the f32 densities. */
void orc_poisson_thomas_f64(const float *e_density, const float *i_density, double pot0,
                            double *pot, double *efield, const orc_phys *ph) {
    const int n = (int)ph->n_g;
    const double dx = ph->dx;
    const double alpha = -dx * dx / ORC_EPSILON0;
    if (n < 3) return;
    double *rho = (double *)malloc(sizeof(double) * n);
    double *g = (double *)malloc(sizeof(double) * n);
    double *w = (double *)malloc(sizeof(double) * n);
    double *f = (double *)malloc(sizeof(double) * n);
    for (int i = 0; i < n; ++i) rho[i] = ORC_E_CHARGE * ((double)i_density[i] - (double)e_density[i]);
    pot[0] = pot0;
    pot[n - 1] = 0.0;
    for (int i = 1; i <= n - 2; ++i) f[i] = alpha * rho[i];
    f[1] -= pot[0];
    f[n - 2] -= pot[n - 1];
    w[1] = 1.0 / -2.0;
    g[1] = f[1] / -2.0;
    for (int i = 2; i <= n - 2; ++i) {
        w[i] = 1.0 / (-2.0 - w[i - 1]);
        g[i] = (f[i] - g[i - 1]) / (-2.0 - w[i - 1]);
    }
    pot[n - 2] = g[n - 2];
    for (int i = n - 3; i > 0; --i) pot[i] = g[i] - w[i] * pot[i + 1];
    const double s = 1.0 / (2.0 * dx);
    for (int i = 1; i <= n - 2; ++i) efield[i] = (pot[i - 1] - pot[i + 1]) * s;
    efield[0] = (pot[0] - pot[1]) / dx - rho[0] * dx / (2.0 * ORC_EPSILON0);
    efield[n - 1] = (pot[n - 2] - pot[n - 1]) / dx + rho[n - 1] * dx / (2.0 * ORC_EPSILON0);
    free(rho); free(g); free(w); free(f);
}

/* solve_poisson_scan_f32, Rust-CUDA/src/main.rs:408-494.  The Thomas
 * recurrences of the unit tridiagonal system have the closed form
 *   G_i = sum_{j<=i} j f_j,  r_i = -G_i / ((i+1) i),  pot_i = i sum_{j=i}^{N-2} r_j,
 * evaluated with two inclusive prefix sums.  The reference's block_scan
 * order is set by cuda-oxide (not vendored); this restatement sums
 * sequentially, so it is a tolerance reference, not a bit-exact one. */
void orc_poisson_scan_f32(const float *e_density, const float *i_density, float pot0,
                          float *pot, float *efield, const orc_phys *ph) {
    const int n = (int)ph->n_g;
    float *rho = (float *)malloc(sizeof(float) * n);
    float *G = (float *)malloc(sizeof(float) * n);
    float *r = (float *)malloc(sizeof(float) * n);
    float *R = (float *)malloc(sizeof(float) * n);
    for (int i = 0; i < n; ++i) rho[i] = ph->e_charge * (i_density[i] - e_density[i]);
    float acc = 0.0f;
    for (int i = 0; i < n; ++i) {
        float gi = 0.0f;
        if (i != 0 && i < n) {
            float fi = ph->alpha * rho[i] - (i == 1 ? pot0 : 0.0f);
            gi = (float)i * fi;
        }
        acc += gi;
        G[i] = acc;
    }
    acc = 0.0f;
    for (int i = 0; i < n; ++i) {
        float ri = 0.0f;
        if (i != 0 && i < n - 1) {
            float hi = -G[i] / ((float)i + 1.0f);
            ri = hi / (float)i;
        }
        r[i] = ri;
        acc += ri;
        R[i] = acc;
    }
    float r_total = R[n - 2];
    for (int i = 0; i < n; ++i) {
        if (i == 0) pot[i] = pot0;
        else if (i < n - 1) pot[i] = (float)i * (r_total - R[i] + r[i]);
        else pot[i] = 0.0f;
    }
    for (int i = 0; i < n; ++i) {
        if (i == 0) efield[i] = (pot[0] - pot[1]) * ph->inv_dx - rho[0] * ph->half_dx_over_eps;
        else if (i == n - 1) efield[i] = (pot[n - 2] - pot[n - 1]) * ph->inv_dx + rho[n - 1] * ph->half_dx_over_eps;
        else efield[i] = (pot[i - 1] - pot[i + 1]) * ph->half_inv_dx;
    }
    free(rho); free(G); free(r); free(R);
}

/* solve_poisson_dps_flexible, Rust-CUDA/src/main.rs:496-564, in double:
 * psi'' = source on n nodes with Dirichlet values at both ends. */
void orc_poisson_dps_flexible_f64(const double *source, double *pot, uint32_t n_,
                                  double psi_left, double psi_right, double dx) {
    const int n = (int)n_;
    double G = 0.0, *r = (double *)malloc(sizeof(double) * n);
    for (int i = 0; i < n; ++i) {
        double gi = 0.0;
        if (i != 0 && i < n) {
            double fi = dx * dx * source[i];
            if (i == 1) fi -= psi_left;
            if (i == n - 2) fi -= psi_right;
            gi = (double)i * fi;
        }
        G += gi;
        r[i] = (i != 0 && i < n - 1) ? (-G / ((double)i + 1.0)) / (double)i : 0.0;
    }
    double tail = 0.0;
    for (int i = n - 2; i >= 1; --i) {
        tail += r[i];
        pot[i] = (double)i * tail;
    }
    pot[0] = psi_left;
    pot[n - 1] = psi_right;
    free(r);
}

/* ------------------------------------------------------------------ */
/* push + absorb + compact                                             */
/* ------------------------------------------------------------------ */

/* move_and_compact, Rust-CUDA/src/main.rs:566-678: CIC-gathered field,
 * v' = v + factor E, x' = x + v' dt, survivors with 0 <= x' <= L kept.
 * The reference writes survivors unordered across blocks; this restatement
 * keeps index order, so comparisons are on the survivor set. */
uint32_t orc_move_and_compact(const float *efield,
                              const float *sx, const float *svx, const float *svy, const float *svz,
                              float *dx_, float *dvx, float *dvy, float *dvz,
                              uint32_t n, float factor, float dt, const orc_phys *ph,
                              uint32_t *src_index) {
    uint32_t m = 0;
    for (uint32_t i = 0; i < n; ++i) {
        float xi = sx[i];
        float vxi = svx[i];
        float pos = xi * ph->inv_dx;
        int p = cell_of(pos, ph->n_g);
        float c2 = pos - (float)p;
        float e_x = (1.0f - c2) * efield[p] + c2 * efield[p + 1];
        float nvx = vxi + factor * e_x;
        float nx = xi + nvx * dt;
        if (nx >= 0.0f && nx <= ph->gap) {
            dx_[m] = nx;
            dvx[m] = nvx;
            dvy[m] = svy[i];
            dvz[m] = svz[i];
            if (src_index) src_index[m] = i;
            ++m;
        }
    }
    return m;
}

/* Boundary check of C/eduPIC.cc:623-667 on the pushed particles of
 * orc_move_and_compact: counts[0] += absorbed at x < 0 (powered electrode),
 * counts[1] += absorbed at x > L (grounded); with ions, the ion energy
 * 1/2 M v^2 / e in f32 (HALF_MI_OVER_E, v after the push) goes to the 1 eV
 * bin floor(E) of that electrode's IFED when below 200 eV (:118-119, :645-657). */
static const float HALF_MI_OVER_E = (float)(0.5 * ORC_AR_MASS / ORC_E_CHARGE);

void orc_wall_count(const float *efield, const float *sx, const float *svx, const float *svy, const float *svz,
                    uint32_t n, float factor, float dt, const orc_phys *ph, int ions, uint64_t counts[2],
                    uint32_t *ifed_pow, uint32_t *ifed_gnd) {
    for (uint32_t i = 0; i < n; ++i) {
        float xi = sx[i];
        float vxi = svx[i];
        float pos = xi * ph->inv_dx;
        int p = cell_of(pos, ph->n_g);
        float c2 = pos - (float)p;
        float e_x = (1.0f - c2) * efield[p] + c2 * efield[p + 1];
        float nvx = vxi + factor * e_x;
        float nx = xi + nvx * dt;
        int side = nx < 0.0f ? 0 : (nx > ph->gap ? 1 : -1);
        if (side < 0) continue;
        counts[side] += 1;
        if (ions) {
            float e = HALF_MI_OVER_E * (nvx * nvx + svy[i] * svy[i] + svz[i] * svz[i]);
            if (e < (float)ORC_N_IFED) (side == 0 ? ifed_pow : ifed_gnd)[(int)e] += 1;
        }
    }
}

/* ------------------------------------------------------------------ */
/* MCC                                                                 */
/* ------------------------------------------------------------------ */

double orc_p_coll_e_exact(const float *sigma_tot_e, float vx, float vy, float vz, const orc_phys *ph) {
    float v2 = vx * vx + vy * vy + vz * vz;
    float energy = ph->half_me_over_e * v2;
    uint32_t idx = energy_index(energy);
    double nu = (double)sigma_tot_e[idx] * sqrt((double)v2);
    return 1.0 - exp(-nu * (double)ph->dt_e);
}

/* check_collisions_e + collision_e, Rust-CUDA/src/main.rs:971-1165; alg:
 * the sines and cosines of the Euler angles, of chi = acos(c) and of
 * eta + pi from their algebraic forms (the fused step's scattering). */
static void check_collisions_e(const float *sigma_tot_e, const float *cs, uint32_t n_active,
                               float *x, float *vx, float *vy, float *vz,
                               uint32_t *r0, uint32_t *r1, uint32_t *r2, uint32_t *r3,
                               float *ix, float *ivx, float *ivy, float *ivz,
                               uint32_t *n_e, uint32_t *n_i, const orc_phys *ph,
                               uint8_t *events, uint32_t *dropped, int alg) {
    const uint32_t R = ORC_CS_RANGES;
    const float me = (float)ORC_E_MASS;
    const float qe = (float)ORC_E_CHARGE;
    const float exc_j = 11.5f * qe;
    const float ion_j = 15.8f * qe;
    for (uint32_t i = 0; i < n_active; ++i) {
        rng4 rs = {{r0[i], r1[i], r2[i], r3[i]}};
        float vxi = vx[i], vyi = vy[i], vzi = vz[i];
        float v2 = vxi * vxi + vyi * vyi + vzi * vzi;
        float energy = ph->half_me_over_e * v2;
        uint32_t idx = energy_index(energy);
        float velocity = sqrtf(v2);
        float nu = sigma_tot_e[idx] * velocity;
        float rand_val = draw(&rs);
        float p_coll = 1.0f - orc_expf(-nu * ph->dt_e);
        uint8_t ev = 0;
        if (rand_val < p_coll) {
            float gx = vxi, gy = vyi, gz = vzi;
            float g = sqrtf(gx * gx + gy * gy + gz * gz);
            float wx = ph->f1 * vxi, wy = ph->f1 * vyi, wz = ph->f1 * vzi;
            float t0 = cs[0 * R + idx];
            float t1 = t0 + cs[1 * R + idx];
            float t2 = t1 + cs[2 * R + idx];
            float st, ct, sp, cp;
            if (alg) euler_angles_alg(gx, gy, gz, &st, &ct, &sp, &cp);
            else euler_angles(gx, gy, gz, &st, &ct, &sp, &cp);
            float chi_s, chi_c, eta;
            float rnd = draw(&rs);
            if (rnd < t0 / t2) {
                ev = 1;
                float c = 1.0f - 2.0f * draw(&rs);
                eta = F_TWO_PI * draw(&rs);
                if (alg) {
                    sincos_of_acos(c, &chi_s, &chi_c);
                } else {
                    float chi = orc_acosf(c);
                    chi_s = orc_sinf(chi); chi_c = orc_cosf(chi);
                }
            } else if (rnd < t1 / t2) {
                ev = 2;
                float en = 0.5f * me * g * g;
                en = fabsf(en - exc_j);
                g = sqrtf(2.0f * en / me);
                float c = 1.0f - 2.0f * draw(&rs);
                eta = F_TWO_PI * draw(&rs);
                if (alg) {
                    sincos_of_acos(c, &chi_s, &chi_c);
                } else {
                    float chi = orc_acosf(c);
                    chi_s = orc_sinf(chi); chi_c = orc_cosf(chi);
                }
            } else {
                ev = 3;
                float en = 0.5f * me * g * g;
                en = fabsf(en - ion_j);
                float e_new = 10.0f * orc_tanf(draw(&rs) * orc_atanf(en / qe / 20.0f)) * qe;
                float e_orig = fabsf(en - e_new);
                g = sqrtf(2.0f * e_orig / me);
                float g_new = sqrtf(2.0f * e_new / me);
                eta = F_TWO_PI * draw(&rs);
                float sc2, cc2, se2, ce2;
                if (alg) {
                    sincos_of_acos(sqrtf(e_new / en), &sc2, &cc2);
                    se2 = -orc_sinf(eta);
                    ce2 = -orc_cosf(eta);
                } else {
                    float chi_new = orc_acosf(sqrtf(e_new / en));
                    float eta_new = eta + F_PI;
                    sc2 = orc_sinf(chi_new); cc2 = orc_cosf(chi_new);
                    se2 = orc_sinf(eta_new); ce2 = orc_cosf(eta_new);
                }
                float ngx, ngy, ngz;
                rotate(g_new, sc2, cc2, se2, ce2, st, ct, sp, cp, &ngx, &ngy, &ngz);
                float a, b, c;
                uint32_t e_slot = *n_e;
                int e_ok = e_slot < ph->capacity;
                if (e_ok) {
                    x[e_slot] = x[i];
                    vx[e_slot] = wx + ph->f2 * ngx;
                    vy[e_slot] = wy + ph->f2 * ngy;
                    vz[e_slot] = wz + ph->f2 * ngz;
                    *n_e = e_slot + 1;
                } else if (dropped) {
                    ++*dropped;
                }
                three_normal(&rs, ph->normal_range, &a, &b, &c);
                uint32_t i_slot = *n_i;
                if (i_slot < ph->capacity) {
                    ix[i_slot] = x[i];
                    ivx[i_slot] = a;
                    ivy[i_slot] = b;
                    ivz[i_slot] = c;
                    *n_i = i_slot + 1;
                } else if (dropped) {
                    ++*dropped;
                }
                if (alg) {
                    sincos_of_acos(sqrtf(e_orig / en), &chi_s, &chi_c);
                } else {
                    float chi = orc_acosf(sqrtf(e_orig / en));
                    chi_s = orc_sinf(chi); chi_c = orc_cosf(chi);
                }
            }
            float ngx, ngy, ngz;
            rotate(g, chi_s, chi_c, orc_sinf(eta), orc_cosf(eta), st, ct, sp, cp, &ngx, &ngy, &ngz);
            vx[i] = wx + ph->f2 * ngx;
            vy[i] = wy + ph->f2 * ngy;
            vz[i] = wz + ph->f2 * ngz;
        }
        r0[i] = rs.s[0]; r1[i] = rs.s[1]; r2[i] = rs.s[2]; r3[i] = rs.s[3];
        if (events) events[i] = ev;
    }
}

void orc_check_collisions_e(const float *sigma_tot_e, const float *cs, uint32_t n_active,
                            float *x, float *vx, float *vy, float *vz,
                            uint32_t *r0, uint32_t *r1, uint32_t *r2, uint32_t *r3,
                            float *ix, float *ivx, float *ivy, float *ivz,
                            uint32_t *n_e, uint32_t *n_i, const orc_phys *ph,
                            uint8_t *events, uint32_t *dropped) {
    check_collisions_e(sigma_tot_e, cs, n_active, x, vx, vy, vz, r0, r1, r2, r3, ix, ivx, ivy, ivz, n_e, n_i, ph,
                       events, dropped, 0);
}

void orc_check_collisions_e_alg(const float *sigma_tot_e, const float *cs, uint32_t n_active,
                                float *x, float *vx, float *vy, float *vz,
                                uint32_t *r0, uint32_t *r1, uint32_t *r2, uint32_t *r3,
                                float *ix, float *ivx, float *ivy, float *ivz,
                                uint32_t *n_e, uint32_t *n_i, const orc_phys *ph,
                                uint8_t *events, uint32_t *dropped) {
    check_collisions_e(sigma_tot_e, cs, n_active, x, vx, vy, vz, r0, r1, r2, r3, ix, ivx, ivy, ivz, n_e, n_i, ph,
                       events, dropped, 1);
}

/* check_collisions_i + collision_i, Rust-CUDA/src/main.rs:1167-1292. */
void orc_check_collisions_i(const float *sigma_tot_i, const float *cs, uint32_t n_active,
                            float *vx, float *vy, float *vz,
                            uint32_t *r0, uint32_t *r1, uint32_t *r2, uint32_t *r3,
                            const orc_phys *ph, uint8_t *events) {
    const uint32_t R = ORC_CS_RANGES;
    for (uint32_t i = 0; i < n_active; ++i) {
        rng4 rs = {{r0[i], r1[i], r2[i], r3[i]}};
        float vxa, vya, vza;
        three_normal(&rs, ph->normal_range, &vxa, &vya, &vza);
        float vxi = vx[i], vyi = vy[i], vzi = vz[i];
        float gx = vxi - vxa, gy = vyi - vya, gz = vzi - vza;
        float g2 = gx * gx + gy * gy + gz * gz;
        float energy = ph->half_mu_over_e * g2;
        uint32_t idx = energy_index(energy);
        float g = sqrtf(g2);
        float nu = sigma_tot_i[idx] * g;
        float rand_val = draw(&rs);
        float p_coll = 1.0f - orc_expf(-nu * ph->dt_i);
        uint8_t ev = 0;
        if (rand_val < p_coll) {
            float t0 = cs[3 * R + idx];
            float t1 = t0 + cs[4 * R + idx];
            float gg = sqrtf(gx * gx + gy * gy + gz * gz);
            float wx = 0.5f * (vxi + vxa), wy = 0.5f * (vyi + vya), wz = 0.5f * (vzi + vza);
            float st, ct, sp, cp;
            euler_angles(gx, gy, gz, &st, &ct, &sp, &cp);
            float rnd = draw(&rs);
            float chi;
            if (rnd < t0 / t1) {
                ev = 4;
                chi = orc_acosf(1.0f - 2.0f * draw(&rs));
            } else {
                ev = 5;
                chi = F_PI;
            }
            float eta = F_TWO_PI * draw(&rs);
            float ngx, ngy, ngz;
            rotate(gg, orc_sinf(chi), orc_cosf(chi), orc_sinf(eta), orc_cosf(eta), st, ct, sp, cp,
                   &ngx, &ngy, &ngz);
            vx[i] = wx + 0.5f * ngx;
            vy[i] = wy + 0.5f * ngy;
            vz[i] = wz + 0.5f * ngz;
        }
        r0[i] = rs.s[0]; r1[i] = rs.s[1]; r2[i] = rs.s[2]; r3[i] = rs.s[3];
        if (events) events[i] = ev;
    }
}

/* ------------------------------------------------------------------ */
/* diagnostics                                                         */
/* ------------------------------------------------------------------ */

/* accumulate_density, Rust-CUDA/src/main.rs:1294-1299. */
void orc_accumulate_density(const float *density, double *cumul, uint32_t n_g) {
    for (uint32_t k = 0; k < n_g; ++k) cumul[k] += (double)density[k];
}

/* accumulate_eepf, Rust-CUDA/src/main.rs:1301-1339: electrons strictly inside
 * (0.45 L, 0.55 L); energy from v_x corrected by half a kick; 0.05 eV bins. */
void orc_accumulate_eepf(const float *x, const float *vx, const float *vy, const float *vz,
                         const float *efield, uint32_t n_active, uint32_t *eepf,
                         const orc_phys *ph) {
    for (uint32_t i = 0; i < n_active; ++i) {
        float xi = x[i];
        if (xi <= ph->min_x || xi >= ph->max_x) continue;
        float pos = xi * ph->inv_dx;
        int p = cell_of(pos, ph->n_g);
        float c2 = pos - (float)p;
        float e_x = (1.0f - c2) * efield[p] + c2 * efield[p + 1];
        float mvx = vx[i] - 0.5f * e_x * ph->eepf_half_kick;
        float v2 = mvx * mvx + vy[i] * vy[i] + vz[i] * vz[i];
        float energy = ph->half_me_over_e * v2;
        float binf = energy / 0.05f;
        if (binf < (float)ORC_N_EEPF) eepf[(uint32_t)binf] += 1;
    }
}

/* XT diagnostics, C/eduPIC.cc:557-576 (electrons) and :599-614 (ions). */
void orc_xt_accumulate(const float *efield, const float *x, const float *vx, const float *vy, const float *vz,
                       uint32_t n, int ions, const float *cs_ion, const orc_phys *ph, double *out) {
    const uint32_t n_g = ph->n_g;
    const float factor = ions ? ph->factor_i : ph->factor_e;
    const float half_m = ions ? HALF_MI_OVER_E : ph->half_me_over_e;
    const float rate_scale = (float)((double)ph->dt_e * ph->gas_density);
    for (uint32_t i = 0; i < n; ++i) {
        float pos = x[i] * ph->inv_dx;
        int p = cell_of(pos, n_g);
        float c2 = pos - (float)p;
        float c1 = 1.0f - c2;
        float e_x = c1 * efield[p] + c2 * efield[p + 1];
        float v = vx[i] + 0.5f * factor * e_x;
        float v2 = v * v + vy[i] * vy[i] + vz[i] * vz[i];
        float energy = half_m * v2;
        out[p] += c1;
        out[p + 1] += c2;
        out[n_g + p] += c1 * v;
        out[n_g + p + 1] += c2 * v;
        out[2 * n_g + p] += c1 * energy;
        out[2 * n_g + p + 1] += c2 * energy;
        if (!ions) {
            float t = fminf(energy / 0.001f + 0.5f, (float)(ORC_CS_RANGES - 1));
            float rate = cs_ion[(uint32_t)t] * sqrtf(v2) * rate_scale;
            out[3 * n_g + p] += c1 * rate;
            out[3 * n_g + p + 1] += c2 * rate;
        }
    }
}
