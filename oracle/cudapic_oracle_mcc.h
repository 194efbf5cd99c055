/*
 * cudapic_oracle_mcc.h -- scalar helpers of the oracle shared by its
 * translation units (cudapic_oracle.c, cudapic_oracle_sens.c): the CIC cell,
 * the xoshiro128+ draws, the energy index and the scattering geometry.
 * TEST INFRASTRUCTURE ONLY, like the rest of the oracle.
 */
#ifndef CUDAPIC_ORACLE_MCC_H
#define CUDAPIC_ORACLE_MCC_H

#include <math.h>
#include "cudapic_oracle.h"

/* The reference computes `pos as usize` and reads node p+1 unguarded
 * (Rust-CUDA/src/main.rs:377-387, 600-603): a particle at exactly x = L
 * (pos == N_G-1) would touch node N_G.  The kernels clamp the cell to
 * [0, N_G-2]; for every pos in [0, N_G-1) the result is identical. */
static inline int cell_of(float pos, uint32_t n_g) {
    int p = (int)pos;
    if (!(pos >= 0.0f)) p = 0; /* negative or NaN */
    if (p > (int)n_g - 2) p = (int)n_g - 2;
    if (p < 0) p = 0;
    return p;
}

#define F_PI     ((float)ORC_PI)
#define F_TWO_PI ((float)(2.0 * ORC_PI))

typedef struct rng4 { uint32_t s[4]; } rng4;

static inline float draw(rng4 *r) { return orc_u32_to_real(orc_xoshiro128p_next(r->s)); }

/* rng_next_three_normal, Rust-CUDA/src/main.rs:908-969: four uniforms,
 * clamped to >= 1e-9, two Box-Muller pairs of which three normals are used.
 * ln(u) is evaluated directly (the reference uses lg2.approx * ln 2). */
static inline void three_normal(rng4 *r, float sigma, float *a, float *b, float *c) {
    float u1 = fmaxf(draw(r), 1e-9f);
    float u2 = fmaxf(draw(r), 1e-9f);
    float u3 = fmaxf(draw(r), 1e-9f);
    float u4 = fmaxf(draw(r), 1e-9f);
    float rad1 = sqrtf(-2.0f * orc_logf(u1));
    float ang1 = F_TWO_PI * u2;
    float z0 = rad1 * orc_cosf(ang1);
    float z1 = rad1 * orc_sinf(ang1);
    float rad2 = sqrtf(-2.0f * orc_logf(u3));
    float ang2 = F_TWO_PI * u4;
    float z2 = rad2 * orc_cosf(ang2);
    *a = z0 * sigma;
    *b = z1 * sigma;
    *c = z2 * sigma;
}

/* Energy index: min(int(E/DE_CS + 0.5), CS_RANGES-1), Rust-CUDA/src/main.rs:1002-1005. */
static inline uint32_t energy_index(float energy) {
    float t = fminf(energy / 0.001f + 0.5f, (float)(ORC_CS_RANGES - 1));
    return (uint32_t)t;
}

/* Euler angles of the relative velocity, Rust-CUDA/src/main.rs:1066-1082. */
static inline void euler_angles(float gx, float gy, float gz, float *st, float *ct, float *sp, float *cp) {
    float theta, phi;
    if (gx == 0.0f) theta = 0.5f * F_PI;
    else theta = orc_atan2f(sqrtf(gy * gy + gz * gz), gx);
    if (gy == 0.0f) phi = (gz > 0.0f) ? 0.5f * F_PI : -0.5f * F_PI;
    else phi = orc_atan2f(gz, gy);
    *st = orc_sinf(theta);
    *ct = orc_cosf(theta);
    *sp = orc_sinf(phi);
    *cp = orc_cosf(phi);
}

/* The same sines and cosines from their algebraic forms (the fused step's
 * scattering, cudapic_b200/csrc/mcc.cuh euler_angles_alg): sin theta = r/|g|,
 * cos theta = gx/|g|, sin phi = gz/r, cos phi = gy/r, r = sqrt(gy^2 + gz^2),
 * with the special cases of euler_angles and cos(+-pi/2) = 0 exactly. */
static inline void euler_angles_alg(float gx, float gy, float gz, float *st, float *ct, float *sp, float *cp) {
    const float r2 = gy * gy + gz * gz;
    const float r = sqrtf(r2);
    if (gx == 0.0f) {
        *st = 1.0f;
        *ct = 0.0f;
    } else {
        const float gn = sqrtf(gx * gx + r2);
        *st = r / gn;
        *ct = gx / gn;
    }
    if (gy == 0.0f) {
        *sp = (gz > 0.0f) ? 1.0f : -1.0f;
        *cp = 0.0f;
    } else {
        *sp = gz / r;
        *cp = gy / r;
    }
}

/* sin and cos of acos(c): sqrt((1 - c)(1 + c)) and c. */
static inline void sincos_of_acos(float c, float *s, float *co) {
    *s = sqrtf(fmaxf(0.0f, (1.0f - c) * (1.0f + c)));
    *co = c;
}

/* Rotation of a relative velocity of magnitude g by (chi, eta) in the frame
 * given by the Euler angles, Rust-CUDA/src/main.rs:1152-1158. */
static inline void rotate(float g, float chi_s, float chi_c, float eta_s, float eta_c,
                          float st, float ct, float sp, float cp,
                          float *gx, float *gy, float *gz) {
    float sc = chi_s, cc = chi_c, se = eta_s, ce = eta_c;
    *gx = g * (ct * cc - st * sc * ce);
    *gy = g * (st * cp * cc + ct * cp * sc * ce - sp * sc * se);
    *gz = g * (st * sp * cc + ct * sp * sc * ce + cp * sc * se);
}

#endif
