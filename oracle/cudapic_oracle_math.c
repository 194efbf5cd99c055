/*
 * cudapic_oracle_math.c -- f32 transcendental functions of the oracle.
 *
 * TEST INFRASTRUCTURE ONLY (see cudapic_oracle.h).
 *
 * The reference evaluates its collision-kernel transcendentals with PTX
 * approximation instructions plus its own 3-term atan polynomial
 * (Rust-CUDA/src/main.rs:680-858).  Those cannot be reproduced on a CPU.  The
 * CUDA kernels of this project instead evaluate each function with a
 * published method built only from IEEE-754 +,-,*,/, sqrt and fmaf, which
 * give identical bits on any IEEE machine when the operation order is fixed.
 * This file restates those methods independently in C:
 *
 *   exp   Cody & Waite (1980) reduction x = k ln2 + r, |r| <= ln2/2, with a
 *         two-word ln2; Taylor polynomial of degree 7 for e^r (truncation
 *         error < 6e-9 relative); scaling by 2^k through the exponent field.
 *   log   x = m 2^e with m in [sqrt(1/2), sqrt(2)); ln m = 2 atanh(s),
 *         s = (m-1)/(m+1), |s| <= 0.1716, series to s^11 (error < 3e-10).
 *   sin/cos  Cody & Waite reduction by pi/2 with a two-word pi/2 (inputs on
 *         this path satisfy |x| < 16); Taylor polynomials of degree 9 (sin)
 *         and 10 (cos) on |r| <= pi/4 (error < 2e-9).
 *   atan  reflection a -> 1/a for a > 1, then the addition formula
 *         atan(a) = pi/6 + atan((a sqrt3 - 1)/(a + sqrt3)) for a > tan(pi/12),
 *         Taylor series to t^13 on |t| <= tan(pi/12) (error < 2e-9).
 *   atan2 quadrant logic on atan of min/max; acos(x) = atan2(sqrt((1-x)(1+x)), x)
 *         (the reference also builds acos from atan2, Rust-CUDA/src/main.rs:840-843);
 *   tan   sin/cos with an IEEE division (the reference does the same with
 *         sin.approx * rcp.approx(cos), Rust-CUDA/src/main.rs:783-788).
 *
 * Polynomials are evaluated by Horner's rule with fmaf in a fixed order.
 * The coefficients are the exact Taylor coefficients rounded to float,
 * written as hexadecimal literals so that no compiler folds them differently.
 */
#include <math.h>
#include <stdint.h>
#include <string.h>
#include "cudapic_oracle.h"

#define DM_LOG2E        0x1.715476p+0f
#define DM_LN2_HI       0x1.62e430p-1f
#define DM_LN2_LO       -0x1.05c610p-29f
#define DM_INV_FACT3    0x1.555556p-3f
#define DM_INV_FACT4    0x1.555556p-5f
#define DM_INV_FACT5    0x1.111112p-7f
#define DM_INV_FACT6    0x1.6c16c2p-10f
#define DM_INV_FACT7    0x1.a01a02p-13f
#define DM_SQRT2        0x1.6a09e6p+0f
#define DM_INV_3        0x1.555556p-2f
#define DM_INV_5        0x1.99999ap-3f
#define DM_INV_7        0x1.24924ap-3f
#define DM_INV_9        0x1.c71c72p-4f
#define DM_INV_11       0x1.745d18p-4f
#define DM_INV_13       0x1.3b13b2p-4f
#define DM_TWO_OVER_PI  0x1.45f306p-1f
#define DM_PIO2_1       0x1.921fb6p+0f
#define DM_PIO2_2       -0x1.777a5cp-25f
#define DM_SIN_C1       -0x1.555556p-3f
#define DM_SIN_C2       0x1.111112p-7f
#define DM_SIN_C3       -0x1.a01a02p-13f
#define DM_SIN_C4       0x1.71de3ap-19f
#define DM_COS_C2       0x1.555556p-5f
#define DM_COS_C3       -0x1.6c16c2p-10f
#define DM_COS_C4       0x1.a01a02p-16f
#define DM_COS_C5       -0x1.27e4fcp-22f
#define DM_SQRT3        0x1.bb67aep+0f
#define DM_PI_6         0x1.0c1524p-1f
#define DM_TAN_PI_12    0x1.126146p-2f
#define DM_PI_2         0x1.921fb6p+0f
#define DM_PI           0x1.921fb6p+1f

static inline uint32_t f2u(float f) { uint32_t u; memcpy(&u, &f, 4); return u; }
static inline float u2f(uint32_t u) { float f; memcpy(&f, &u, 4); return f; }

/* p * 2^k for integer k in [-252, 254]: two exact power-of-two scalings, so
 * that only the final product can round (subnormal results). */
static inline float scale2i(float p, int k) {
    int k1 = k / 2;
    int k2 = k - k1;
    return (p * u2f((uint32_t)(k1 + 127) << 23)) * u2f((uint32_t)(k2 + 127) << 23);
}

float orc_expf(float x) {
    if (x != x) return x;
    if (x > 88.72283f) return INFINITY;
    if (x < -103.9721f) return 0.0f;
    float k = rintf(x * DM_LOG2E);
    float r = fmaf(-k, DM_LN2_HI, x);
    r = fmaf(-k, DM_LN2_LO, r);
    float p = DM_INV_FACT7;
    p = fmaf(p, r, DM_INV_FACT6);
    p = fmaf(p, r, DM_INV_FACT5);
    p = fmaf(p, r, DM_INV_FACT4);
    p = fmaf(p, r, DM_INV_FACT3);
    p = fmaf(p, r, 0.5f);
    p = fmaf(p, r, 1.0f);
    p = fmaf(p, r, 1.0f);
    return scale2i(p, (int)k);
}

float orc_logf(float x) {
    if (x != x) return x;
    if (x < 0.0f) return NAN;
    if (x == 0.0f) return -INFINITY;
    if (x == INFINITY) return x;
    int e0 = 0;
    if (x < 0x1p-126f) { x = x * 0x1p23f; e0 = -23; }
    uint32_t b = f2u(x);
    int e = (int)(b >> 23) - 127 + e0;
    float m = u2f((b & 0x007fffffu) | 0x3f800000u);
    if (m > DM_SQRT2) { m = m * 0.5f; e = e + 1; }
    float f = m - 1.0f;
    float s = f / (m + 1.0f);
    float z = s * s;
    float p = DM_INV_11;
    p = fmaf(p, z, DM_INV_9);
    p = fmaf(p, z, DM_INV_7);
    p = fmaf(p, z, DM_INV_5);
    p = fmaf(p, z, DM_INV_3);
    float t = 2.0f * s;
    float lnm = fmaf(t * z, p, t);
    float ef = (float)e;
    return fmaf(ef, DM_LN2_HI, fmaf(ef, DM_LN2_LO, lnm));
}

/* Reduce x by pi/2: returns r in about [-pi/4, pi/4] and the quadrant. */
static inline float reduce_pio2(float x, int *quadrant) {
    float k = rintf(x * DM_TWO_OVER_PI);
    float r = fmaf(-k, DM_PIO2_1, x);
    r = fmaf(-k, DM_PIO2_2, r);
    *quadrant = ((int)k) & 3;
    return r;
}

static inline float sin_poly(float r) {
    float z = r * r;
    float p = DM_SIN_C4;
    p = fmaf(p, z, DM_SIN_C3);
    p = fmaf(p, z, DM_SIN_C2);
    p = fmaf(p, z, DM_SIN_C1);
    return fmaf(r * z, p, r);
}

static inline float cos_poly(float r) {
    float z = r * r;
    float p = DM_COS_C5;
    p = fmaf(p, z, DM_COS_C4);
    p = fmaf(p, z, DM_COS_C3);
    p = fmaf(p, z, DM_COS_C2);
    p = fmaf(p, z, -0.5f);
    return fmaf(z, p, 1.0f);
}

static inline void sincos_det(float x, float *s, float *c) {
    int q;
    float r = reduce_pio2(x, &q);
    float sp = sin_poly(r);
    float cp = cos_poly(r);
    switch (q) {
    case 0: *s = sp; *c = cp; break;
    case 1: *s = cp; *c = -sp; break;
    case 2: *s = -sp; *c = -cp; break;
    default: *s = -cp; *c = sp; break;
    }
}

float orc_sinf(float x) { float s, c; sincos_det(x, &s, &c); return s; }
float orc_cosf(float x) { float s, c; sincos_det(x, &s, &c); return c; }
float orc_tanf(float x) { float s, c; sincos_det(x, &s, &c); return s / c; }

/* atan on a in [0, 1]. */
static inline float atan_unit(float a) {
    float base = 0.0f;
    float t = a;
    if (a > DM_TAN_PI_12) {
        t = (a * DM_SQRT3 - 1.0f) / (a + DM_SQRT3);
        base = DM_PI_6;
    }
    float z = t * t;
    float p = DM_INV_13;
    p = fmaf(p, z, -DM_INV_11);
    p = fmaf(p, z, DM_INV_9);
    p = fmaf(p, z, -DM_INV_7);
    p = fmaf(p, z, DM_INV_5);
    p = fmaf(p, z, -DM_INV_3);
    float r = fmaf(t * z, p, t);
    return base + r;
}

float orc_atanf(float x) {
    float ax = fabsf(x);
    float r;
    if (ax > 1.0f) r = DM_PI_2 - atan_unit(1.0f / ax);
    else r = atan_unit(ax);
    return x < 0.0f ? -r : r;
}

float orc_atan2f(float y, float x) {
    float ax = fabsf(x), ay = fabsf(y);
    float mx = ax > ay ? ax : ay;
    float mn = ax > ay ? ay : ax;
    float a = mx == 0.0f ? 0.0f : mn / mx;
    float r = atan_unit(a);
    if (ay > ax) r = DM_PI_2 - r;
    if (x < 0.0f) r = DM_PI - r;
    return y < 0.0f ? -r : r;
}

float orc_acosf(float x) {
    float s = sqrtf(fabsf((1.0f - x) * (1.0f + x)));
    return orc_atan2f(s, x);
}

void orc_math_apply(int fn, const float *in, const float *in2, float *out, uint32_t n) {
    for (uint32_t i = 0; i < n; ++i) {
        float v = in[i];
        switch (fn) {
        case 0: out[i] = orc_expf(v); break;
        case 1: out[i] = orc_logf(v); break;
        case 2: out[i] = orc_sinf(v); break;
        case 3: out[i] = orc_cosf(v); break;
        case 4: out[i] = orc_tanf(v); break;
        case 5: out[i] = orc_atanf(v); break;
        case 6: out[i] = orc_acosf(v); break;
        case 7: out[i] = orc_atan2f(v, in2[i]); break;
        default: out[i] = NAN; break;
        }
    }
}
