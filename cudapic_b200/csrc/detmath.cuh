// detmath.cuh -- f32 transcendental functions of the collision kernels.
//
// The reference evaluates them with PTX approximation instructions
// (sqrt/sin/cos/ex2/lg2/rcp.approx) and its own 3-term atan polynomial
// (Rust-CUDA/src/main.rs:680-858).  Here every function is built from
// IEEE-754 +, -, *, /, sqrt and fmaf in a fixed order, so the result is the
// same bit pattern on any IEEE machine.  That makes collision decisions and
// post-collision velocities reproducible by a CPU restatement.  The file is
// compiled with -fmad=false: no a*b+c is contracted unless written as fmaf.
//
// Methods (all published, coefficients are exact Taylor coefficients
// rounded to float, written in hexadecimal):
//   exp    Cody & Waite (1980) reduction x = k ln2 + r with two-word ln2,
//          degree-7 Taylor polynomial for e^r on |r| <= ln2/2.
//   log    x = m 2^e, m in [sqrt(1/2), sqrt(2)); ln m = 2 atanh((m-1)/(m+1)),
//          series to s^11.
//   sin/cos  Cody & Waite reduction by pi/2 (two-word pi/2, valid for the
//          |x| < 16 met on this path); Taylor degree 9 / 10 on |r| <= pi/4.
//   atan   reflection 1/a for a > 1; atan(a) = pi/6 + atan((a sqrt3-1)/(a+sqrt3))
//          for a > tan(pi/12); Taylor series to t^13.
//   atan2  quadrant logic on atan(min/max); acos(x) = atan2(sqrt((1-x)(1+x)), x).
// Measured against libm in double: all within 2.7 ulp over the input ranges
// of this path.
#pragma once

#include <cstdint>

namespace cudapic {
namespace dm {

constexpr float LOG2E = 0x1.715476p+0f;
constexpr float LN2_HI = 0x1.62e430p-1f;
constexpr float LN2_LO = -0x1.05c610p-29f;
constexpr float INV_FACT3 = 0x1.555556p-3f;
constexpr float INV_FACT4 = 0x1.555556p-5f;
constexpr float INV_FACT5 = 0x1.111112p-7f;
constexpr float INV_FACT6 = 0x1.6c16c2p-10f;
constexpr float INV_FACT7 = 0x1.a01a02p-13f;
constexpr float SQRT2 = 0x1.6a09e6p+0f;
constexpr float INV_3 = 0x1.555556p-2f;
constexpr float INV_5 = 0x1.99999ap-3f;
constexpr float INV_7 = 0x1.24924ap-3f;
constexpr float INV_9 = 0x1.c71c72p-4f;
constexpr float INV_11 = 0x1.745d18p-4f;
constexpr float INV_13 = 0x1.3b13b2p-4f;
constexpr float TWO_OVER_PI = 0x1.45f306p-1f;
constexpr float PIO2_1 = 0x1.921fb6p+0f;
constexpr float PIO2_2 = -0x1.777a5cp-25f;
constexpr float SIN_C1 = -0x1.555556p-3f;
constexpr float SIN_C2 = 0x1.111112p-7f;
constexpr float SIN_C3 = -0x1.a01a02p-13f;
constexpr float SIN_C4 = 0x1.71de3ap-19f;
constexpr float COS_C2 = 0x1.555556p-5f;
constexpr float COS_C3 = -0x1.6c16c2p-10f;
constexpr float COS_C4 = 0x1.a01a02p-16f;
constexpr float COS_C5 = -0x1.27e4fcp-22f;
constexpr float SQRT3 = 0x1.bb67aep+0f;
constexpr float PI_6 = 0x1.0c1524p-1f;
constexpr float TAN_PI_12 = 0x1.126146p-2f;
constexpr float PI_2 = 0x1.921fb6p+0f;
constexpr float PI = 0x1.921fb6p+1f;

// p * 2^k, k in [-252, 254], by two exact power-of-two scalings.
__device__ __forceinline__ float scale2i(float p, int k) {
    int k1 = k / 2;
    int k2 = k - k1;
    return (p * __uint_as_float((uint32_t)(k1 + 127) << 23)) * __uint_as_float((uint32_t)(k2 + 127) << 23);
}

__device__ __forceinline__ float expf_det(float x) {
    if (x != x) return x;
    if (x > 88.72283f) return __int_as_float(0x7f800000);
    if (x < -103.9721f) return 0.0f;
    float k = rintf(x * LOG2E);
    float r = fmaf(-k, LN2_HI, x);
    r = fmaf(-k, LN2_LO, r);
    float p = INV_FACT7;
    p = fmaf(p, r, INV_FACT6);
    p = fmaf(p, r, INV_FACT5);
    p = fmaf(p, r, INV_FACT4);
    p = fmaf(p, r, INV_FACT3);
    p = fmaf(p, r, 0.5f);
    p = fmaf(p, r, 1.0f);
    p = fmaf(p, r, 1.0f);
    return scale2i(p, (int)k);
}

__device__ __forceinline__ float logf_det(float x) {
    if (x != x) return x;
    if (x < 0.0f) return __int_as_float(0x7fc00000);
    if (x == 0.0f) return __int_as_float(0xff800000);
    if (x == __int_as_float(0x7f800000)) return x;
    int e0 = 0;
    if (x < 0x1p-126f) {
        x = x * 0x1p23f;
        e0 = -23;
    }
    uint32_t b = __float_as_uint(x);
    int e = (int)(b >> 23) - 127 + e0;
    float m = __uint_as_float((b & 0x007fffffu) | 0x3f800000u);
    if (m > SQRT2) {
        m = m * 0.5f;
        e = e + 1;
    }
    float f = m - 1.0f;
    float s = f / (m + 1.0f);
    float z = s * s;
    float p = INV_11;
    p = fmaf(p, z, INV_9);
    p = fmaf(p, z, INV_7);
    p = fmaf(p, z, INV_5);
    p = fmaf(p, z, INV_3);
    float t = 2.0f * s;
    float lnm = fmaf(t * z, p, t);
    float ef = (float)e;
    return fmaf(ef, LN2_HI, fmaf(ef, LN2_LO, lnm));
}

__device__ __forceinline__ float sin_poly(float r) {
    float z = r * r;
    float p = SIN_C4;
    p = fmaf(p, z, SIN_C3);
    p = fmaf(p, z, SIN_C2);
    p = fmaf(p, z, SIN_C1);
    return fmaf(r * z, p, r);
}

__device__ __forceinline__ float cos_poly(float r) {
    float z = r * r;
    float p = COS_C5;
    p = fmaf(p, z, COS_C4);
    p = fmaf(p, z, COS_C3);
    p = fmaf(p, z, COS_C2);
    p = fmaf(p, z, -0.5f);
    return fmaf(z, p, 1.0f);
}

__device__ __forceinline__ void sincosf_det(float x, float *s, float *c) {
    float k = rintf(x * TWO_OVER_PI);
    float r = fmaf(-k, PIO2_1, x);
    r = fmaf(-k, PIO2_2, r);
    int q = ((int)k) & 3;
    float sp = sin_poly(r);
    float cp = cos_poly(r);
    float ss, cc;
    if (q == 0) {
        ss = sp; cc = cp;
    } else if (q == 1) {
        ss = cp; cc = -sp;
    } else if (q == 2) {
        ss = -sp; cc = -cp;
    } else {
        ss = -cp; cc = sp;
    }
    *s = ss;
    *c = cc;
}

__device__ __forceinline__ float sinf_det(float x) { float s, c; sincosf_det(x, &s, &c); return s; }
__device__ __forceinline__ float cosf_det(float x) { float s, c; sincosf_det(x, &s, &c); return c; }
__device__ __forceinline__ float tanf_det(float x) { float s, c; sincosf_det(x, &s, &c); return s / c; }

__device__ __forceinline__ float atan_unit(float a) {
    float base = 0.0f;
    float t = a;
    if (a > TAN_PI_12) {
        t = (a * SQRT3 - 1.0f) / (a + SQRT3);
        base = PI_6;
    }
    float z = t * t;
    float p = INV_13;
    p = fmaf(p, z, -INV_11);
    p = fmaf(p, z, INV_9);
    p = fmaf(p, z, -INV_7);
    p = fmaf(p, z, INV_5);
    p = fmaf(p, z, -INV_3);
    float r = fmaf(t * z, p, t);
    return base + r;
}

__device__ __forceinline__ float atanf_det(float x) {
    float ax = fabsf(x);
    float r;
    if (ax > 1.0f) r = PI_2 - atan_unit(1.0f / ax);
    else r = atan_unit(ax);
    return x < 0.0f ? -r : r;
}

__device__ __forceinline__ float atan2f_det(float y, float x) {
    float ax = fabsf(x), ay = fabsf(y);
    float mx = ax > ay ? ax : ay;
    float mn = ax > ay ? ay : ax;
    float a = mx == 0.0f ? 0.0f : mn / mx;
    float r = atan_unit(a);
    if (ay > ax) r = PI_2 - r;
    if (x < 0.0f) r = PI - r;
    return y < 0.0f ? -r : r;
}

__device__ __forceinline__ float acosf_det(float x) {
    float s = sqrtf(fabsf((1.0f - x) * (1.0f + x)));
    return atan2f_det(s, x);
}

}  // namespace dm
}  // namespace cudapic
