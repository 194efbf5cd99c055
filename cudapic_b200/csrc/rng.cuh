// rng.cuh -- xoshiro128+ 1.0 per-slot streams (Rust-CUDA/src/main.rs:860-969).
//
// The state of slot i lives in four u32 planes rng0..rng3[i].  A kernel loads
// the four words once, draws as many numbers as the particle needs from
// registers and stores the state once.
#pragma once

#include <cstdint>

#include "detmath.cuh"

namespace cudapic {

struct Xoshiro128p {
    uint32_t s0, s1, s2, s3;

    __device__ __forceinline__ uint32_t next() {
        uint32_t result = s0 + s3;
        uint32_t t = s1 << 9;
        s2 ^= s0;
        s3 ^= s1;
        s1 ^= s2;
        s0 ^= s3;
        s2 ^= t;
        s3 = __funnelshift_l(s3, s3, 11);
        return result;
    }

    // u32_to_real (Rust-CUDA/src/main.rs:883-885): 23 high bits as a float
    // in [0, 1), exact.
    __device__ __forceinline__ float uniform() {
        return __uint_as_float(0x3F800000u | (next() >> 9)) - 1.0f;
    }

    // rng_next_three_normal (Rust-CUDA/src/main.rs:908-969): four uniforms
    // clamped to >= 1e-9, Box-Muller on (u1,u2) and (u3,u4), three of the four
    // normals returned, scaled by sigma.  ln(u) is evaluated directly (the
    // reference forms it as lg2.approx(u) * ln 2).
    __device__ __forceinline__ void three_normal(float sigma, float &a, float &b, float &c) {
        float u1 = fmaxf(uniform(), 1e-9f);
        float u2 = fmaxf(uniform(), 1e-9f);
        float u3 = fmaxf(uniform(), 1e-9f);
        float u4 = fmaxf(uniform(), 1e-9f);
        float rad1 = sqrtf(-2.0f * dm::logf_det(u1));
        float ang1 = 6.28318530717958647692f * u2;
        float s1, c1;
        dm::sincosf_det(ang1, &s1, &c1);
        float z0 = rad1 * c1;
        float z1 = rad1 * s1;
        float rad2 = sqrtf(-2.0f * dm::logf_det(u3));
        float ang2 = 6.28318530717958647692f * u4;
        float z2 = rad2 * dm::cosf_det(ang2);
        a = z0 * sigma;
        b = z1 * sigma;
        c = z2 * sigma;
    }
};

}  // namespace cudapic
