// kernels_misc.cu -- RNG seeding (jump), the RNG known-answer wrapper and
// the math self-evaluation entry point.
//
// References: xoshiro128_seed_streams, Rust-CUDA/src/main.rs:1446-1496 (host,
// O(128 n) sequential jumps); xoshiro128p_test_wrapper, :1341-1357.
//
// Seeding on the GPU: xoshiro128+ is linear over GF(2), so stream k = J^k m
// (m = master state, J = the 128x128 bit matrix of one jump).  The matrices
// J^(2^b), b = 4..27, are generated at build time (gen_jump_tables.py) into
// constant memory.  Thread t produces streams 16t..16t+15: it forms J^(16t) m
// from the set bits of 16t (one 128-column matrix-vector product per level,
// all lanes reading the same column: a constant-cache broadcast), then
// applies 15 sequential jumps.  Bit-identical to the sequential host loop.
#include "common.cuh"
#include "detmath.cuh"
#include "internal.h"
#include "rng.cuh"
#include "tma.cuh"

#include "generated/jump_tables.inc"

namespace cudapic {

constexpr uint32_t SEED_CHUNK = 1u << CUDAPIC_JUMP_FIRST_LEVEL;

__device__ __forceinline__ uint4 jump_seq(uint4 s) {
    const uint32_t J[4] = {0x8764000bu, 0xf542d2d3u, 0x6fa035c3u, 0x77f2db5bu};
    uint4 acc = make_uint4(0, 0, 0, 0);
    Xoshiro128p r{s.x, s.y, s.z, s.w};
#pragma unroll
    for (int w = 0; w < 4; ++w) {
#pragma unroll
        for (int b = 0; b < 32; ++b) {
            if (J[w] & (1u << b)) {
                acc.x ^= r.s0;
                acc.y ^= r.s1;
                acc.z ^= r.s2;
                acc.w ^= r.s3;
            }
            r.next();
        }
    }
    return acc;
}

__global__ void __launch_bounds__(256)
    seed_streams_kernel(uint4 master, uint32_t n, uint32_t *__restrict__ r0, uint32_t *__restrict__ r1,
                        uint32_t *__restrict__ r2, uint32_t *__restrict__ r3) {
    const uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
    const uint64_t k0 = (uint64_t)t * SEED_CHUNK;
    if (k0 >= n) return;
    uint4 s = master;
    for (int l = 0; l < CUDAPIC_JUMP_LEVELS; ++l) {
        const uint32_t use = 0u - (uint32_t)((k0 >> (l + CUDAPIC_JUMP_FIRST_LEVEL)) & 1u);
        uint4 acc = make_uint4(0, 0, 0, 0);
        const uint32_t words[4] = {s.x, s.y, s.z, s.w};
#pragma unroll
        for (int w = 0; w < 4; ++w) {
#pragma unroll 8
            for (int b = 0; b < 32; ++b) {
                const uint32_t m = 0u - ((words[w] >> b) & 1u);
                const uint4 c = c_jump_pow[l][w * 32 + b];
                acc.x ^= c.x & m;
                acc.y ^= c.y & m;
                acc.z ^= c.z & m;
                acc.w ^= c.w & m;
            }
        }
        s.x = (acc.x & use) | (s.x & ~use);
        s.y = (acc.y & use) | (s.y & ~use);
        s.z = (acc.z & use) | (s.z & ~use);
        s.w = (acc.w & use) | (s.w & ~use);
    }
    for (uint32_t c = 0; c < SEED_CHUNK; ++c) {
        const uint64_t k = k0 + c;
        if (k >= n) break;
        r0[k] = s.x;
        r1[k] = s.y;
        r2[k] = s.z;
        r3[k] = s.w;
        if (c + 1 < SEED_CHUNK && k + 1 < n) s = jump_seq(s);
    }
}

__global__ void xoshiro_test_kernel(uint32_t s0, uint32_t s1, uint32_t s2, uint32_t s3, uint32_t *dest) {
    Xoshiro128p r{s0, s1, s2, s3};
    dest[0] = r.next();
    dest[1] = r.s0;
    dest[2] = r.s1;
    dest[3] = r.s2;
    dest[4] = r.s3;
}

__global__ void math_eval_kernel(int fn, const float *__restrict__ in, const float *__restrict__ in2,
                                 float *__restrict__ out, uint32_t n) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float v = in[i];
    float r;
    switch (fn) {
    case 0: r = dm::expf_det(v); break;
    case 1: r = dm::logf_det(v); break;
    case 2: r = dm::sinf_det(v); break;
    case 3: r = dm::cosf_det(v); break;
    case 4: r = dm::tanf_det(v); break;
    case 5: r = dm::atanf_det(v); break;
    case 6: r = dm::acosf_det(v); break;
    default: r = dm::atan2f_det(v, in2[i]); break;
    }
    out[i] = r;
}

// Self-test of the bounded waits: thread 0 arms an mbarrier for 16 bytes of
// transfer that no copy will deliver, and every thread waits on it with a
// limit of `limit` SM clocks.  The wait runs out and the CTA reports
// CUDAPIC_DEVERR_TIMEOUT into dev_err, the route a stage wait of the
// streaming kernels takes when a bulk copy does not complete.  No copy is
// issued, so nothing is in flight when the kernel returns.
__global__ void wait_timeout_probe_kernel(uint32_t *dev_err, long long limit) {
    __shared__ __align__(8) uint64_t bar;
    if (threadIdx.x == 0) {
        mbar_init(&bar, 1);
        fence_mbar_init();
    }
    __syncthreads();
    if (threadIdx.x == 0) mbar_arrive_expect_tx(&bar, 16u);
    __syncthreads();
    const bool ok = mbar_wait_bounded(&bar, 0u, limit);
    if (__syncthreads_or(!ok) && threadIdx.x == 0) set_dev_err(dev_err, CUDAPIC_DEVERR_TIMEOUT);
}

int launch_wait_timeout_probe(uint32_t *dev_err, long long limit, cudaStream_t stream) {
    wait_timeout_probe_kernel<<<1, 64, 0, stream>>>(dev_err, limit);
    return check_launch("wait_timeout_probe");
}

}  // namespace cudapic

using namespace cudapic;

extern "C" int cudapic_xoshiro128p_test_wrapper(uint32_t s0, uint32_t s1, uint32_t s2, uint32_t s3, uint32_t *dest,
                                                cudapic_stream_t stream) {
    CUDAPIC_REQUIRE(dest, "xoshiro128p_test_wrapper: null pointer");
    xoshiro_test_kernel<<<1, 1, 0, (cudaStream_t)stream>>>(s0, s1, s2, s3, dest);
    return check_launch("xoshiro128p_test_wrapper");
}

extern "C" int cudapic_xoshiro128_seed_streams(const uint32_t master[4], uint32_t n, uint32_t *rng0,
                                               uint32_t *rng1, uint32_t *rng2, uint32_t *rng3,
                                               cudapic_stream_t stream) {
    CUDAPIC_REQUIRE(master && rng0 && rng1 && rng2 && rng3, "xoshiro128_seed_streams: null pointer");
    CUDAPIC_REQUIRE((master[0] | master[1] | master[2] | master[3]) != 0u,
                    "xoshiro128_seed_streams: master state must not be all zero");
    CUDAPIC_REQUIRE((uint64_t)n <= (1ull << (CUDAPIC_JUMP_FIRST_LEVEL + CUDAPIC_JUMP_LEVELS)),
                    "xoshiro128_seed_streams: n > 2^28");
    if (n == 0) return CUDAPIC_OK;
    const uint32_t threads = (n + SEED_CHUNK - 1) / SEED_CHUNK;
    const uint4 m = make_uint4(master[0], master[1], master[2], master[3]);
    seed_streams_kernel<<<(threads + 255) / 256, 256, 0, (cudaStream_t)stream>>>(m, n, rng0, rng1, rng2, rng3);
    return check_launch("xoshiro128_seed_streams");
}

extern "C" int cudapic_math_eval(int fn, const float *in, const float *in2, float *out, uint32_t n,
                                 cudapic_stream_t stream) {
    CUDAPIC_REQUIRE(in && out && fn >= 0 && fn <= 7 && (fn != 7 || in2), "math_eval: bad arguments");
    if (n == 0) return CUDAPIC_OK;
    math_eval_kernel<<<(n + 255) / 256, 256, 0, (cudaStream_t)stream>>>(fn, in, in2, out, n);
    return check_launch("math_eval");
}
