// common.cuh -- shared device helpers of the cudaPIC kernels.
#pragma once

#include <cuda_runtime.h>
#include <cstdint>

#include "../../include/cudapic.h"

namespace cudapic {

constexpr uint32_t CS_RANGES = 1000000u;   // Rust-CUDA/src/main.rs:72
constexpr float DE_CS_F = 0.001f;          // DE_CS as Real, :73
constexpr uint32_t N_EEPF = 2000u;         // :78
constexpr float DE_EEPF_F = 0.05f;         // :79
constexpr float PI_F = 3.14159265358979323846f;
constexpr float TWO_PI_F = 6.28318530717958647692f;

// Physical constants as f32 (`E_MASS as Real`, ... in Rust-CUDA/src/main.rs).
constexpr float E_MASS_F = 9.10938356e-31f;
constexpr float E_CHARGE_F = 1.60217662e-19f;
// 1/2 M_Ar / e as f32: the ion energy in eV of the flux-energy distributions
constexpr float HALF_MI_OVER_E = (float)(0.5 * 6.63352090e-26 / 1.60217662e-19);

__device__ __forceinline__ void set_dev_err(uint32_t *err, uint32_t bits) {
    if (err) atomicOr(err, bits);
}

// Live count of a species: *n clamped to the capacity (a larger count can
// only come from an overflowed spawn counter; the excess slots were never
// written).
__device__ __forceinline__ uint32_t load_count(const uint32_t *n, uint32_t capacity, uint32_t *err) {
    uint32_t v = *n;
    if (v > capacity) {
        set_dev_err(err, CUDAPIC_DEVERR_ACTIVE);
        v = capacity;
    }
    return v;
}

// CIC cell of a particle.  The reference truncates x*INV_DX and reads node
// p+1 unguarded (Rust-CUDA/src/main.rs:377-387, 600-603); a particle at
// exactly x = L would touch node N_G.  The cell is clamped to [0, N_G-2];
// for every in-range position the result equals the reference's.
__device__ __forceinline__ int cell_of(float pos, uint32_t n_g) {
    int p = (int)pos;
    if (!(pos >= 0.0f)) p = 0;
    if (p > (int)n_g - 2) p = (int)n_g - 2;
    if (p < 0) p = 0;
    return p;
}

// A slot that an in-place electron step emptied (inplace.cuh): its electron
// left through an electrode and x holds a negative marker.  Live positions
// are in [0, L]; kernels that read electron slots skip dead ones.
__device__ __forceinline__ bool slot_dead(float x) { return x < 0.0f; }

__device__ __forceinline__ bool pos_in_range(float pos, uint32_t n_g) {
    return pos >= 0.0f && pos <= (float)(n_g - 1);
}

// Programmatic dependent launch: waits until the grids this one depends on
// have completed and their memory is visible (a no-op for a launch without
// the PDL attribute), then lets the next kernel of the stream be scheduled.
// Called before the first global access that another kernel may touch.
__device__ __forceinline__ void grid_dep_wait() {
    asm volatile("griddepcontrol.wait;" ::: "memory");
    asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
}

// End of a kernel that counted particles into link.src: the last CTA to
// finish publishes the count (StepLink, internal.h).  Every thread fences its
// own counter atomics before the CTA's ticket is taken.
__device__ __forceinline__ void publish_count(uint32_t *ticket, uint32_t *dst, uint32_t *src, int clear_src,
                                              uint32_t capacity) {
    if (!ticket) return;
    __threadfence();
    __syncthreads();
    if (threadIdx.x == 0) {
        const uint32_t t = atomicAdd(ticket, 1u);
        if (t == gridDim.x - 1) {
            __threadfence();
            const uint32_t v = clear_src ? atomicExch(src, 0u) : atomicAdd(src, 0u);
            *dst = v < capacity ? v : capacity;
            *ticket = 0u;
        }
    }
}

__device__ __forceinline__ unsigned lanemask_lt() {
    unsigned m;
    asm("mov.u32 %0, %%lanemask_lt;" : "=r"(m));
    return m;
}

}  // namespace cudapic
