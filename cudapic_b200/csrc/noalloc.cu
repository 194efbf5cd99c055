// noalloc.cu -- the fused electron step for callers that cannot allocate.
//
// cudapic_step_electrons needs one scratch word from its caller: a slot
// counter, zero on entry, that collects the survivors and spawned electrons;
// the caller then copies it into its electron count.  Some callers cannot
// provide it: a host whose device memory belongs to its own pool or
// framework and hands this library only its particle buffers (a managed
// runtime calling through cgo, JNI or ctypes; a plugin with a fixed memory
// budget), or code that must not call cudaMalloc because it synchronises the
// device.  cudapic_step_electrons_noalloc takes no scratch from the caller:
// the slot counter and the completion ticket of the kernel live in the
// library-owned array below, and the last CTA of the kernel writes the new
// count into the caller's n_e in place, so no copy follows the launch.
//
// The array is a file-scope __device__ variable: every GPU that loads the
// library holds its 256 bytes until the process exits.  Host code cannot use
// the array's name as a device address; every call looks the address up with
// cudaGetSymbolAddress in the calling thread's current context (a cheap
// host-side lookup), so a context of the caller's own, or the module that a
// cudaDeviceReset reloads, gets its own array's address.  Calls share the
// array, so two calls whose kernels overlap on one GPU race on its counters.
#include <cuda_runtime.h>

#include "internal.h"

// [0] slot counter of the survivors and spawned electrons, [1] CTA ticket;
// the rest is unused.  Both must be zero when a kernel starts.
static __device__ __align__(256) uint32_t g_step_scratch[CUDAPIC_NOALLOC_SCRATCH_BYTES / sizeof(uint32_t)];

namespace {

// Device address of g_step_scratch in the current context.
int scratch_address(uint32_t **out) {
    void *p = nullptr;
    CUDAPIC_CHECK(cudapic::check_cuda(cudaGetSymbolAddress(&p, g_step_scratch),
                                      "step_electrons_noalloc: cudaGetSymbolAddress"));
    *out = static_cast<uint32_t *>(p);
    return CUDAPIC_OK;
}

}  // namespace

using namespace cudapic;

extern "C" int cudapic_step_electrons_noalloc(const float *efield, const float *src_x, const float *src_vx,
                                              const float *src_vy, const float *src_vz, float *dst_x, float *dst_vx,
                                              float *dst_vy, float *dst_vz, uint32_t *rng0, uint32_t *rng1,
                                              uint32_t *rng2, uint32_t *rng3, const float *total_cs_e, const float *cs,
                                              float sigma_max_e, float *i_x, float *i_vx, float *i_vy, float *i_vz,
                                              uint32_t *n_e, uint32_t *n_i, float *e_next_density,
                                              float *i_next_density, const cudapic_grid *grid,
                                              cudapic_stream_t stream) {
    CUDAPIC_CHECK(validate_grid(grid));
    CUDAPIC_REQUIRE(efield && src_x && src_vx && src_vy && src_vz && dst_x && dst_vx && dst_vy && dst_vz && rng0 &&
                        rng1 && rng2 && rng3 && total_cs_e && cs && i_x && i_vx && i_vy && i_vz && n_e && n_i &&
                        e_next_density && i_next_density,
                    "step_electrons_noalloc: null pointer");
    CUDAPIC_REQUIRE(sigma_max_e >= 0.0f, "step_electrons_noalloc: sigma_max_e must be the largest entry of total_cs_e");
    // The shared 32-bit slot counter may overshoot the capacity briefly while
    // spawns that do not fit give their claims back; below 2^31 it never wraps.
    CUDAPIC_REQUIRE(grid->capacity <= CUDAPIC_NOALLOC_MAX_CAPACITY,
                    "step_electrons_noalloc: capacity exceeds CUDAPIC_NOALLOC_MAX_CAPACITY (2^31) slots");
    const void *planes[8] = {src_x, src_vx, src_vy, src_vz, rng0, rng1, rng2, rng3};
    CUDAPIC_REQUIRE(electron_step_eligible(planes, 8, grid->capacity),
                    "step_electrons_noalloc: planes must be 16-byte aligned and capacity a multiple of 4");
    uint32_t *scratch = nullptr;
    CUDAPIC_CHECK(scratch_address(&scratch));
    // the array keeps the previous call's contents: both counters start at zero
    CUDAPIC_CHECK(check_cuda(cudaMemsetAsync(scratch, 0, 2 * sizeof(uint32_t), (cudaStream_t)stream),
                             "step_electrons_noalloc: clear scratch"));
    StepLink link;
    link.ticket = scratch + 1;
    link.dst = n_e;
    link.src = scratch;
    link.clear_src = 1;
    return launch_electron_step(efield, src_x, src_vx, src_vy, src_vz, dst_x, dst_vx, dst_vy, dst_vz, rng0, rng1, rng2,
                                rng3, total_cs_e, cs, sigma_max_e, i_x, i_vx, i_vy, i_vz, scratch, n_e, n_i,
                                e_next_density, i_next_density, *grid, (cudaStream_t)stream, link);
}
