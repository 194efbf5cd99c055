// batch.cpp -- the batch driver: many discharges stepped in lockstep, one
// launch per kernel of the step for all of them.
//
// Reference: main()'s per-step sequence (Rust-CUDA/src/main.rs:1725-1808),
// which runs one discharge; the fused driver of state.cpp runs it per
// discharge with one captured graph of 2 N_SUB steps.  A batch runs the same
// sequence -- Poisson, [ion push], fused electron step, [ion collisions],
// [EEPF] -- for every discharge of the batch in one launch each
// (kernels_batch.cu), in one captured graph of 2 N_SUB steps.
//
// The discharges stay cudapic_state objects: their buffers, counters,
// tables and measurements are used in place, and every state API call keeps
// working between batch runs.  The batch records each state's buffer
// orientation when it builds its descriptors; a run checks that nothing else
// moved a state since (else it rebuilds them) and afterwards stores the
// states' new sides, step counts and measurement windows.
#include <cuda_runtime.h>

#include <algorithm>
#include <array>
#include <cstring>
#include <new>
#include <vector>

#include "batch_internal.h"
#include "internal.h"
#include "state_impl.h"

using namespace cudapic;

struct cudapic_batch {
    int device = 0;
    std::vector<cudapic_state *> states;
    cudaStream_t stream = nullptr;
    std::vector<cudaEvent_t> ready;  // per state: its stream's work before a run
    cudaEvent_t done = nullptr;
    BatchDisc *desc = nullptr;
    uint32_t *counts = nullptr;      // [2][D] written by the batched Poisson solve
    uint32_t max_n_g = 0, flags = 0;
    uint64_t cap_sum = 0;
    bool built = false;
    // orientation of each state at the build: e side, i side, e_cur, i_cur
    std::vector<std::array<int, 4>> origin;
    // roles relative to the build (the same for every discharge)
    int se = 0, si = 0, ecur = 0, icur = 0;
    cudaGraphExec_t graph[2] = {nullptr, nullptr};  // [measure]
    int graph_key[2][4] = {{-1, -1, -1, -1}, {-1, -1, -1, -1}};

    uint32_t count() const { return (uint32_t)states.size(); }
};

namespace {

void destroy_graphs(cudapic_batch *b) {
    for (auto &g : b->graph) {
        if (g) cudaGraphExecDestroy(g);
        g = nullptr;
    }
}

bool oriented(const cudapic_batch *b, uint32_t k) {
    const cudapic_state *s = b->states[k];
    const auto &o = b->origin[k];
    return s->side[0] == (o[0] ^ b->se) && s->side[1] == (o[1] ^ b->si) && s->e_cur == (o[2] ^ b->ecur) &&
           s->i_cur == (o[3] ^ b->icur);
}

// Descriptors of the states as they are oriented now; roles back to zero.
int build(cudapic_batch *b) {
    const uint32_t D = b->count();
    std::vector<BatchDisc> host(D);
    b->origin.resize(D);
    for (uint32_t k = 0; k < D; ++k) {
        cudapic_state *s = b->states[k];
        BatchDisc &d = host[k];
        std::memset(&d, 0, sizeof(d));
        d.g = s->grid;
        for (int sp = 0; sp < 2; ++sp) {
            for (int side = 0; side < 2; ++side) {
                const int a = s->side[sp] ^ side;
                d.x[sp][side] = s->x[sp][a];
                d.vx[sp][side] = s->vx[sp][a];
                d.vy[sp][side] = s->vy[sp][a];
                d.vz[sp][side] = s->vz[sp][a];
            }
            for (int p = 0; p < 4; ++p) d.rng[sp][p] = s->rng[sp][p];
        }
        for (int r = 0; r < 2; ++r) {
            d.e_dens[r] = s->e_dens[s->e_cur ^ r];
            d.i_dens[r] = s->i_dens[s->i_cur ^ r];
        }
        d.counters = s->counters;
        d.efield = s->efield;
        d.pot = s->pot;
        d.pot0_table = s->pot0_table;
        d.cs = s->cs;
        d.sigma_tot_e = s->sigma_tot_e;
        d.sigma_tot_i = s->sigma_tot_i;
        d.sigma_max_e = s->sigma_max_e;
        d.wall = s->wall;
        d.mcount = s->mcount;
        d.cumul_e = s->cumul_e;
        d.cumul_i = s->cumul_i;
        d.esum = s->esum;
        d.eepf = s->eepf;
        b->origin[k] = {s->side[0], s->side[1], s->e_cur, s->i_cur};
    }
    CUDAPIC_CHECK(check_cuda(cudaMemcpy(b->desc, host.data(), D * sizeof(BatchDisc), cudaMemcpyHostToDevice),
                             "batch: upload descriptors"));
    b->se = b->si = b->ecur = b->icur = 0;
    destroy_graphs(b);
    b->built = true;
    return CUDAPIC_OK;
}

// One step of every discharge (the order of state.cpp's fused step).
int enqueue_batch_step(cudapic_batch *b, bool ion_step, bool measure) {
    PdlScope pdl(true);
    const uint32_t D = b->count();
    cudaStream_t st = b->stream;
    if (ion_step) b->icur ^= 1;  // the buffer that collected the period's ion deposits becomes current
    CUDAPIC_CHECK(launch_batch_poisson(b->desc, b->counts, D, b->max_n_g, b->flags, b->ecur, b->icur, ion_step ? 1 : 0,
                                       measure ? 1 : 0, st));
    if (ion_step) {
        StepRoles ri{};
        ri.src = b->si;
        ri.dst = b->si ^ 1;
        ri.ion_side = b->si ^ 1;
        ri.dens = b->icur ^ 1;
        ri.dens_i = b->icur ^ 1;
        ri.measure = measure ? 1 : 0;
        CUDAPIC_CHECK(launch_batch_step(false, b->desc, b->counts + D, D, b->cap_sum, b->max_n_g, ri, st));
        b->si ^= 1;
    }
    StepRoles re{};
    re.src = b->se;
    re.dst = b->se ^ 1;
    re.ion_side = b->si;
    re.dens = b->ecur ^ 1;
    re.dens_i = b->icur ^ 1;
    re.measure = measure ? 1 : 0;
    CUDAPIC_CHECK(launch_batch_step(true, b->desc, b->counts, D, b->cap_sum, b->max_n_g, re, st));
    b->se ^= 1;
    b->ecur ^= 1;
    if (ion_step) CUDAPIC_CHECK(launch_batch_collisions_i(b->desc, D, b->cap_sum, b->si, measure ? 1 : 0, st));
    if (measure) CUDAPIC_CHECK(launch_batch_eepf(b->desc, D, b->cap_sum, b->se, st));
    return CUDAPIC_OK;
}

int build_graph(cudapic_batch *b, uint64_t first_step, bool measure) {
    const int m = measure ? 1 : 0;
    cudapic_state *s0 = b->states[0];
    const uint64_t period = 2ull * s0->params.n_sub;
    const int roles0[4] = {b->se, b->si, b->ecur, b->icur};
    cudaGraph_t graph = nullptr;
    CUDAPIC_CHECK(check_cuda(cudaStreamBeginCapture(b->stream, cudaStreamCaptureModeThreadLocal), "begin capture"));
    int rc = CUDAPIC_OK;
    for (uint64_t k = 0; k < period && rc == CUDAPIC_OK; ++k)
        rc = enqueue_batch_step(b, state_is_ion_step(s0, first_step + k), measure);
    cudaError_t e = cudaStreamEndCapture(b->stream, &graph);
    // 2 N_SUB steps return every role to its start
    b->se = roles0[0];
    b->si = roles0[1];
    b->ecur = roles0[2];
    b->icur = roles0[3];
    std::memcpy(b->graph_key[m], roles0, sizeof(roles0));
    if (rc != CUDAPIC_OK) {
        if (graph) cudaGraphDestroy(graph);
        return rc;
    }
    CUDAPIC_CHECK(check_cuda(e, "end capture"));
    e = cudaGraphInstantiate(&b->graph[m], graph, 0);
    cudaGraphDestroy(graph);
    return check_cuda(e, "cudaGraphInstantiate");
}

}  // namespace

extern "C" int cudapic_batch_create(cudapic_state *const *states, uint32_t count, cudapic_batch **out) {
    CUDAPIC_REQUIRE(states && out, "batch_create: null pointer");
    *out = nullptr;
    CUDAPIC_REQUIRE(count >= 1 && count <= BATCH_MAX_DISCHARGES, "batch_create: count must be in [1, 1024]");
    const cudapic_state *s0 = states[0];
    CUDAPIC_REQUIRE(s0, "batch_create: null state");
    uint64_t cap_sum = 0;
    uint32_t max_n_g = 0;
    for (uint32_t k = 0; k < count; ++k) {
        const cudapic_state *s = states[k];
        CUDAPIC_REQUIRE(s, "batch_create: null state");
        for (uint32_t j = 0; j < k; ++j) CUDAPIC_REQUIRE(states[j] != s, "batch_create: a state appears twice");
        CUDAPIC_REQUIRE(s->device == s0->device, "batch_create: the states must share one device");
        CUDAPIC_REQUIRE(s->params.n_t == s0->params.n_t && s->params.n_sub == s0->params.n_sub,
                        "batch_create: the states must share N_T and N_SUB");
        CUDAPIC_REQUIRE((s->params.flags & CUDAPIC_FLAG_POISSON_F32_SCAN) ==
                            (s0->params.flags & CUDAPIC_FLAG_POISSON_F32_SCAN),
                        "batch_create: the states must share the Poisson arithmetic flag");
        CUDAPIC_REQUIRE(s->graphs_enabled, "batch_create: N_T must be a multiple of N_SUB");
        const void *planes[8] = {s->x[0][0], s->x[0][1], s->vx[0][0], s->vx[0][1],
                                 s->rng[0][0], s->rng[0][1], s->rng[0][2], s->rng[0][3]};
        CUDAPIC_REQUIRE(electron_step_eligible(planes, 8, s->grid.capacity), "batch_create: unaligned state buffers");
        cap_sum += s->grid.capacity;
        max_n_g = std::max(max_n_g, s->grid.n_g);
    }
    CUDAPIC_REQUIRE(cap_sum <= 0x80000000ull, "batch_create: the capacities must sum to at most 2^31");
    DeviceGuard dg(s0->device);
    cudapic_batch *b = new (std::nothrow) cudapic_batch();
    if (!b) return fail(CUDAPIC_ERR_ARG, "batch_create: out of host memory");
    b->device = s0->device;
    b->states.assign(states, states + count);
    b->cap_sum = cap_sum;
    b->max_n_g = max_n_g;
    b->flags = s0->params.flags;
    auto cleanup = [&](int rc) {
        cudapic_batch_destroy(b);
        return rc;
    };
    int rc;
    if ((rc = check_cuda(cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking), "batch: stream")) ||
        (rc = check_cuda(cudaEventCreateWithFlags(&b->done, cudaEventDisableTiming), "batch: event")) ||
        (rc = check_cuda(cudaMalloc(&b->desc, count * sizeof(BatchDisc)), "batch: descriptors")) ||
        (rc = check_cuda(cudaMalloc(&b->counts, 2ull * count * sizeof(uint32_t)), "batch: counts")))
        return cleanup(rc);
    b->ready.assign(count, nullptr);
    for (auto &ev : b->ready)
        if ((rc = check_cuda(cudaEventCreateWithFlags(&ev, cudaEventDisableTiming), "batch: event")))
            return cleanup(rc);
    *out = b;
    return CUDAPIC_OK;
}

extern "C" int cudapic_batch_destroy(cudapic_batch *b) {
    if (!b) return CUDAPIC_OK;
    DeviceGuard dg(b->device);
    if (b->stream) cudaStreamSynchronize(b->stream);
    destroy_graphs(b);
    for (auto ev : b->ready)
        if (ev) cudaEventDestroy(ev);
    if (b->done) cudaEventDestroy(b->done);
    if (b->desc) cudaFree(b->desc);
    if (b->counts) cudaFree(b->counts);
    if (b->stream) cudaStreamDestroy(b->stream);
    delete b;
    return CUDAPIC_OK;
}

extern "C" cudapic_stream_t cudapic_batch_stream(const cudapic_batch *b) {
    return b ? (cudapic_stream_t)b->stream : nullptr;
}

extern "C" int cudapic_batch_synchronize(cudapic_batch *b) {
    if (!b) return fail(CUDAPIC_ERR_ARG, "batch_synchronize: null batch");
    DeviceGuard dg(b->device);
    return check_cuda(cudaStreamSynchronize(b->stream), "batch_synchronize");
}

extern "C" int cudapic_batch_run_steps(cudapic_batch *b, uint64_t n_steps) {
    if (!b) return fail(CUDAPIC_ERR_ARG, "batch_run_steps: null batch");
    DeviceGuard dg(b->device);
    const uint32_t D = b->count();
    cudapic_state *s0 = b->states[0];
    const uint64_t steps0 = s0->steps_done;
    const bool measure = s0->measure;
    bool stale = !b->built;
    for (uint32_t k = 0; k < D; ++k) {
        const cudapic_state *s = b->states[k];
        CUDAPIC_REQUIRE(s->steps_done == steps0, "batch_run_steps: the states are at different steps");
        CUDAPIC_REQUIRE(s->measure == measure, "batch_run_steps: the states differ in measurement mode");
        CUDAPIC_REQUIRE(s->fused, "batch_run_steps: a state is in unfused (reference sequence) mode");
        if (b->built && !oriented(b, k)) stale = true;
    }
    if (stale) CUDAPIC_CHECK(build(b));
    // after every state's pending work (uploads, seeding, its own steps)
    for (uint32_t k = 0; k < D; ++k) {
        CUDAPIC_CHECK(check_cuda(cudaEventRecord(b->ready[k], b->states[k]->stream), "batch: record"));
        CUDAPIC_CHECK(check_cuda(cudaStreamWaitEvent(b->stream, b->ready[k], 0), "batch: wait"));
    }
    for (uint32_t k = 0; k < D; ++k)
        if (!b->states[k]->dens_valid) CUDAPIC_CHECK(state_prime_fused(b->states[k], b->stream));
    const uint64_t period = 2ull * s0->params.n_sub;
    uint64_t step = steps0;
    int rc = CUDAPIC_OK;
    while (n_steps > 0 && rc == CUDAPIC_OK) {
        if ((step % period) == 0 && n_steps >= period) {
            const int m = measure ? 1 : 0;
            const int key[4] = {b->se, b->si, b->ecur, b->icur};
            if (b->graph[m] && std::memcmp(key, b->graph_key[m], sizeof(key)) != 0) {
                cudaGraphExecDestroy(b->graph[m]);
                b->graph[m] = nullptr;
            }
            if (!b->graph[m]) rc = build_graph(b, step, measure);
            if (rc == CUDAPIC_OK) rc = check_cuda(cudaGraphLaunch(b->graph[m], b->stream), "batch: graph launch");
            if (rc == CUDAPIC_OK) {
                step += period;
                n_steps -= period;
            }
            continue;
        }
        rc = enqueue_batch_step(b, state_is_ion_step(s0, step), measure);
        if (rc == CUDAPIC_OK) {
            step += 1;
            n_steps -= 1;
        }
    }
    // the states' bookkeeping follows what was enqueued
    const uint64_t done_steps = step - steps0;
    for (uint32_t k = 0; k < D; ++k) {
        cudapic_state *s = b->states[k];
        const auto &o = b->origin[k];
        s->side[0] = o[0] ^ b->se;
        s->side[1] = o[1] ^ b->si;
        s->e_cur = o[2] ^ b->ecur;
        s->i_cur = o[3] ^ b->icur;
        s->steps_done = step;
        if (s->measure) s->measure_steps += done_steps;
    }
    // every state's own stream continues after the batch's work
    const int rc2 = check_cuda(cudaEventRecord(b->done, b->stream), "batch: record");
    for (uint32_t k = 0; k < D && rc2 == CUDAPIC_OK; ++k)
        CUDAPIC_CHECK(check_cuda(cudaStreamWaitEvent(b->states[k]->stream, b->done, 0), "batch: wait"));
    return rc != CUDAPIC_OK ? rc : rc2;
}
