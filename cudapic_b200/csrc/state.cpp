// state.cpp -- the simulation state and the per-step driver of libcudapic.
//
// Reference: GpuSimState (Rust-CUDA/src/main.rs:131-350) owns SoA particle
// buffers preallocated to MAX_PARTICLES, ping-pong tmp_* buffers, 4 RNG
// planes per species, the device counters n_electrons / n_ions /
// alive_counter, the grid arrays, the cross-section tables and the
// measurement accumulators; main() (:1725-1808) enqueues, for every time
// step t, the launches and memsets below in this order.  Here:
//  * capacity, N_G, ... are runtime values (cudapic_params);
//  * each species owns its own ping-pong pair (the reference rotates one
//    shared tmp set between the species), so pointer swaps are per species;
//  * the RF phase pot0 = V cos(2 pi t / N_T) is a device table indexed by a
//    device step counter advanced by the Poisson kernel, so one captured CUDA
//    graph of 2 * N_SUB steps (electron and ion buffers back on the side
//    they started) is replayed for every RF phase;
//  * a device particle-step counter (electrons every step, ions every N_SUB
//    steps) measures the work actually done.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <string>
#include <new>
#include <vector>

#include "batch_internal.h"
#include "internal.h"
#include "state_impl.h"

namespace {
constexpr long long MBAR_PROBE_MAX_CYCLES = 1ll << 31;  // the streaming kernels' own limit
}

using namespace cudapic;

namespace cudapic {

int state_prime_fused(cudapic_state *s, cudaStream_t st) {
    const cudapic_grid &g = s->grid;
    const size_t nb = g.n_g * sizeof(float);
    const int E = 0, I = 1;
    // the reference's deposit of the current positions (Rust-CUDA/src/main.rs:1729-1739)
    CUDAPIC_CHECK(check_cuda(cudaMemsetAsync(s->e_density(), 0, nb, st), "memset e_density"));
    CUDAPIC_CHECK(cudapic_get_density(s->x[E][s->side[E]], s->e_density(), s->n_e(), &g, (cudapic_stream_t)st));
    // the published-count kernels expect their slot counters and ticket at zero
    CUDAPIC_CHECK(check_cuda(cudaMemsetAsync(s->alive(), 0, sizeof(uint32_t), st), "memset alive"));
    CUDAPIC_CHECK(check_cuda(cudaMemsetAsync(s->alive_i(), 0, 2 * sizeof(uint32_t), st), "memset alive_i"));
    // both ion buffers hold the density of the present ions
    CUDAPIC_CHECK(check_cuda(cudaMemsetAsync(s->i_dens[s->i_cur], 0, nb, st), "memset i_density"));
    CUDAPIC_CHECK(cudapic_get_density(s->x[I][s->side[I]], s->i_dens[s->i_cur], s->n_i(), &g, (cudapic_stream_t)st));
    CUDAPIC_CHECK(check_cuda(cudaMemcpyAsync(s->i_dens[s->i_cur ^ 1], s->i_dens[s->i_cur], nb,
                                             cudaMemcpyDeviceToDevice, st), "copy i_density"));
    s->dens_valid = true;
    return CUDAPIC_OK;
}

bool state_is_ion_step(const cudapic_state *s, uint64_t step) {
    return ((step % s->params.n_t) % s->params.n_sub) == 0;
}

int state_alloc(cudapic_state *s, void **p, size_t bytes) {
    void *ptr = nullptr;
    const cudaError_t e = cudaMalloc(&ptr, std::max<size_t>(bytes, 256));
    if (e != cudaSuccess) return check_cuda(e, "cudaMalloc");
    s->allocations.push_back(ptr);
    *p = ptr;
    return CUDAPIC_OK;
}

void state_release(cudapic_state *s, void *p) {
    auto it = std::find(s->allocations.begin(), s->allocations.end(), p);
    if (it == s->allocations.end()) return;
    s->allocations.erase(it);
    cudaFree(p);
}

void state_drop_graphs(cudapic_state *s) {
    for (auto &g : s->graph) {
        if (g) cudaGraphExecDestroy(g);
        g = nullptr;
    }
}

}  // namespace cudapic

namespace {

template <typename T>
int dalloc(cudapic_state *s, T **p, size_t count) {
    void *ptr = nullptr;
    size_t bytes = std::max<size_t>(count * sizeof(T), 256);
    cudaError_t e = cudaMalloc(&ptr, bytes);
    if (e != cudaSuccess) return check_cuda(e, "cudaMalloc");
    s->allocations.push_back(ptr);
    *p = static_cast<T *>(ptr);
    return CUDAPIC_OK;
}

void destroy_graphs(cudapic_state *s) {
    for (auto &g : s->graph) {
        if (g) cudaGraphExecDestroy(g);
        g = nullptr;
    }
}

// Particle part of a fused-mode step: [ion push] -> electron step ->
// [ion collisions] -> [measurement]; the kernels publish the particle counts
// themselves (StepLink), so the step holds no copy or memset node.  The
// electron step is the compacting fused kernel (kernels_step.cu) when
// `compact` or when the in-place step is off, else the in-place stream and
// scatter passes (kernels_inplace.cu: electrons stay in their slots,
// absorbed ones are marked dead, colliders recorded in the other side's
// planes and scattered by the second kernel).  Either way an
// electron draws from the RNG stream of the slot it occupies when the step
// starts.  Returns CUDAPIC_ERR_NOT_SUPPORTED, having
// enqueued nothing, when the electron planes are not aligned for the fused
// kernels.
int enqueue_fused_particles(cudapic_state *s, bool ion_step, float *e_next, float *i_acc, bool compact,
                            int next_ion) {
    const cudapic_grid &g = s->grid;
    cudaStream_t st = s->stream;
    const int E = 0, I = 1;
    int se = s->side[E], si = s->side[I];
    const void *planes[8] = {s->x[E][se], s->vx[E][se], s->vy[E][se], s->vz[E][se],
                             s->rng[E][0], s->rng[E][1], s->rng[E][2], s->rng[E][3]};
    if (!electron_step_eligible(planes, 8, g.capacity)) return CUDAPIC_ERR_NOT_SUPPORTED;
    if (ion_step) {
        StepLink li;
        li.ticket = s->ticket();
        li.dst = s->n_i();
        li.src = s->alive_i();
        li.clear_src = 1;
        CUDAPIC_CHECK(launch_move_and_compact(s->efield, s->x[I][si], s->vx[I][si], s->vy[I][si], s->vz[I][si],
                                              s->x[I][si ^ 1], s->vx[I][si ^ 1], s->vy[I][si ^ 1],
                                              s->vz[I][si ^ 1], s->alive_i(), s->n_i(), g.factor_i, g.dt_i, g, st,
                                              i_acc, li, s->measure ? s->wall + 1 : nullptr, true));
        si ^= 1;
        s->side[I] = si;
    }
    if (s->inplace && !compact) {
        const InplacePlanes pl{s->x[E][se], s->vx[E][se], s->vy[E][se], s->vz[E][se],
                               s->rng[E][0], s->rng[E][1], s->rng[E][2], s->rng[E][3],
                               s->x[I][si], s->vx[I][si], s->vy[I][si], s->vz[I][si]};
        // the collider records live in the other sides' planes (free until the
        // next compaction and ion push)
        const CollList list{reinterpret_cast<uint32_t *>(s->x[E][se ^ 1]), s->vx[E][se ^ 1], s->vy[E][se ^ 1],
                            s->vz[E][se ^ 1], reinterpret_cast<uint32_t *>(s->x[I][si ^ 1]),
                            reinterpret_cast<uint32_t *>(s->vx[I][si ^ 1]),
                            reinterpret_cast<uint32_t *>(s->vy[I][si ^ 1]),
                            reinterpret_cast<uint32_t *>(s->vz[I][si ^ 1])};
        CUDAPIC_CHECK(launch_electron_inplace(pl, s->efield, s->sigma_tot_e, s->cs, s->sigma_max_e, s->n_e(), list,
                                              s->counters + CTR_COLL_COUNT, e_next, g, st,
                                              s->measure ? s->wall : nullptr, s->counters + CTR_SPAWN_FROM));
        // the next step's solve in the scatter pass: only when nothing that
        // reads this step's field or adds to the densities follows it
        // (measurement, the spawn-collision pass) and a next step exists
        const bool ahead = next_ion >= 0 && s->solve_ahead && !s->measure && !s->spawn_collide &&
                           g.n_g <= POISSON_AHEAD_MAX_NG;
        PoissonAhead pa{};
        if (ahead) {
            // the buffer roles enqueue_step gives the next step: e_next becomes
            // current, the buffer read now collects; on an ion step the ion
            // collector becomes current and the current one collects
            pa.e_density = e_next;
            pa.zero_a = s->e_dens[s->e_cur];
            pa.i_density = next_ion ? s->i_dens[s->i_cur ^ 1] : s->i_dens[s->i_cur];
            pa.zero_b = next_ion ? s->i_dens[s->i_cur] : nullptr;
            pa.pot = s->pot;
            pa.efield = s->efield;
            pa.pot0_table = s->pot0_table;
            pa.step_counter = s->step_counter();
        }
        CUDAPIC_CHECK(launch_electron_scatter(pl, list, s->cs, s->counters + CTR_COLL_COUNT,
                                              s->counters + CTR_COLL_TICKET, s->n_e(), s->n_i(), g, st, e_next, i_acc,
                                              s->measure ? s->mcount : nullptr, ahead ? &pa : nullptr));
        s->poisson_ahead = ahead;
        if (s->spawn_collide)
            CUDAPIC_CHECK(launch_spawn_collide(pl, s->sigma_tot_e, s->cs, s->counters + CTR_SPAWN_FROM, s->n_e(),
                                               s->n_i(), g, st, e_next, i_acc, s->measure ? s->mcount : nullptr));
    } else {
        StepLink le;
        le.ticket = s->ticket();
        le.dst = s->n_e();
        le.src = s->alive();
        le.clear_src = 1;
        CUDAPIC_CHECK(launch_electron_step(s->efield, s->x[E][se], s->vx[E][se], s->vy[E][se], s->vz[E][se],
                                           s->x[E][se ^ 1], s->vx[E][se ^ 1], s->vy[E][se ^ 1], s->vz[E][se ^ 1],
                                           s->rng[E][0], s->rng[E][1], s->rng[E][2], s->rng[E][3], s->sigma_tot_e,
                                           s->cs, s->sigma_max_e, s->x[I][si], s->vx[I][si], s->vy[I][si],
                                           s->vz[I][si], s->alive(), s->n_e(), s->n_i(), e_next, i_acc, g, st, le,
                                           s->measure ? s->wall : nullptr, s->measure ? s->mcount : nullptr));
        se ^= 1;
        s->side[E] = se;
    }
    s->e_cur ^= 1;
    if (ion_step) {
        CUDAPIC_CHECK(launch_collisions_i(s->sigma_tot_i, s->cs, s->n_i(), s->vx[I][si], s->vy[I][si],
                                          s->vz[I][si], s->rng[I][0], s->rng[I][1], s->rng[I][2], s->rng[I][3],
                                          nullptr, g, st, s->measure ? s->mcount + 1 : nullptr, s->ion_k));
    }
    if (s->measure) {
        CUDAPIC_CHECK(launch_eepf(s->x[E][se], s->vx[E][se], s->vy[E][se], s->vz[E][se], s->efield, s->n_e(),
                                  s->eepf, g, st, s->esum, s->mcount + 2));
    }
    return CUDAPIC_OK;
}

// One reference time step (Rust-CUDA/src/main.rs:1728-1807).  compact: a
// fused-mode step that closes the holes of earlier in-place steps.
// next_ion: whether the step after this one is an ion step (1 / 0), or -1
// when this is the last step of a run or graph (no solve ahead).
int enqueue_step(cudapic_state *s, bool ion_step, bool compact, int next_ion) {
    PdlScope pdl(s->overlap);
    const cudapic_grid &g = s->grid;
    cudaStream_t st = s->stream;
    const int E = 0, I = 1;
    const uint32_t n_g = g.n_g;
    const size_t nb = n_g * sizeof(float);
    int se = s->side[E], si = s->side[I];
    const bool fused = s->fused;
    float *e_next = nullptr, *i_acc = nullptr, *zero_b = nullptr;

    if (fused && !s->dens_valid) {
        CUDAPIC_CHECK(state_prime_fused(s, st));
    } else if (!fused) {
        // the reference's deposit of the current positions (Rust-CUDA/src/main.rs:1729-1739)
        CUDAPIC_CHECK(check_cuda(cudaMemsetAsync(s->e_density(), 0, nb, st), "memset e_density"));
        CUDAPIC_CHECK(cudapic_get_density(s->x[E][se], s->e_density(), s->n_e(), &g, (cudapic_stream_t)st));
        if (ion_step) {
            CUDAPIC_CHECK(check_cuda(cudaMemsetAsync(s->i_density(), 0, nb, st), "memset i_density"));
            CUDAPIC_CHECK(cudapic_get_density(s->x[I][si], s->i_density(), s->n_i(), &g, (cudapic_stream_t)st));
        }
    }
    if (fused) {
        // e_dens[e_cur] holds the density of the present electrons; the other
        // buffer collects the next step's.  On an ion step the ion buffer
        // that collected the period's deposits becomes current and the other
        // one starts collecting.  The Poisson kernel clears the collectors.
        e_next = s->e_dens[s->e_cur ^ 1];
        if (ion_step) {
            s->i_cur ^= 1;
            zero_b = s->i_dens[s->i_cur ^ 1];
        }
        i_acc = s->i_dens[s->i_cur ^ 1];
    }
    if (!s->poisson_ahead)  // else the previous step's scatter pass solved it, and cleared the collectors
        CUDAPIC_CHECK(launch_poisson(s->e_density(), s->i_density(), s->pot, s->efield, 0.0f, s->pot0_table,
                                     s->step_counter(), g, st, e_next, zero_b));
    s->poisson_ahead = false;
    if (s->measure) {
        CUDAPIC_CHECK(cudapic_accumulate_density(s->e_density(), s->cumul_e, &g, (cudapic_stream_t)st));
        if (ion_step) CUDAPIC_CHECK(cudapic_accumulate_density(s->i_density(), s->cumul_i, &g, (cudapic_stream_t)st));
        if (s->xt) {  // XT diagnostics: the grid of this step and the particles before their push
            CUDAPIC_CHECK(launch_xt_grid(s->pot, s->efield, s->e_density(), s->i_density(), s->step_counter(), g,
                                         s->n_xt, s->xt, st));
            CUDAPIC_CHECK(launch_xt_particles(false, s->x[E][se], s->vx[E][se], s->vy[E][se], s->vz[E][se], s->n_e(),
                                              s->efield, s->cs, s->step_counter(), g, s->n_xt, s->xt, st));
            if (ion_step)
                CUDAPIC_CHECK(launch_xt_particles(true, s->x[I][si], s->vx[I][si], s->vy[I][si], s->vz[I][si],
                                                  s->n_i(), s->efield, s->cs, s->step_counter(), g, s->n_xt, s->xt,
                                                  st));
        }
    }
    if (fused) {
        const int rc = enqueue_fused_particles(s, ion_step, e_next, i_acc, compact, next_ion);
        if (rc != CUDAPIC_ERR_NOT_SUPPORTED) return rc;  // else: buffers not aligned for the fused kernel
    }
    // electrons: push + compact into the other side
    CUDAPIC_CHECK(check_cuda(cudaMemsetAsync(s->alive(), 0, sizeof(uint32_t), st), "memset alive"));
    CUDAPIC_CHECK(launch_move_and_compact(s->efield, s->x[E][se], s->vx[E][se], s->vy[E][se], s->vz[E][se],
                                          s->x[E][se ^ 1], s->vx[E][se ^ 1], s->vy[E][se ^ 1], s->vz[E][se ^ 1],
                                          s->alive(), s->n_e(), g.factor_e, g.dt_e, g, st, e_next, StepLink(),
                                          s->measure ? s->wall : nullptr, false));
    se ^= 1;
    s->side[E] = se;
    CUDAPIC_CHECK(check_cuda(cudaMemcpyAsync(s->n_e(), s->alive(), sizeof(uint32_t), cudaMemcpyDeviceToDevice, st),
                             "copy alive -> n_e"));
    if (ion_step) {
        CUDAPIC_CHECK(check_cuda(cudaMemsetAsync(s->alive(), 0, sizeof(uint32_t), st), "memset alive"));
        CUDAPIC_CHECK(launch_move_and_compact(s->efield, s->x[I][si], s->vx[I][si], s->vy[I][si], s->vz[I][si],
                                              s->x[I][si ^ 1], s->vx[I][si ^ 1], s->vy[I][si ^ 1],
                                              s->vz[I][si ^ 1], s->alive(), s->n_i(), g.factor_i, g.dt_i, g, st,
                                              i_acc, StepLink(), s->measure ? s->wall + 1 : nullptr, true));
        si ^= 1;
        s->side[I] = si;
        CUDAPIC_CHECK(check_cuda(
            cudaMemcpyAsync(s->n_i(), s->alive(), sizeof(uint32_t), cudaMemcpyDeviceToDevice, st), "copy alive -> n_i"));
        CUDAPIC_CHECK(check_cuda(
            cudaMemcpyAsync(s->alive(), s->n_e(), sizeof(uint32_t), cudaMemcpyDeviceToDevice, st), "copy n_e -> alive"));
    }
    CUDAPIC_CHECK(launch_collisions_e(s->sigma_tot_e, s->cs, s->n_e(), s->x[E][se], s->vx[E][se], s->vy[E][se],
                                      s->vz[E][se], s->rng[E][0], s->rng[E][1], s->rng[E][2], s->rng[E][3],
                                      s->x[I][si], s->vx[I][si], s->vy[I][si], s->vz[I][si], s->alive(), s->n_i(),
                                      nullptr, g, st, e_next, i_acc, s->measure ? s->mcount : nullptr));
    CUDAPIC_CHECK(check_cuda(cudaMemcpyAsync(s->n_e(), s->alive(), sizeof(uint32_t), cudaMemcpyDeviceToDevice, st),
                             "copy alive -> n_e"));
    if (fused) s->e_cur ^= 1;
    if (ion_step) {
        CUDAPIC_CHECK(launch_collisions_i(s->sigma_tot_i, s->cs, s->n_i(), s->vx[I][si], s->vy[I][si],
                                          s->vz[I][si], s->rng[I][0], s->rng[I][1], s->rng[I][2], s->rng[I][3],
                                          nullptr, g, st, s->measure ? s->mcount + 1 : nullptr));
    }
    if (s->measure) {
        CUDAPIC_CHECK(launch_eepf(s->x[E][se], s->vx[E][se], s->vy[E][se], s->vz[E][se], s->efield, s->n_e(),
                                  s->eepf, g, st, s->esum, s->mcount + 2));
    }
    return CUDAPIC_OK;
}

bool is_ion_step(const cudapic_state *s, uint64_t step) { return state_is_ion_step(s, step); }

// In-place mode: the electron planes are compacted by the step before every
// N_SUB-th step (the last step of each half of a graph period) and by the
// last step of every run, so they are compact whenever a caller sees them.
bool is_compact_step(const cudapic_state *s, uint64_t step) { return ((step + 1) % s->params.n_sub) == 0; }

// Graph period: 2 * N_SUB steps returns both species to their starting
// side; requires N_T % N_SUB == 0 so that the ion-step pattern repeats.
uint64_t graph_period(const cudapic_state *s) { return 2ull * s->params.n_sub; }

int build_graph(cudapic_state *s) {
    const int m = s->measure ? 1 : 0;
    if (s->graph[m]) return CUDAPIC_OK;
    cudaGraph_t graph = nullptr;
    const uint64_t period = graph_period(s);
    const int side0[2] = {s->side[0], s->side[1]};
    const int cur0[2] = {s->e_cur, s->i_cur};
    CUDAPIC_CHECK(check_cuda(cudaStreamBeginCapture(s->stream, cudaStreamCaptureModeThreadLocal), "begin capture"));
    int rc = CUDAPIC_OK;
    for (uint64_t k = 0; k < period && rc == CUDAPIC_OK; ++k)
        rc = enqueue_step(s, is_ion_step(s, s->steps_done + k),
                          is_compact_step(s, s->steps_done + k) || k + 1 == period,
                          k + 1 == period ? -1 : (int)is_ion_step(s, s->steps_done + k + 1));
    cudaError_t e = cudaStreamEndCapture(s->stream, &graph);
    // a graph of 2 N_SUB steps returns every ping-pong role to its start
    s->poisson_ahead = false;  // the last captured step solved nothing ahead (a failed capture may have)
    s->side[0] = side0[0];
    s->side[1] = side0[1];
    s->e_cur = cur0[0];
    s->i_cur = cur0[1];
    s->graph_key[m][0] = side0[0];
    s->graph_key[m][1] = side0[1];
    s->graph_key[m][2] = cur0[0];
    s->graph_key[m][3] = cur0[1];
    if (rc != CUDAPIC_OK) {
        if (graph) cudaGraphDestroy(graph);
        return rc;
    }
    CUDAPIC_CHECK(check_cuda(e, "end capture"));
    e = cudaGraphInstantiate(&s->graph[m], graph, 0);
    cudaGraphDestroy(graph);
    s->graph_gen[m] = tuning_generation();
    return check_cuda(e, "cudaGraphInstantiate");
}

}  // namespace

extern "C" int cudapic_state_create(const cudapic_params *p, int device, cudapic_state **out) {
    if (!p || !out) return fail(CUDAPIC_ERR_ARG, "state_create: null pointer");
    *out = nullptr;
    cudapic_grid grid;
    CUDAPIC_CHECK(cudapic_grid_from_params(p, &grid));
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0)
        return fail(CUDAPIC_ERR_NOT_SUPPORTED, "state_create: no CUDA device");
    if (device < 0 || device >= ndev) return fail(CUDAPIC_ERR_ARG, "state_create: bad device index");
    DeviceGuard dg(device);
    cudaDeviceProp prop;
    CUDAPIC_CHECK(check_cuda(cudaGetDeviceProperties(&prop, device), "cudaGetDeviceProperties"));
    if (prop.major < 10)
        return fail(CUDAPIC_ERR_NOT_SUPPORTED, "state_create: libcudapic is built for sm_100a (B200)");

    cudapic_state *s = new (std::nothrow) cudapic_state();
    if (!s) return fail(CUDAPIC_ERR_ARG, "state_create: out of host memory");
    s->device = device;
    s->params = *p;
    // capacity rounded up to a multiple of 4 for the bulk-copy push path
    s->params.capacity = (p->capacity + 3u) & ~3u;
    s->grid = grid;
    s->grid.capacity = s->params.capacity;
    s->graphs_enabled = (p->n_t % p->n_sub) == 0;

    auto cleanup = [&](int rc) {
        cudapic_state_destroy(s);
        return rc;
    };
    int rc;
    if ((rc = check_cuda(cudaStreamCreateWithFlags(&s->stream, cudaStreamNonBlocking), "cudaStreamCreate")) !=
        CUDAPIC_OK)
        return cleanup(rc);
    s->own_stream = true;
    const size_t cap = s->params.capacity;
    for (int sp = 0; sp < 2; ++sp) {
        for (int side = 0; side < 2; ++side) {
            if ((rc = dalloc(s, &s->x[sp][side], cap)) || (rc = dalloc(s, &s->vx[sp][side], cap)) ||
                (rc = dalloc(s, &s->vy[sp][side], cap)) || (rc = dalloc(s, &s->vz[sp][side], cap)))
                return cleanup(rc);
        }
        for (int k = 0; k < 4; ++k)
            if ((rc = dalloc(s, &s->rng[sp][k], cap))) return cleanup(rc);
    }
    const size_t n_g = p->n_g;
    if ((rc = dalloc(s, &s->counters, 64)) || (rc = dalloc(s, &s->efield, n_g)) || (rc = dalloc(s, &s->pot, n_g)) ||
        (rc = dalloc(s, &s->e_dens[0], n_g)) || (rc = dalloc(s, &s->e_dens[1], n_g)) ||
        (rc = dalloc(s, &s->i_dens[0], n_g)) || (rc = dalloc(s, &s->i_dens[1], n_g)) ||
        (rc = dalloc(s, &s->pot0_table, p->n_t)) || (rc = dalloc(s, &s->cs, 5ull * CUDAPIC_CS_RANGES)) ||
        (rc = dalloc(s, &s->sigma_tot_e, CUDAPIC_CS_RANGES)) || (rc = dalloc(s, &s->sigma_tot_i, CUDAPIC_CS_RANGES)) ||
        (rc = dalloc(s, &s->cumul_e, n_g)) || (rc = dalloc(s, &s->cumul_i, n_g)) || (rc = dalloc(s, &s->eepf, 2000)) ||
        (rc = dalloc(s, &s->wall, 2)) || (rc = dalloc(s, &s->mcount, 3)) || (rc = dalloc(s, &s->esum, 1)))
        return cleanup(rc);
    s->grid.dev_err = s->dev_err();
    s->grid.work = s->work();

    // zero everything that is read before written
    for (int sp = 0; sp < 2; ++sp)
        for (int side = 0; side < 2; ++side)
            for (float *b : {s->x[sp][side], s->vx[sp][side], s->vy[sp][side], s->vz[sp][side]})
                if ((rc = check_cuda(cudaMemsetAsync(b, 0, cap * sizeof(float), s->stream), "memset")))
                    return cleanup(rc);
    if ((rc = check_cuda(cudaMemsetAsync(s->counters, 0, 64 * sizeof(uint32_t), s->stream), "memset")) ||
        (rc = check_cuda(cudaMemsetAsync(s->efield, 0, n_g * sizeof(float), s->stream), "memset")) ||
        (rc = check_cuda(cudaMemsetAsync(s->pot, 0, n_g * sizeof(float), s->stream), "memset")) ||
        (rc = check_cuda(cudaMemsetAsync(s->e_dens[0], 0, n_g * sizeof(float), s->stream), "memset")) ||
        (rc = check_cuda(cudaMemsetAsync(s->e_dens[1], 0, n_g * sizeof(float), s->stream), "memset")) ||
        (rc = check_cuda(cudaMemsetAsync(s->i_dens[0], 0, n_g * sizeof(float), s->stream), "memset")) ||
        (rc = check_cuda(cudaMemsetAsync(s->i_dens[1], 0, n_g * sizeof(float), s->stream), "memset")) ||
        (rc = check_cuda(cudaMemsetAsync(s->cumul_e, 0, n_g * sizeof(double), s->stream), "memset")) ||
        (rc = check_cuda(cudaMemsetAsync(s->wall, 0, 2 * sizeof(cudapic_wall_counters), s->stream), "memset")) ||
        (rc = check_cuda(cudaMemsetAsync(s->mcount, 0, 3 * sizeof(unsigned long long), s->stream), "memset")) ||
        (rc = check_cuda(cudaMemsetAsync(s->esum, 0, sizeof(double), s->stream), "memset")) ||
        (rc = check_cuda(cudaMemsetAsync(s->cumul_i, 0, n_g * sizeof(double), s->stream), "memset")) ||
        (rc = check_cuda(cudaMemsetAsync(s->eepf, 0, 2000 * sizeof(uint32_t), s->stream), "memset")))
        return cleanup(rc);

    // RF boundary table: (V cos(2 pi t / N_T)) as f32, Rust-CUDA/src/main.rs:1741
    std::vector<float> table(p->n_t);
    for (uint32_t t = 0; t < p->n_t; ++t)
        table[t] = (float)(p->voltage * std::cos(((double)t / (double)p->n_t) * (2.0 * 3.141592653589793)));
    // cross sections (host, all threads), Rust-CUDA/src/main.rs:1649, 1378-1444
    std::vector<float> cs(5ull * CUDAPIC_CS_RANGES), se(CUDAPIC_CS_RANGES), si(CUDAPIC_CS_RANGES);
    if ((rc = cudapic_cross_sections(grid.gas_density, cs.data(), se.data(), si.data()))) return cleanup(rc);
    s->sigma_max_e = *std::max_element(se.begin(), se.end());
    s->ion_k = ion_reject_k(*std::max_element(si.begin(), si.end()), s->grid);
    table_coll_freqs(se.data(), si.data(), &s->max_e_coll_freq, &s->max_i_coll_freq);
    if ((rc = check_cuda(cudaMemcpyAsync(s->pot0_table, table.data(), table.size() * sizeof(float),
                                         cudaMemcpyHostToDevice, s->stream), "upload pot0 table")) ||
        (rc = check_cuda(cudaMemcpyAsync(s->cs, cs.data(), cs.size() * sizeof(float), cudaMemcpyHostToDevice, s->stream),
                         "upload cs")) ||
        (rc = check_cuda(cudaMemcpyAsync(s->sigma_tot_e, se.data(), se.size() * sizeof(float), cudaMemcpyHostToDevice,
                                         s->stream), "upload sigma_tot_e")) ||
        (rc = check_cuda(cudaMemcpyAsync(s->sigma_tot_i, si.data(), si.size() * sizeof(float), cudaMemcpyHostToDevice,
                                         s->stream), "upload sigma_tot_i")) ||
        (rc = check_cuda(cudaStreamSynchronize(s->stream), "state_create sync")))
        return cleanup(rc);
    *out = s;
    return CUDAPIC_OK;
}

extern "C" int cudapic_state_destroy(cudapic_state *s) {
    if (!s) return CUDAPIC_OK;
    DeviceGuard dg(s->device);
    if (s->stream) cudaStreamSynchronize(s->stream);
    destroy_graphs(s);
    for (void *p : s->allocations) cudaFree(p);
    if (s->own_stream && s->stream) cudaStreamDestroy(s->stream);
    delete s;
    return CUDAPIC_OK;
}

extern "C" int cudapic_state_set_stream(cudapic_state *s, cudapic_stream_t stream) {
    if (!s) return fail(CUDAPIC_ERR_ARG, "state_set_stream: null state");
    DeviceGuard dg(s->device);
    CUDAPIC_CHECK(check_cuda(cudaStreamSynchronize(s->stream), "state_set_stream sync"));
    if (s->own_stream) cudaStreamDestroy(s->stream);
    s->own_stream = false;
    s->stream = (cudaStream_t)stream;
    destroy_graphs(s);
    return CUDAPIC_OK;
}

extern "C" cudapic_stream_t cudapic_state_stream(const cudapic_state *s) {
    return s ? (cudapic_stream_t)s->stream : nullptr;
}

extern "C" int cudapic_state_grid(const cudapic_state *s, cudapic_grid *out) {
    if (!s || !out) return fail(CUDAPIC_ERR_ARG, "state_grid: null pointer");
    *out = s->grid;
    return CUDAPIC_OK;
}

extern "C" int cudapic_state_buffers(const cudapic_state *s, cudapic_buffers *o) {
    if (!s || !o) return fail(CUDAPIC_ERR_ARG, "state_buffers: null pointer");
    std::memset(o, 0, sizeof(*o));
    for (int sp = 0; sp < 2; ++sp) {
        const int a = s->side[sp], b = a ^ 1;
        o->x[sp] = s->x[sp][a];
        o->vx[sp] = s->vx[sp][a];
        o->vy[sp] = s->vy[sp][a];
        o->vz[sp] = s->vz[sp][a];
        o->tmp_x[sp] = s->x[sp][b];
        o->tmp_vx[sp] = s->vx[sp][b];
        o->tmp_vy[sp] = s->vy[sp][b];
        o->tmp_vz[sp] = s->vz[sp][b];
        for (int k = 0; k < 4; ++k) o->rng[sp][k] = s->rng[sp][k];
    }
    o->sigma_max_e = s->sigma_max_e;
    o->n_electrons = s->n_e();
    o->n_ions = s->n_i();
    o->alive_counter = s->alive();
    o->efield = s->efield;
    o->pot = s->pot;
    o->e_density = s->e_density();
    o->i_density = s->i_density();
    o->cs = s->cs;
    o->sigma_tot_e = s->sigma_tot_e;
    o->sigma_tot_i = s->sigma_tot_i;
    o->cumul_e_density = s->cumul_e;
    o->cumul_i_density = s->cumul_i;
    o->eepf = s->eepf;
    o->dev_err = s->dev_err();
    o->work = s->work();
    return CUDAPIC_OK;
}

extern "C" int cudapic_state_upload(cudapic_state *s, int species, const float *x, const float *vx, const float *vy,
                                    const float *vz, uint32_t n) {
    if (!s || (species != 0 && species != 1)) return fail(CUDAPIC_ERR_ARG, "state_upload: bad state/species");
    if (n > s->params.capacity) return fail(CUDAPIC_ERR_CAPACITY, "state_upload: n exceeds capacity");
    if (n && (!x || !vx || !vy || !vz)) return fail(CUDAPIC_ERR_ARG, "state_upload: null pointer");
    DeviceGuard dg(s->device);
    const int a = s->side[species];
    const size_t bytes = (size_t)n * sizeof(float);
    s->dens_valid = false;  // the next step recomputes the densities from the particles
    if (n) {
        CUDAPIC_CHECK(check_cuda(cudaMemcpyAsync(s->x[species][a], x, bytes, cudaMemcpyHostToDevice, s->stream), "upload x"));
        CUDAPIC_CHECK(check_cuda(cudaMemcpyAsync(s->vx[species][a], vx, bytes, cudaMemcpyHostToDevice, s->stream), "upload vx"));
        CUDAPIC_CHECK(check_cuda(cudaMemcpyAsync(s->vy[species][a], vy, bytes, cudaMemcpyHostToDevice, s->stream), "upload vy"));
        CUDAPIC_CHECK(check_cuda(cudaMemcpyAsync(s->vz[species][a], vz, bytes, cudaMemcpyHostToDevice, s->stream), "upload vz"));
    }
    uint32_t *cnt = species == 0 ? s->n_e() : s->n_i();
    const uint32_t count = n;
    CUDAPIC_CHECK(check_cuda(cudaMemcpyAsync(cnt, &count, sizeof(uint32_t), cudaMemcpyHostToDevice, s->stream),
                             "upload count"));
    return check_cuda(cudaStreamSynchronize(s->stream), "upload sync");
}

extern "C" int cudapic_state_download(cudapic_state *s, int species, float *x, float *vx, float *vy, float *vz,
                                      uint32_t max_n, uint32_t *n_out) {
    if (!s || (species != 0 && species != 1)) return fail(CUDAPIC_ERR_ARG, "state_download: bad state/species");
    DeviceGuard dg(s->device);
    uint32_t n = 0;
    uint32_t *cnt = species == 0 ? s->n_e() : s->n_i();
    CUDAPIC_CHECK(check_cuda(cudaMemcpyAsync(&n, cnt, sizeof(uint32_t), cudaMemcpyDeviceToHost, s->stream), "read count"));
    CUDAPIC_CHECK(check_cuda(cudaStreamSynchronize(s->stream), "download sync"));
    n = std::min(n, s->params.capacity);
    if (n_out) *n_out = n;
    const uint32_t m = std::min(n, max_n);
    const int a = s->side[species];
    const size_t bytes = (size_t)m * sizeof(float);
    if (m) {
        if (!x || !vx || !vy || !vz) return fail(CUDAPIC_ERR_ARG, "state_download: null pointer");
        CUDAPIC_CHECK(check_cuda(cudaMemcpyAsync(x, s->x[species][a], bytes, cudaMemcpyDeviceToHost, s->stream), "download x"));
        CUDAPIC_CHECK(check_cuda(cudaMemcpyAsync(vx, s->vx[species][a], bytes, cudaMemcpyDeviceToHost, s->stream), "download vx"));
        CUDAPIC_CHECK(check_cuda(cudaMemcpyAsync(vy, s->vy[species][a], bytes, cudaMemcpyDeviceToHost, s->stream), "download vy"));
        CUDAPIC_CHECK(check_cuda(cudaMemcpyAsync(vz, s->vz[species][a], bytes, cudaMemcpyDeviceToHost, s->stream), "download vz"));
    }
    return check_cuda(cudaStreamSynchronize(s->stream), "download sync");
}

extern "C" int cudapic_state_seed(cudapic_state *s, const uint32_t e_master[4], const uint32_t i_master[4]) {
    if (!s || !e_master || !i_master) return fail(CUDAPIC_ERR_ARG, "state_seed: null pointer");
    DeviceGuard dg(s->device);
    CUDAPIC_CHECK(cudapic_xoshiro128_seed_streams(e_master, s->params.capacity, s->rng[0][0], s->rng[0][1],
                                                  s->rng[0][2], s->rng[0][3], (cudapic_stream_t)s->stream));
    CUDAPIC_CHECK(cudapic_xoshiro128_seed_streams(i_master, s->params.capacity, s->rng[1][0], s->rng[1][1],
                                                  s->rng[1][2], s->rng[1][3], (cudapic_stream_t)s->stream));
    return CUDAPIC_OK;
}

// eduPIC's time step DT_E = 1 / (f N_T) in double (C/eduPIC.cc:65-69).
static double dt_e_double(const cudapic_state *s) {
    return 1.0 / (s->params.frequency * (double)s->params.n_t);
}

extern "C" int cudapic_state_save(cudapic_state *s, const char *path) {
    if (!s || !path) return fail(CUDAPIC_ERR_ARG, "state_save: null pointer");
    DeviceGuard dg(s->device);
    const uint32_t cap = s->params.capacity;
    std::vector<float> e[4], i[4];
    for (int a = 0; a < 4; ++a) {
        e[a].resize(cap);
        i[a].resize(cap);
    }
    uint32_t ne = 0, ni = 0;
    CUDAPIC_CHECK(cudapic_state_download(s, 0, e[0].data(), e[1].data(), e[2].data(), e[3].data(), cap, &ne));
    CUDAPIC_CHECK(cudapic_state_download(s, 1, i[0].data(), i[1].data(), i[2].data(), i[3].data(), cap, &ni));
    const float *ep[4] = {e[0].data(), e[1].data(), e[2].data(), e[3].data()};
    const float *ip[4] = {i[0].data(), i[1].data(), i[2].data(), i[3].data()};
    const double time = (double)s->steps_done * dt_e_double(s);  // eduPIC's Time
    CUDAPIC_CHECK(cudapic_picdata_write(path, time, (uint32_t)(s->steps_done / s->params.n_t), ep, ne, ip, ni));
    std::vector<uint32_t> planes[2][4];
    for (int sp = 0; sp < 2; ++sp)
        for (int k = 0; k < 4; ++k) {
            planes[sp][k].resize(cap);
            CUDAPIC_CHECK(check_cuda(cudaMemcpyAsync(planes[sp][k].data(), s->rng[sp][k], cap * sizeof(uint32_t),
                                                     cudaMemcpyDeviceToHost, s->stream), "state_save: download rng"));
        }
    CUDAPIC_CHECK(check_cuda(cudaStreamSynchronize(s->stream), "state_save sync"));
    return rng_sidecar_write(path, cap, planes);
}

extern "C" int cudapic_state_load(cudapic_state *s, const char *path) {
    if (!s || !path) return fail(CUDAPIC_ERR_ARG, "state_load: null pointer");
    DeviceGuard dg(s->device);
    double time = 0.0;
    uint32_t cycles = 0, ne = 0, ni = 0;
    CUDAPIC_CHECK(cudapic_picdata_read_header(path, &time, &cycles, &ne, &ni));
    const uint32_t cap = s->params.capacity;
    if (ne > cap || ni > cap) return fail(CUDAPIC_ERR_CAPACITY, "state_load: more particles than the capacity");
    std::vector<float> e[4], i[4];
    for (int a = 0; a < 4; ++a) {
        e[a].resize(std::max<uint32_t>(ne, 1));
        i[a].resize(std::max<uint32_t>(ni, 1));
    }
    float *ep[4] = {e[0].data(), e[1].data(), e[2].data(), e[3].data()};
    float *ip[4] = {i[0].data(), i[1].data(), i[2].data(), i[3].data()};
    CUDAPIC_CHECK(cudapic_picdata_read(path, ep, ne, ip, ni));
    CUDAPIC_CHECK(cudapic_state_upload(s, 0, ep[0], ep[1], ep[2], ep[3], ne));
    CUDAPIC_CHECK(cudapic_state_upload(s, 1, ip[0], ip[1], ip[2], ip[3], ni));
    // the step count (and with it the RF phase and the ion subcycle) from eduPIC's Time
    const double steps = time > 0.0 ? std::floor(time / dt_e_double(s) + 0.5) : 0.0;
    s->steps_done = (uint64_t)steps;
    const uint32_t counter = (uint32_t)(s->steps_done & 0xffffffffu);
    CUDAPIC_CHECK(check_cuda(cudaMemcpyAsync(s->step_counter(), &counter, sizeof(uint32_t), cudaMemcpyHostToDevice,
                                             s->stream), "state_load: step counter"));
    std::vector<uint32_t> planes[2][4];
    const int rc = rng_sidecar_read(path, cap, planes);
    if (rc == CUDAPIC_ERR_NOT_SUPPORTED) {  // an eduPIC file: fresh streams from the reference master seeds
        const uint32_t em[4] = {0x12345678u, 0x11112222u, 0x22223333u, 0x33334444u};
        const uint32_t im[4] = {0x44445555u, 0x55556666u, 0x66667777u, 0x77778888u};
        CUDAPIC_CHECK(cudapic_state_seed(s, em, im));
    } else {
        CUDAPIC_CHECK(rc);
        for (int sp = 0; sp < 2; ++sp)
            for (int k = 0; k < 4; ++k)
                CUDAPIC_CHECK(check_cuda(cudaMemcpyAsync(s->rng[sp][k], planes[sp][k].data(), cap * sizeof(uint32_t),
                                                         cudaMemcpyHostToDevice, s->stream), "state_load: rng"));
    }
    return check_cuda(cudaStreamSynchronize(s->stream), "state_load sync");
}

extern "C" int cudapic_state_set_overlap(cudapic_state *s, int on) {
    if (!s) return fail(CUDAPIC_ERR_ARG, "state_set_overlap: null state");
    DeviceGuard dg(s->device);
    CUDAPIC_CHECK(check_cuda(cudaStreamSynchronize(s->stream), "state_set_overlap sync"));
    s->overlap = on != 0;
    destroy_graphs(s);
    return CUDAPIC_OK;
}

extern "C" int cudapic_state_set_fused(cudapic_state *s, int on) {
    if (!s) return fail(CUDAPIC_ERR_ARG, "state_set_fused: null state");
    DeviceGuard dg(s->device);
    CUDAPIC_CHECK(check_cuda(cudaStreamSynchronize(s->stream), "state_set_fused sync"));
    s->fused = on != 0;
    s->dens_valid = false;
    destroy_graphs(s);
    return CUDAPIC_OK;
}

extern "C" int cudapic_state_set_inplace(cudapic_state *s, int on) {
    if (!s) return fail(CUDAPIC_ERR_ARG, "state_set_inplace: null state");
    DeviceGuard dg(s->device);
    CUDAPIC_CHECK(check_cuda(cudaStreamSynchronize(s->stream), "state_set_inplace sync"));
    s->inplace = on != 0;
    destroy_graphs(s);
    return CUDAPIC_OK;
}

extern "C" int cudapic_state_set_spawn_collide(cudapic_state *s, int on) {
    if (!s) return fail(CUDAPIC_ERR_ARG, "state_set_spawn_collide: null state");
    DeviceGuard dg(s->device);
    CUDAPIC_CHECK(check_cuda(cudaStreamSynchronize(s->stream), "state_set_spawn_collide sync"));
    s->spawn_collide = on != 0;
    destroy_graphs(s);
    return CUDAPIC_OK;
}

extern "C" int cudapic_state_set_solve_ahead(cudapic_state *s, int on) {
    if (!s) return fail(CUDAPIC_ERR_ARG, "state_set_solve_ahead: null state");
    DeviceGuard dg(s->device);
    CUDAPIC_CHECK(check_cuda(cudaStreamSynchronize(s->stream), "state_set_solve_ahead sync"));
    s->solve_ahead = on != 0;
    destroy_graphs(s);
    return CUDAPIC_OK;
}

extern "C" int cudapic_state_set_graphs(cudapic_state *s, int on) {
    if (!s) return fail(CUDAPIC_ERR_ARG, "state_set_graphs: null state");
    DeviceGuard dg(s->device);
    CUDAPIC_CHECK(check_cuda(cudaStreamSynchronize(s->stream), "state_set_graphs sync"));
    destroy_graphs(s);
    s->graphs_enabled = on != 0 && (s->params.n_t % s->params.n_sub) == 0;
    return CUDAPIC_OK;
}

extern "C" int cudapic_state_set_measure(cudapic_state *s, int on) {
    if (!s) return fail(CUDAPIC_ERR_ARG, "state_set_measure: null state");
    DeviceGuard dg(s->device);
    const size_t n_g = s->params.n_g;
    if (on && !s->xt && s->params.n_t % XT_BIN == 0) {
        const uint32_t n_xt = s->params.n_t / XT_BIN;
        void *p = nullptr;
        CUDAPIC_CHECK(state_alloc(s, &p, (size_t)XT_RAW * n_g * n_xt * sizeof(double)));
        s->xt = static_cast<double *>(p);
        s->n_xt = n_xt;
        destroy_graphs(s);
    }
    if (s->xt)
        CUDAPIC_CHECK(check_cuda(cudaMemsetAsync(s->xt, 0, (size_t)XT_RAW * n_g * s->n_xt * sizeof(double), s->stream),
                                 "zero xt"));
    CUDAPIC_CHECK(check_cuda(cudaMemsetAsync(s->cumul_e, 0, n_g * sizeof(double), s->stream), "zero cumul_e"));
    CUDAPIC_CHECK(check_cuda(cudaMemsetAsync(s->cumul_i, 0, n_g * sizeof(double), s->stream), "zero cumul_i"));
    CUDAPIC_CHECK(check_cuda(cudaMemsetAsync(s->eepf, 0, 2000 * sizeof(uint32_t), s->stream), "zero eepf"));
    CUDAPIC_CHECK(check_cuda(cudaMemsetAsync(s->wall, 0, 2 * sizeof(cudapic_wall_counters), s->stream), "zero wall"));
    CUDAPIC_CHECK(check_cuda(cudaMemsetAsync(s->mcount, 0, 3 * sizeof(unsigned long long), s->stream), "zero counts"));
    CUDAPIC_CHECK(check_cuda(cudaMemsetAsync(s->esum, 0, sizeof(double), s->stream), "zero esum"));
    s->measure_steps = 0;
    s->measure = on != 0;
    return CUDAPIC_OK;
}

extern "C" int cudapic_state_run_steps(cudapic_state *s, uint64_t n_steps) {
    if (!s) return fail(CUDAPIC_ERR_ARG, "state_run_steps: null state");
    DeviceGuard dg(s->device);
    const uint64_t period = graph_period(s);
    while (n_steps > 0) {
        const bool primed = !s->fused || s->dens_valid;  // a priming step is never captured
        if (s->graphs_enabled && primed && (s->steps_done % period) == 0 && n_steps >= period) {
            const int m = s->measure ? 1 : 0;
            const int key[4] = {s->side[0], s->side[1], s->e_cur, s->i_cur};
            if (s->graph[m] && (std::memcmp(key, s->graph_key[m], sizeof(key)) != 0 ||
                                s->graph_gen[m] != tuning_generation())) {
                cudaGraphExecDestroy(s->graph[m]);  // buffer roles or launch shapes differ from the captured ones
                s->graph[m] = nullptr;
            }
            int rc = build_graph(s);
            if (rc != CUDAPIC_OK) {
                s->graphs_enabled = false;  // fall back to direct launches
                continue;
            }
            CUDAPIC_CHECK(check_cuda(cudaGraphLaunch(s->graph[m], s->stream), "cudaGraphLaunch"));
            s->steps_done += period;
            if (s->measure) s->measure_steps += period;
            n_steps -= period;
            continue;
        }
        CUDAPIC_CHECK(enqueue_step(s, is_ion_step(s, s->steps_done),
                                   is_compact_step(s, s->steps_done) || n_steps == 1,
                                   n_steps == 1 ? -1 : (int)is_ion_step(s, s->steps_done + 1)));
        s->steps_done += 1;
        if (s->measure) s->measure_steps += 1;
        n_steps -= 1;
    }
    return CUDAPIC_OK;
}

extern "C" int cudapic_state_counts(cudapic_state *s, uint32_t *n_e, uint32_t *n_i) {
    if (!s) return fail(CUDAPIC_ERR_ARG, "state_counts: null state");
    DeviceGuard dg(s->device);
    uint32_t c[2];
    CUDAPIC_CHECK(check_cuda(cudaMemcpyAsync(c, s->counters, sizeof(c), cudaMemcpyDeviceToHost, s->stream), "read counts"));
    CUDAPIC_CHECK(check_cuda(cudaStreamSynchronize(s->stream), "counts sync"));
    if (n_e) *n_e = std::min(c[0], s->params.capacity);
    if (n_i) *n_i = std::min(c[1], s->params.capacity);
    return CUDAPIC_OK;
}

extern "C" int cudapic_state_device_error(cudapic_state *s, uint32_t *bits) {
    if (!s || !bits) return fail(CUDAPIC_ERR_ARG, "state_device_error: null pointer");
    DeviceGuard dg(s->device);
    CUDAPIC_CHECK(check_cuda(cudaMemcpyAsync(bits, s->dev_err(), sizeof(uint32_t), cudaMemcpyDeviceToHost, s->stream),
                             "read device error word"));
    CUDAPIC_CHECK(check_cuda(cudaStreamSynchronize(s->stream), "device error sync"));
    if (*bits & (CUDAPIC_DEVERR_SPAWN_E | CUDAPIC_DEVERR_SPAWN_I | CUDAPIC_DEVERR_ACTIVE))
        return fail(CUDAPIC_ERR_CAPACITY, "device reported a capacity overflow");
    if (*bits & CUDAPIC_DEVERR_TIMEOUT) return fail(CUDAPIC_ERR_TIMEOUT, "device reported a wait timeout");
    return CUDAPIC_OK;
}

extern "C" int cudapic_state_clear_device_error(cudapic_state *s) {
    if (!s) return fail(CUDAPIC_ERR_ARG, "state_clear_device_error: null state");
    DeviceGuard dg(s->device);
    return check_cuda(cudaMemsetAsync(s->dev_err(), 0, sizeof(uint32_t), s->stream), "clear device error word");
}

extern "C" int cudapic_state_debug_wait_timeout(cudapic_state *s, long long limit_cycles) {
    if (!s) return fail(CUDAPIC_ERR_ARG, "state_debug_wait_timeout: null state");
    CUDAPIC_REQUIRE(limit_cycles > 0 && limit_cycles <= MBAR_PROBE_MAX_CYCLES,
                    "state_debug_wait_timeout: limit_cycles must be in [1, 2^31]");
    DeviceGuard dg(s->device);
    return launch_wait_timeout_probe(s->dev_err(), limit_cycles, s->stream);
}

extern "C" int cudapic_state_work(cudapic_state *s, unsigned long long *particle_steps) {
    if (!s || !particle_steps) return fail(CUDAPIC_ERR_ARG, "state_work: null pointer");
    DeviceGuard dg(s->device);
    CUDAPIC_CHECK(check_cuda(cudaMemcpyAsync(particle_steps, s->work(), sizeof(unsigned long long),
                                             cudaMemcpyDeviceToHost, s->stream), "read work"));
    return check_cuda(cudaStreamSynchronize(s->stream), "work sync");
}

extern "C" int cudapic_state_steps_done(const cudapic_state *s, uint64_t *steps) {
    if (!s || !steps) return fail(CUDAPIC_ERR_ARG, "state_steps_done: null pointer");
    *steps = s->steps_done;
    return CUDAPIC_OK;
}

extern "C" int cudapic_state_synchronize(cudapic_state *s) {
    if (!s) return fail(CUDAPIC_ERR_ARG, "state_synchronize: null state");
    DeviceGuard dg(s->device);
    return check_cuda(cudaStreamSynchronize(s->stream), "state_synchronize");
}

extern "C" int cudapic_state_report(cudapic_state *s, cudapic_report *out) {
    if (!s || !out) return fail(CUDAPIC_ERR_ARG, "state_report: null pointer");
    DeviceGuard dg(s->device);
    const cudapic_params &p = s->params;
    const uint32_t n_g = p.n_g;
    std::vector<double> cumul(n_g);
    cudapic_wall_counters wall[2];
    unsigned long long mc[3];
    double esum = 0.0;
    uint32_t counts[2];
    CUDAPIC_CHECK(check_cuda(cudaMemcpyAsync(cumul.data(), s->cumul_e, n_g * sizeof(double), cudaMemcpyDeviceToHost,
                                             s->stream), "report: density"));
    CUDAPIC_CHECK(check_cuda(cudaMemcpyAsync(wall, s->wall, sizeof(wall), cudaMemcpyDeviceToHost, s->stream),
                             "report: wall"));
    CUDAPIC_CHECK(check_cuda(cudaMemcpyAsync(mc, s->mcount, sizeof(mc), cudaMemcpyDeviceToHost, s->stream),
                             "report: counts"));
    CUDAPIC_CHECK(check_cuda(cudaMemcpyAsync(&esum, s->esum, sizeof(double), cudaMemcpyDeviceToHost, s->stream),
                             "report: energy"));
    CUDAPIC_CHECK(check_cuda(cudaMemcpyAsync(counts, s->counters, sizeof(counts), cudaMemcpyDeviceToHost, s->stream),
                             "report: particle counts"));
    CUDAPIC_CHECK(check_cuda(cudaStreamSynchronize(s->stream), "report sync"));
    // eduPIC's formulas (C/eduPIC.cc:930-1008), with its constants
    const double e_charge = 1.60217662e-19, e_mass = 9.10938356e-31, eps0 = 8.85418781e-12;
    const double dt_e = dt_e_double(s), dt_i = dt_e * (double)p.n_sub;
    const double dx = p.gap / (double)(n_g - 1);
    const uint64_t steps = s->measure_steps;
    const double sim_time = (double)steps * dt_e;
    cudapic_report r{};
    r.steps_measured = steps;
    r.density_center = steps ? cumul[n_g / 2] / (double)steps : 0.0;
    r.plasma_freq = e_charge * std::sqrt(r.density_center / eps0 / e_mass);
    r.mean_energy_center = mc[2] ? esum / (double)mc[2] : NAN;
    const double kT = 2.0 * r.mean_energy_center * e_charge / 3.0;
    r.debye_length = std::sqrt(eps0 * kT / r.density_center) / e_charge;
    const double n_e = std::min(counts[0], p.capacity), n_i = std::min(counts[1], p.capacity);
    r.e_coll_freq = (double)mc[0] / sim_time / n_e;
    r.i_coll_freq = (double)mc[1] / sim_time / n_i;
    r.wp_dt_e = r.plasma_freq * dt_e;
    r.dx_over_debye = dx / r.debye_length;
    r.max_e_coll_dt_e = s->max_e_coll_freq * dt_e;
    r.max_i_coll_dt_i = s->max_i_coll_freq * dt_i;
    r.conditions_ok = !(r.wp_dt_e > 0.2) && !(r.dx_over_debye > 1.0) && !(r.max_e_coll_dt_e > 0.05) &&
                      !(r.max_i_coll_dt_i > 0.05);
    r.cfl_max_energy = cfl_max_energy(p);
    const double flux = p.weight / p.electrode_area / sim_time;
    r.ion_flux_pow = (double)wall[1].abs_pow * flux;
    r.ion_flux_gnd = (double)wall[1].abs_gnd * flux;
    r.e_flux_pow = (double)wall[0].abs_pow * flux;
    r.e_flux_gnd = (double)wall[0].abs_gnd * flux;
    double hp = 0.0, hg = 0.0, mp = 0.0, mg = 0.0;  // save_ifed, :824-844 (1 eV bins)
    for (int k = 0; k < CUDAPIC_N_IFED; ++k) {
        hp += wall[1].ifed_pow[k];
        hg += wall[1].ifed_gnd[k];
        mp += (k + 0.5) * wall[1].ifed_pow[k];
        mg += (k + 0.5) * wall[1].ifed_gnd[k];
    }
    r.mean_ion_energy_pow = hp > 0.0 ? mp / hp : NAN;
    r.mean_ion_energy_gnd = hg > 0.0 ? mg / hg : NAN;
    CUDAPIC_CHECK(xt_power(s, &r.power_e, &r.power_i));  // C/eduPIC.cc:1011-1026
    *out = r;
    return CUDAPIC_OK;
}

extern "C" int cudapic_state_write_info(cudapic_state *s, const char *path) {
    if (!s || !path) return fail(CUDAPIC_ERR_ARG, "state_write_info: null pointer");
    cudapic_report r;
    CUDAPIC_CHECK(cudapic_state_report(s, &r));
    const cudapic_params &p = s->params;
    FILE *f = std::fopen(path, "w");
    if (!f) return fail(CUDAPIC_ERR_ARG, std::string("state_write_info: cannot open ") + path);
    const char *rule = "--------------------------------------------------------------------------------\n";
    // the lines of check_and_save_info, C/eduPIC.cc:940-1008
    std::fprintf(f, "########################## eduPIC simulation report ############################\n");
    std::fprintf(f, "Simulation parameters:\n");
    std::fprintf(f, "Gap distance                          = %12.3e [m]\n", p.gap);
    std::fprintf(f, "# of grid divisions                   = %12d\n", (int)p.n_g);
    std::fprintf(f, "Frequency                             = %12.3e [Hz]\n", p.frequency);
    std::fprintf(f, "# of time steps / period              = %12d\n", (int)p.n_t);
    std::fprintf(f, "# of electron / ion time steps        = %12d\n", (int)p.n_sub);
    std::fprintf(f, "Voltage amplitude                     = %12.3e [V]\n", p.voltage);
    std::fprintf(f, "Pressure (Ar)                         = %12.3e [Pa]\n", p.pressure);
    std::fprintf(f, "Temperature                           = %12.3e [K]\n", p.temperature);
    std::fprintf(f, "Superparticle weight                  = %12.3e\n", p.weight);
    std::fprintf(f, "# of simulation cycles in this run    = %12d\n", (int)(r.steps_measured / p.n_t));
    std::fprintf(f, "%s", rule);
    std::fprintf(f, "Plasma characteristics:\n");
    std::fprintf(f, "Electron density @ center             = %12.3e [m^{-3}]\n", r.density_center);
    std::fprintf(f, "Plasma frequency @ center             = %12.3e [rad/s]\n", r.plasma_freq);
    std::fprintf(f, "Debye length @ center                 = %12.3e [m]\n", r.debye_length);
    std::fprintf(f, "Electron collision frequency          = %12.3e [1/s]\n", r.e_coll_freq);
    std::fprintf(f, "Ion collision frequency               = %12.3e [1/s]\n", r.i_coll_freq);
    std::fprintf(f, "%s", rule);
    std::fprintf(f, "Stability and accuracy conditions:\n");
    std::fprintf(f, "Plasma frequency @ center * DT_E      = %12.3f (OK if less than 0.20)\n", r.wp_dt_e);
    std::fprintf(f, "DX / Debye length @ center            = %12.3f (OK if less than 1.00)\n", r.dx_over_debye);
    std::fprintf(f, "Max. electron coll. frequency * DT_E  = %12.3f (OK if less than 0.05)\n", r.max_e_coll_dt_e);
    std::fprintf(f, "Max. ion coll. frequency * DT_I       = %12.3f (OK if less than 0.05)\n", r.max_i_coll_dt_i);
    if (!r.conditions_ok) {
        std::fprintf(f, "%s", rule);
        std::fprintf(f, "** STABILITY AND ACCURACY CONDITION(S) VIOLATED - REFINE SIMULATION SETTINGS! **\n");
        std::fprintf(f, "%s", rule);
    } else {
        std::fprintf(f, "Max e- energy for CFL condition       = %12.3f [eV]\n", r.cfl_max_energy);
        std::fprintf(f, "Check EEPF to ensure that CFL is fulfilled for the majority of the electrons!\n");
        std::fprintf(f, "%s", rule);
        std::fprintf(f, "Particle characteristics at the electrodes:\n");
        std::fprintf(f, "Ion flux at powered electrode         = %12.3e [m^{-2} s^{-1}]\n", r.ion_flux_pow);
        std::fprintf(f, "Ion flux at grounded electrode        = %12.3e [m^{-2} s^{-1}]\n", r.ion_flux_gnd);
        std::fprintf(f, "Mean ion energy at powered electrode  = %12.3e [eV]\n", r.mean_ion_energy_pow);
        std::fprintf(f, "Mean ion energy at grounded electrode = %12.3e [eV]\n", r.mean_ion_energy_gnd);
        std::fprintf(f, "Electron flux at powered electrode    = %12.3e [m^{-2} s^{-1}]\n", r.e_flux_pow);
        std::fprintf(f, "Electron flux at grounded electrode   = %12.3e [m^{-2} s^{-1}]\n", r.e_flux_gnd);
        std::fprintf(f, "%s", rule);
        if (!std::isnan(r.power_e)) {  // :1011-1026
            std::fprintf(f, "Absorbed power calculated as <j*E>:\n");
            std::fprintf(f, "Electron power density (average)      = %12.3e [W m^{-3}]\n", r.power_e);
            std::fprintf(f, "Ion power density (average)           = %12.3e [W m^{-3}]\n", r.power_i);
            std::fprintf(f, "Total power density(average)          = %12.3e [W m^{-3}]\n", r.power_e + r.power_i);
            std::fprintf(f, "%s", rule);
        }
    }
    const bool ok = std::fclose(f) == 0;
    return ok ? CUDAPIC_OK : fail(CUDAPIC_ERR_ARG, std::string("state_write_info: write failed: ") + path);
}

extern "C" int cudapic_state_wall_counters(cudapic_state *s, cudapic_wall_counters out[2]) {
    if (!s || !out) return fail(CUDAPIC_ERR_ARG, "state_wall_counters: null pointer");
    DeviceGuard dg(s->device);
    CUDAPIC_CHECK(check_cuda(cudaMemcpyAsync(out, s->wall, 2 * sizeof(cudapic_wall_counters), cudaMemcpyDeviceToHost,
                                             s->stream), "download wall counters"));
    return check_cuda(cudaStreamSynchronize(s->stream), "wall counters sync");
}

extern "C" int cudapic_state_download_measurements(cudapic_state *s, double *cumul_e, double *cumul_i,
                                                   uint32_t *eepf) {
    if (!s) return fail(CUDAPIC_ERR_ARG, "state_download_measurements: null state");
    DeviceGuard dg(s->device);
    const size_t n_g = s->params.n_g;
    if (cumul_e)
        CUDAPIC_CHECK(check_cuda(cudaMemcpyAsync(cumul_e, s->cumul_e, n_g * sizeof(double), cudaMemcpyDeviceToHost, s->stream), "download cumul_e"));
    if (cumul_i)
        CUDAPIC_CHECK(check_cuda(cudaMemcpyAsync(cumul_i, s->cumul_i, n_g * sizeof(double), cudaMemcpyDeviceToHost, s->stream), "download cumul_i"));
    if (eepf)
        CUDAPIC_CHECK(check_cuda(cudaMemcpyAsync(eepf, s->eepf, 2000 * sizeof(uint32_t), cudaMemcpyDeviceToHost, s->stream), "download eepf"));
    return check_cuda(cudaStreamSynchronize(s->stream), "download measurements sync");
}
