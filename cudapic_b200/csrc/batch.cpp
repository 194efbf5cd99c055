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
// The discharges stay cudapic_state objects.  While a batch exists their
// particle planes (both sides of both species and the RNG planes) live in
// one pool owned by the batch, each discharge at an element offset, so the
// kernels take the plane bases as launch parameters; the states point into
// the pool, and every state call keeps working between batch runs.  The
// pool's side 0 / 1 are the same roles for every discharge; a state moved
// on its own is brought back to the batch's side by a copy.  Destroying the
// batch gives every state its own planes back.  Each state's densities,
// counters, tables and measurements are used in place through a
// per-discharge descriptor, rebuilt when a state's density roles moved.
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
    uint32_t *counts = nullptr;      // [2][D] written by the batched Poisson solve; [2D]: scatter ticket
    bool inplace = true;             // in-place electron steps between compacting ones (all states in-place)
    float *pool = nullptr;           // POOL_PLANES x pool_len elements
    uint64_t pool_len = 0;
    std::vector<uint32_t> off;       // element offset of each discharge
    uint32_t pooled = 0;             // states [0, pooled) point into the pool
    uint32_t max_n_g = 0, flags = 0;
    uint64_t cap_sum = 0;
    bool built = false;
    // density roles of each state at the build: e_cur, i_cur; its XT buffer
    std::vector<std::array<int, 2>> origin;
    std::vector<double *> xt_at_build;
    int se = 0, si = 0;              // pool sides of the electrons and ions (absolute)
    int ecur = 0, icur = 0;          // density roles relative to the build
    cudaGraphExec_t graph[2] = {nullptr, nullptr};  // [measure]
    int graph_key[2][4] = {{-1, -1, -1, -1}, {-1, -1, -1, -1}};
    uint64_t graph_gen[2] = {0, 0};                  // tuning generation at capture

    uint32_t count() const { return (uint32_t)states.size(); }
    float *plane(int p) const { return pool + (uint64_t)p * pool_len; }
};

namespace {

void destroy_graphs(cudapic_batch *b) {
    for (auto &g : b->graph) {
        if (g) cudaGraphExecDestroy(g);
        g = nullptr;
    }
}

// Points a state's particle planes at planes[0..23] (pool order: its range
// of the pool, or its own buffers again).
void point_state(cudapic_state *s, float *const *planes) {
    for (int sp = 0; sp < 2; ++sp) {
        for (int side = 0; side < 2; ++side) {
            s->x[sp][side] = planes[pool_plane(sp, side, 0)];
            s->vx[sp][side] = planes[pool_plane(sp, side, 1)];
            s->vy[sp][side] = planes[pool_plane(sp, side, 2)];
            s->vz[sp][side] = planes[pool_plane(sp, side, 3)];
        }
        for (int k = 0; k < 4; ++k) s->rng[sp][k] = reinterpret_cast<uint32_t *>(planes[pool_rng_plane(sp, k)]);
    }
    state_drop_graphs(s);
}

// The state's 24 planes in pool order (pool side j = the state's side
// side[sp] ^ j, so the live side lands on pool side 0).
void state_planes(const cudapic_state *s, float *out[POOL_PLANES]) {
    for (int sp = 0; sp < 2; ++sp) {
        for (int j = 0; j < 2; ++j) {
            const int a = s->side[sp] ^ j;
            out[pool_plane(sp, j, 0)] = s->x[sp][a];
            out[pool_plane(sp, j, 1)] = s->vx[sp][a];
            out[pool_plane(sp, j, 2)] = s->vy[sp][a];
            out[pool_plane(sp, j, 3)] = s->vz[sp][a];
        }
        for (int k = 0; k < 4; ++k) out[pool_rng_plane(sp, k)] = reinterpret_cast<float *>(s->rng[sp][k]);
    }
}

// Moves every state's planes into the pool (live side to pool side 0).
int pool_states(cudapic_batch *b) {
    for (uint32_t k = 0; k < b->count(); ++k) {
        cudapic_state *s = b->states[k];
        const size_t bytes = (size_t)s->params.capacity * sizeof(float);
        CUDAPIC_CHECK(check_cuda(cudaStreamSynchronize(s->stream), "batch: state sync"));
        float *from[POOL_PLANES], *to[POOL_PLANES];
        state_planes(s, from);
        for (int p = 0; p < POOL_PLANES; ++p) {
            to[p] = b->plane(p) + b->off[k];
            CUDAPIC_CHECK(check_cuda(cudaMemcpyAsync(to[p], from[p], bytes, cudaMemcpyDeviceToDevice, b->stream),
                                     "batch: pool copy"));
        }
        CUDAPIC_CHECK(check_cuda(cudaStreamSynchronize(b->stream), "batch: pool sync"));
        for (int p = 0; p < POOL_PLANES; ++p) state_release(s, from[p]);
        point_state(s, to);
        s->side[0] = s->side[1] = 0;
        s->batch = b;
        b->pooled = k + 1;
    }
    return CUDAPIC_OK;
}

// Gives every pooled state its own planes back (the pool's contents, same sides).
int unpool_states(cudapic_batch *b) {
    while (b->pooled > 0) {
        const uint32_t k = b->pooled - 1;
        cudapic_state *s = b->states[k];
        const size_t bytes = (size_t)s->params.capacity * sizeof(float);
        float *own[POOL_PLANES];
        for (int p = 0; p < POOL_PLANES; ++p) {
            void *ptr = nullptr;
            CUDAPIC_CHECK(state_alloc(s, &ptr, bytes));
            own[p] = static_cast<float *>(ptr);
            CUDAPIC_CHECK(check_cuda(cudaMemcpyAsync(own[p], b->plane(p) + b->off[k], bytes,
                                                     cudaMemcpyDeviceToDevice, b->stream), "batch: unpool copy"));
        }
        CUDAPIC_CHECK(check_cuda(cudaStreamSynchronize(b->stream), "batch: unpool sync"));
        point_state(s, own);
        s->batch = nullptr;
        b->pooled = k;
    }
    return CUDAPIC_OK;
}

// Descriptors of the states' per-discharge buffers, density roles as they
// are oriented now (relative roles back to zero).
int build(cudapic_batch *b) {
    const uint32_t D = b->count();
    std::vector<BatchDisc> host(D);
    b->origin.resize(D);
    b->xt_at_build.resize(D);
    for (uint32_t k = 0; k < D; ++k) {
        cudapic_state *s = b->states[k];
        BatchDisc &d = host[k];
        std::memset(&d, 0, sizeof(d));
        d.g = s->grid;
        d.off = b->off[k];
        for (int r = 0; r < 2; ++r) {
            d.e_dens[r] = s->e_dens[s->e_cur ^ r];
            d.i_dens[r] = s->i_dens[s->i_cur ^ r];
        }
        d.counters = s->counters;
        d.efield = s->efield;
        d.pot = s->pot;
        d.pot0_table = s->pot0_table;
        // the per-process cross sections are argon's, whatever the discharge
        // (host.cpp cs_range: only the totals scale with the gas density), so
        // every discharge reads the first state's copy: the scattering's
        // gathers share one L2-resident table instead of one per discharge
        d.cs = b->states[0]->cs;
        d.sigma_tot_e = s->sigma_tot_e;
        d.sigma_tot_i = s->sigma_tot_i;
        d.sigma_max_e = s->sigma_max_e;
        d.ion_k = s->ion_k;
        d.wall = s->wall;
        d.mcount = s->mcount;
        d.cumul_e = s->cumul_e;
        d.cumul_i = s->cumul_i;
        d.esum = s->esum;
        d.eepf = s->eepf;
        d.xt = s->xt;
        d.n_xt = s->n_xt;
        b->xt_at_build[k] = s->xt;
        b->origin[k] = {s->e_cur, s->i_cur};
    }
    CUDAPIC_CHECK(check_cuda(cudaMemcpy(b->desc, host.data(), D * sizeof(BatchDisc), cudaMemcpyHostToDevice),
                             "batch: upload descriptors"));
    b->ecur = b->icur = 0;
    destroy_graphs(b);
    b->built = true;
    return CUDAPIC_OK;
}

StepPlanes step_planes(const cudapic_batch *b, int sp, int src, int ion_side) {
    StepPlanes pl;
    pl.sx = b->plane(pool_plane(sp, src, 0));
    pl.svx = b->plane(pool_plane(sp, src, 1));
    pl.svy = b->plane(pool_plane(sp, src, 2));
    pl.svz = b->plane(pool_plane(sp, src, 3));
    pl.dx = b->plane(pool_plane(sp, src ^ 1, 0));
    pl.dvx = b->plane(pool_plane(sp, src ^ 1, 1));
    pl.dvy = b->plane(pool_plane(sp, src ^ 1, 2));
    pl.dvz = b->plane(pool_plane(sp, src ^ 1, 3));
    pl.rng0 = reinterpret_cast<uint32_t *>(b->plane(pool_rng_plane(sp, 0)));
    pl.rng1 = reinterpret_cast<uint32_t *>(b->plane(pool_rng_plane(sp, 1)));
    pl.rng2 = reinterpret_cast<uint32_t *>(b->plane(pool_rng_plane(sp, 2)));
    pl.rng3 = reinterpret_cast<uint32_t *>(b->plane(pool_rng_plane(sp, 3)));
    pl.ix = b->plane(pool_plane(1, ion_side, 0));
    pl.ivx = b->plane(pool_plane(1, ion_side, 1));
    pl.ivy = b->plane(pool_plane(1, ion_side, 2));
    pl.ivz = b->plane(pool_plane(1, ion_side, 3));
    return pl;
}

SidePlanes side_planes(const cudapic_batch *b, int sp, int side) {
    SidePlanes s;
    s.x = b->plane(pool_plane(sp, side, 0));
    s.vx = b->plane(pool_plane(sp, side, 1));
    s.vy = b->plane(pool_plane(sp, side, 2));
    s.vz = b->plane(pool_plane(sp, side, 3));
    s.rng0 = reinterpret_cast<uint32_t *>(b->plane(pool_rng_plane(sp, 0)));
    s.rng1 = reinterpret_cast<uint32_t *>(b->plane(pool_rng_plane(sp, 1)));
    s.rng2 = reinterpret_cast<uint32_t *>(b->plane(pool_rng_plane(sp, 2)));
    s.rng3 = reinterpret_cast<uint32_t *>(b->plane(pool_rng_plane(sp, 3)));
    return s;
}

// Per-kernel timing of uncaptured steps (cudapic_batch_profile_steps): an
// event before and after every kernel group of a step.
struct BatchProfile {
    std::vector<cudaEvent_t> ev;   // pairs, in the order of `kind`
    std::vector<int> kind;         // CUDAPIC_BATCH_K_*
    int mark(int k, cudaStream_t st, bool end) {
        cudaEvent_t e = nullptr;
        CUDAPIC_CHECK(check_cuda(cudaEventCreate(&e), "batch profile: event"));
        ev.push_back(e);
        if (!end) kind.push_back(k);
        return check_cuda(cudaEventRecord(e, st), "batch profile: record");
    }
    ~BatchProfile() {
        for (auto e : ev) cudaEventDestroy(e);
    }
};

// As in the one-discharge driver: the electron step before every N_SUB-th
// step compacts (and the last step of every run), the others run in place.
bool batch_compact_step(const cudapic_state *s0, uint64_t step) { return ((step + 1) % s0->params.n_sub) == 0; }

// One step of every discharge (the order of state.cpp's fused step).
int enqueue_batch_step(cudapic_batch *b, bool ion_step, bool measure, bool compact, BatchProfile *prof = nullptr) {
    PdlScope pdl(prof == nullptr);  // the profiler's events sit between the kernels
    const uint32_t D = b->count();
    cudaStream_t st = b->stream;
    auto begin = [&](int k) { return prof ? prof->mark(k, st, false) : CUDAPIC_OK; };
    auto finish = [&](int k) { return prof ? prof->mark(k, st, true) : CUDAPIC_OK; };
    if (ion_step) b->icur ^= 1;  // the buffer that collected the period's ion deposits becomes current
    CUDAPIC_CHECK(begin(CUDAPIC_BATCH_K_POISSON));
    CUDAPIC_CHECK(launch_batch_poisson(b->desc, b->counts, D, b->max_n_g, b->flags, b->ecur, b->icur, ion_step ? 1 : 0,
                                       measure ? 1 : 0, st));
    CUDAPIC_CHECK(finish(CUDAPIC_BATCH_K_POISSON));
    if (measure) {  // XT diagnostics: the particles before their push
        CUDAPIC_CHECK(launch_batch_xt_particles(false, side_planes(b, 0, b->se), b->desc, D, b->max_n_g, b->cap_sum,
                                                st));
        if (ion_step)
            CUDAPIC_CHECK(launch_batch_xt_particles(true, side_planes(b, 1, b->si), b->desc, D, b->max_n_g,
                                                    b->cap_sum, st));
    }
    StepRoles r{};
    r.dens_i = b->icur ^ 1;
    r.measure = measure ? 1 : 0;
    if (ion_step) {
        r.dens = b->icur ^ 1;
        CUDAPIC_CHECK(begin(CUDAPIC_BATCH_K_ION_PUSH));
        CUDAPIC_CHECK(launch_batch_step(false, step_planes(b, 1, b->si, b->si ^ 1), b->desc, b->counts + D, D,
                                        b->cap_sum, b->max_n_g, r, st));
        CUDAPIC_CHECK(finish(CUDAPIC_BATCH_K_ION_PUSH));
        b->si ^= 1;
    }
    r.dens = b->ecur ^ 1;
    if (b->inplace && !compact) {
        // in place: the electrons stay on their side, collider records go to
        // the other sides' planes of both species, the scatter pass follows
        const SidePlanes es = side_planes(b, 0, b->se);
        const SidePlanes is = side_planes(b, 1, b->si);
        const InplacePlanes pl{es.x, es.vx, es.vy, es.vz, es.rng0, es.rng1, es.rng2, es.rng3,
                               is.x, is.vx, is.vy, is.vz};
        const SidePlanes os = side_planes(b, 0, b->se ^ 1);
        const SidePlanes oi = side_planes(b, 1, b->si ^ 1);
        const CollList list{reinterpret_cast<uint32_t *>(os.x), os.vx, os.vy, os.vz,
                            reinterpret_cast<uint32_t *>(oi.x), reinterpret_cast<uint32_t *>(oi.vx),
                            reinterpret_cast<uint32_t *>(oi.vy), reinterpret_cast<uint32_t *>(oi.vz)};
        CUDAPIC_CHECK(begin(CUDAPIC_BATCH_K_ELECTRON_INPLACE));
        CUDAPIC_CHECK(launch_batch_inplace(pl, list, b->desc, b->counts, D, b->cap_sum, b->max_n_g, r, st));
        CUDAPIC_CHECK(finish(CUDAPIC_BATCH_K_ELECTRON_INPLACE));
        CUDAPIC_CHECK(begin(CUDAPIC_BATCH_K_ELECTRON_SCATTER));
        CUDAPIC_CHECK(launch_batch_scatter(pl, list, b->desc, D, b->cap_sum, r, b->counts + 2 * D, st));
        CUDAPIC_CHECK(finish(CUDAPIC_BATCH_K_ELECTRON_SCATTER));
    } else {
        CUDAPIC_CHECK(begin(CUDAPIC_BATCH_K_ELECTRON_STEP));
        CUDAPIC_CHECK(launch_batch_step(true, step_planes(b, 0, b->se, b->si), b->desc, b->counts, D, b->cap_sum,
                                        b->max_n_g, r, st));
        CUDAPIC_CHECK(finish(CUDAPIC_BATCH_K_ELECTRON_STEP));
        b->se ^= 1;
    }
    b->ecur ^= 1;
    if (ion_step) {
        CUDAPIC_CHECK(begin(CUDAPIC_BATCH_K_ION_COLLISIONS));
        CUDAPIC_CHECK(launch_batch_collisions_i(side_planes(b, 1, b->si), b->desc, D, b->cap_sum, measure ? 1 : 0, st));
        CUDAPIC_CHECK(finish(CUDAPIC_BATCH_K_ION_COLLISIONS));
    }
    if (measure) CUDAPIC_CHECK(launch_batch_eepf(side_planes(b, 0, b->se), b->desc, D, b->cap_sum, st));
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
        rc = enqueue_batch_step(b, state_is_ion_step(s0, first_step + k), measure,
                                batch_compact_step(s0, first_step + k) || k + 1 == period);
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
    b->graph_gen[m] = tuning_generation();
    return check_cuda(e, "cudaGraphInstantiate");
}

}  // namespace

extern "C" int cudapic_batch_create(cudapic_state *const *states, uint32_t count, cudapic_batch **out) {
    CUDAPIC_REQUIRE(states && out, "batch_create: null pointer");
    *out = nullptr;
    CUDAPIC_REQUIRE(count >= 1 && count <= BATCH_MAX_DISCHARGES, "batch_create: count must be in [1, 1024]");
    const cudapic_state *s0 = states[0];
    CUDAPIC_REQUIRE(s0, "batch_create: null state");
    uint64_t cap_sum = 0, pool_len = 0;
    uint32_t max_n_g = 0;
    std::vector<uint32_t> off(count);
    for (uint32_t k = 0; k < count; ++k) {
        const cudapic_state *s = states[k];
        CUDAPIC_REQUIRE(s, "batch_create: null state");
        for (uint32_t j = 0; j < k; ++j) CUDAPIC_REQUIRE(states[j] != s, "batch_create: a state appears twice");
        CUDAPIC_REQUIRE(!s->batch, "batch_create: a state already belongs to a batch");
        CUDAPIC_REQUIRE(s->device == s0->device, "batch_create: the states must share one device");
        CUDAPIC_REQUIRE(s->params.n_t == s0->params.n_t && s->params.n_sub == s0->params.n_sub,
                        "batch_create: the states must share N_T and N_SUB");
        CUDAPIC_REQUIRE((s->params.flags & CUDAPIC_FLAG_POISSON_F32_SCAN) ==
                            (s0->params.flags & CUDAPIC_FLAG_POISSON_F32_SCAN),
                        "batch_create: the states must share the Poisson arithmetic flag");
        CUDAPIC_REQUIRE(s->graphs_enabled || (s->params.n_t % s->params.n_sub) == 0,
                        "batch_create: N_T must be a multiple of N_SUB");
        off[k] = (uint32_t)pool_len;
        cap_sum += s->grid.capacity;
        pool_len += (s->grid.capacity + 63u) & ~63ull;
        max_n_g = std::max(max_n_g, s->grid.n_g);
        CUDAPIC_REQUIRE(pool_len <= 0x80000000ull, "batch_create: the capacities must sum to at most 2^31");
    }
    DeviceGuard dg(s0->device);
    cudapic_batch *b = new (std::nothrow) cudapic_batch();
    if (!b) return fail(CUDAPIC_ERR_ARG, "batch_create: out of host memory");
    b->device = s0->device;
    b->cap_sum = cap_sum;
    b->pool_len = pool_len;
    b->off = off;
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
        (rc = check_cuda(cudaMalloc(&b->counts, (2ull * count + 8) * sizeof(uint32_t)), "batch: counts")) ||
        (rc = check_cuda(cudaMemset(b->counts, 0, (2ull * count + 8) * sizeof(uint32_t)), "batch: counts")) ||
        (rc = check_cuda(cudaMalloc(&b->pool, (size_t)POOL_PLANES * pool_len * sizeof(float)), "batch: pool")))
        return cleanup(rc);
    b->ready.assign(count, nullptr);
    for (auto &ev : b->ready)
        if ((rc = check_cuda(cudaEventCreateWithFlags(&ev, cudaEventDisableTiming), "batch: event")))
            return cleanup(rc);
    // the states join only once everything else is in place
    b->states.assign(states, states + count);
    if ((rc = pool_states(b))) {
        // a state moved already points into the pool: give the planes back
        unpool_states(b);
        return cleanup(rc);
    }
    *out = b;
    return CUDAPIC_OK;
}

extern "C" int cudapic_batch_destroy(cudapic_batch *b) {
    if (!b) return CUDAPIC_OK;
    DeviceGuard dg(b->device);
    if (b->stream) cudaStreamSynchronize(b->stream);
    const int rc = unpool_states(b);
    if (rc != CUDAPIC_OK) {
        // some states still point into the pool: keep it (and the batch's
        // other buffers) rather than leave them dangling
        return rc;
    }
    destroy_graphs(b);
    for (auto ev : b->ready)
        if (ev) cudaEventDestroy(ev);
    if (b->done) cudaEventDestroy(b->done);
    if (b->desc) cudaFree(b->desc);
    if (b->counts) cudaFree(b->counts);
    if (b->pool) cudaFree(b->pool);
    if (b->stream) cudaStreamDestroy(b->stream);
    delete b;
    return rc;
}

extern "C" cudapic_stream_t cudapic_batch_stream(const cudapic_batch *b) {
    return b ? (cudapic_stream_t)b->stream : nullptr;
}

extern "C" int cudapic_batch_synchronize(cudapic_batch *b) {
    if (!b) return fail(CUDAPIC_ERR_ARG, "batch_synchronize: null batch");
    DeviceGuard dg(b->device);
    return check_cuda(cudaStreamSynchronize(b->stream), "batch_synchronize");
}

namespace {

// Checks the states and brings them to where the batch's kernels expect
// them: descriptors current, after each state's pending work, live sides on
// the batch's sides, fused densities primed.
int prepare_run(cudapic_batch *b) {
    const uint32_t D = b->count();
    cudapic_state *s0 = b->states[0];
    const uint64_t steps0 = s0->steps_done;
    const bool measure = s0->measure;
    bool stale = !b->built;
    bool inplace = true;
    for (uint32_t k = 0; k < D; ++k) {
        const cudapic_state *s = b->states[k];
        inplace = inplace && s->inplace;
        CUDAPIC_REQUIRE(s->steps_done == steps0, "batch_run_steps: the states are at different steps");
        CUDAPIC_REQUIRE(s->measure == measure, "batch_run_steps: the states differ in measurement mode");
        CUDAPIC_REQUIRE(s->fused, "batch_run_steps: a state is in unfused (reference sequence) mode");
        if (b->built && (s->e_cur != (b->origin[k][0] ^ b->ecur) || s->i_cur != (b->origin[k][1] ^ b->icur) ||
                         s->xt != b->xt_at_build[k]))
            stale = true;
    }
    if (inplace != b->inplace) {
        b->inplace = inplace;
        destroy_graphs(b);
    }
    if (stale) CUDAPIC_CHECK(build(b));
    // after every state's pending work (uploads, seeding, its own steps)
    for (uint32_t k = 0; k < D; ++k) {
        CUDAPIC_CHECK(check_cuda(cudaEventRecord(b->ready[k], b->states[k]->stream), "batch: record"));
        CUDAPIC_CHECK(check_cuda(cudaStreamWaitEvent(b->stream, b->ready[k], 0), "batch: wait"));
    }
    // a state stepped on its own lives on the other pool side: copy it back
    for (uint32_t k = 0; k < D; ++k) {
        cudapic_state *s = b->states[k];
        const int want[2] = {b->se, b->si};
        const size_t bytes = (size_t)s->params.capacity * sizeof(float);
        for (int sp = 0; sp < 2; ++sp) {
            if (s->side[sp] == want[sp]) continue;
            for (int c = 0; c < 4; ++c)
                CUDAPIC_CHECK(check_cuda(
                    cudaMemcpyAsync(b->plane(pool_plane(sp, want[sp], c)) + b->off[k],
                                    b->plane(pool_plane(sp, s->side[sp], c)) + b->off[k], bytes,
                                    cudaMemcpyDeviceToDevice, b->stream), "batch: side copy"));
            s->side[sp] = want[sp];
            state_drop_graphs(s);
        }
    }
    for (uint32_t k = 0; k < D; ++k)
        if (!b->states[k]->dens_valid) CUDAPIC_CHECK(state_prime_fused(b->states[k], b->stream));
    return CUDAPIC_OK;
}

// The states' bookkeeping after steps [steps0, step) were enqueued; every
// state's own stream continues after the batch's work.
int finish_run(cudapic_batch *b, uint64_t steps0, uint64_t step) {
    const uint32_t D = b->count();
    const uint64_t done_steps = step - steps0;
    for (uint32_t k = 0; k < D; ++k) {
        cudapic_state *s = b->states[k];
        s->side[0] = b->se;
        s->side[1] = b->si;
        s->e_cur = b->origin[k][0] ^ b->ecur;
        s->i_cur = b->origin[k][1] ^ b->icur;
        s->steps_done = step;
        if (s->measure) s->measure_steps += done_steps;
    }
    CUDAPIC_CHECK(check_cuda(cudaEventRecord(b->done, b->stream), "batch: record"));
    for (uint32_t k = 0; k < D; ++k)
        CUDAPIC_CHECK(check_cuda(cudaStreamWaitEvent(b->states[k]->stream, b->done, 0), "batch: wait"));
    return CUDAPIC_OK;
}

}  // namespace

extern "C" int cudapic_batch_run_steps(cudapic_batch *b, uint64_t n_steps) {
    if (!b) return fail(CUDAPIC_ERR_ARG, "batch_run_steps: null batch");
    DeviceGuard dg(b->device);
    CUDAPIC_CHECK(prepare_run(b));
    cudapic_state *s0 = b->states[0];
    const uint64_t steps0 = s0->steps_done;
    const bool measure = s0->measure;
    const uint64_t period = 2ull * s0->params.n_sub;
    uint64_t step = steps0;
    int rc = CUDAPIC_OK;
    while (n_steps > 0 && rc == CUDAPIC_OK) {
        if ((step % period) == 0 && n_steps >= period) {
            const int m = measure ? 1 : 0;
            const int key[4] = {b->se, b->si, b->ecur, b->icur};
            if (b->graph[m] && (std::memcmp(key, b->graph_key[m], sizeof(key)) != 0 ||
                                b->graph_gen[m] != tuning_generation())) {
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
        rc = enqueue_batch_step(b, state_is_ion_step(s0, step), measure,
                                batch_compact_step(s0, step) || n_steps == 1);
        if (rc == CUDAPIC_OK) {
            step += 1;
            n_steps -= 1;
        }
    }
    // the states' bookkeeping follows what was enqueued
    const int rc2 = finish_run(b, steps0, step);
    return rc != CUDAPIC_OK ? rc : rc2;
}

extern "C" int cudapic_batch_profile_steps(cudapic_batch *b, uint64_t n_steps, double ms[CUDAPIC_BATCH_KERNELS],
                                           uint64_t launches[CUDAPIC_BATCH_KERNELS]) {
    if (!b) return fail(CUDAPIC_ERR_ARG, "batch_profile_steps: null batch");
    CUDAPIC_REQUIRE(ms && launches, "batch_profile_steps: null pointer");
    CUDAPIC_REQUIRE(n_steps <= 4096, "batch_profile_steps: at most 4096 steps per call");
    DeviceGuard dg(b->device);
    CUDAPIC_CHECK(prepare_run(b));
    cudapic_state *s0 = b->states[0];
    const uint64_t steps0 = s0->steps_done;
    const bool measure = s0->measure;
    uint64_t step = steps0;
    BatchProfile prof;
    int rc = CUDAPIC_OK;
    for (; step < steps0 + n_steps && rc == CUDAPIC_OK; ++step)
        rc = enqueue_batch_step(b, state_is_ion_step(s0, step), measure,
                                batch_compact_step(s0, step) || step + 1 == steps0 + n_steps, &prof);
    if (rc != CUDAPIC_OK) --step;  // the failed step was not (completely) enqueued
    const int rc2 = finish_run(b, steps0, step);
    CUDAPIC_CHECK(rc);
    CUDAPIC_CHECK(rc2);
    CUDAPIC_CHECK(check_cuda(cudaStreamSynchronize(b->stream), "batch profile: sync"));
    for (int k = 0; k < CUDAPIC_BATCH_KERNELS; ++k) {
        ms[k] = 0.0;
        launches[k] = 0;
    }
    for (size_t j = 0; j < prof.kind.size(); ++j) {
        float t = 0.0f;
        CUDAPIC_CHECK(check_cuda(cudaEventElapsedTime(&t, prof.ev[2 * j], prof.ev[2 * j + 1]), "batch profile: time"));
        ms[prof.kind[j]] += t;
        launches[prof.kind[j]] += 1;
    }
    return CUDAPIC_OK;
}
