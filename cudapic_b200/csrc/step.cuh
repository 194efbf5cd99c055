// step.cuh -- the tile pipeline of the fused particle steps, shared by the
// one-discharge kernel (kernels_step.cu) and the batched kernels
// (kernels_batch.cu).
//
// A segment is a contiguous range [beg, end) of one species of one
// discharge.  step_segment<U, MCC> streams its SoA planes through shared
// memory with cp.async.bulk on an mbarrier ring, pushes every particle
// (Rust-CUDA/src/main.rs:596-620), compacts the survivors into the other
// side (ballots, one warp scan and one atomicAdd per tile, :566-678) and
// deposits them into the next density in 2^-20 fixed point (push.cuh).
// With MCC (electrons) it also runs the collision test and the scattering
// (check_collisions_e / collision_e, :971-1165) with the RNG stream of each
// particle's source slot; without (ions) it is the ion push of the driver.
#pragma once
#include "batch_internal.h"
#include "common.cuh"
#include "mcc.cuh"
#include "push.cuh"
#include "tma.cuh"

namespace cudapic {

constexpr int ES_THREADS = 256;
constexpr int ES_WARPS = ES_THREADS / 32;
constexpr int ES_MAX_STAGES = 6;  // pipeline depth: cudapic_tuning.step_stages

// U (cudapic_tuning.step_rows, 1, 2 or 4): particles per thread and tile,
// so a tile holds 256 U particles.  Planes: x, vx, vy, vz (+ rng0..3 with
// MCC).  Colliders wait in one CTA-wide queue until DRAIN_AT are pending
// (or the segment ends); the queue then never holds more than
// DRAIN_AT - 1 + TILE entries.
template <int U, bool MCC>
struct StepShape {
    static constexpr int TILE = ES_THREADS * U;
    static constexpr int PLANES = MCC ? 8 : 4;
    static constexpr int DRAIN_AT = 4 * ES_THREADS;
    static constexpr int QCAP = MCC ? DRAIN_AT + TILE : 0;
    static constexpr int NSEG = U * ES_WARPS;  // (row, warp) segments of a tile
    static_assert(U * ES_WARPS <= 32, "one warp scans the (row, warp) counts");
};

// Dynamic shared memory: [stages][PLANES][TILE] staged planes, E[ef_pad],
// the 64-bit deposit accumulator [ef_pad], [copies][ef_pad] fixed-point
// histograms, the warps' collider queues, the stage mbarriers.  copies == 0
// selects the large-grid deposit: one f32 histogram [ef_pad] in the
// accumulator's place and no copies (push.cuh dep_add_f32).
template <int U, bool MCC>
__host__ __device__ constexpr size_t step_smem_bytes(int stages, int copies, uint32_t ef_pad) {
    using S = StepShape<U, MCC>;
    return (size_t)stages * S::PLANES * S::TILE * 4 +
           (copies ? (size_t)ef_pad * (4 + 8) + (size_t)copies * ef_pad * 4 : (size_t)ef_pad * (4 + 4)) +
           (size_t)S::QCAP * 4 + (size_t)stages * sizeof(uint64_t);
}

// A per-discharge pointer of a segment's StepDisc that the tile loop uses
// rarely.  SH: the StepDisc is in shared memory (the batched kernels) and
// the pointer is reloaded where it is used, so that no register holds it
// across the loop; otherwise it is read as is (kernel parameters).
template <bool SH, typename T>
__device__ __forceinline__ T *dcp(T *const &field) {
    if constexpr (SH) {
        uint64_t v;
        asm volatile("ld.shared.u64 %0, [%1];" : "=l"(v) : "r"(smem_addr(&field)));
        return reinterpret_cast<T *>(v);
    } else {
        return field;
    }
}

// Per-discharge buffers and constants of a segment.
struct StepDisc {
    const float *efield;
    const float *sigma_tot, *cs;              // MCC: total and per-process cross sections
    float sigma_max;                          // MCC: largest entry of sigma_tot
    float factor, dt;                         // push constants of the species
    uint32_t *alive;                          // destination slot counter
    uint32_t *n_i;                            // MCC: ion count (spawn slots)
    float *dens;                              // next density of the species (survivors)
    float *dens_i;                            // MCC: next ion density (spawned ions)
    cudapic_wall_counters *wall;              // absorbed particles (may be null)
    unsigned long long *coll;                 // MCC: collision events (may be null)
};

template <int U, bool MCC>
struct StepSmem {
    uint32_t *in;
    float *ef;
    unsigned long long *acc;
    uint32_t *hist;
    uint32_t *queue;
    uint64_t *bar;
    uint32_t (*offs)[StepShape<U, MCC>::NSEG];  // [3][NSEG]
    uint32_t *s_base;                            // [3]
    uint32_t (*ccnt)[StepShape<U, MCC>::NSEG];   // [3][NSEG] colliders per (row, warp) (MCC)

    __device__ __forceinline__ StepSmem(unsigned char *smem, int stages, int copies, uint32_t ef_pad,
                                        uint32_t (*offs_)[StepShape<U, MCC>::NSEG], uint32_t *s_base_,
                                        uint32_t (*ccnt_)[StepShape<U, MCC>::NSEG]) {
        using S = StepShape<U, MCC>;
        in = reinterpret_cast<uint32_t *>(smem);
        ef = reinterpret_cast<float *>(in + stages * S::PLANES * S::TILE);
        acc = reinterpret_cast<unsigned long long *>(ef + ef_pad);  // the f32 histogram when copies == 0
        hist = copies ? reinterpret_cast<uint32_t *>(acc + ef_pad) : reinterpret_cast<uint32_t *>(ef + 2u * ef_pad);
        queue = hist + (uint32_t)copies * ef_pad;
        bar = reinterpret_cast<uint64_t *>(queue + S::QCAP);
        offs = offs_;
        s_base = s_base_;
        ccnt = ccnt_;
    }
    // end of the carved region (the batched kernels put their plan there)
    __device__ __forceinline__ unsigned char *end(int stages) const {
        return reinterpret_cast<unsigned char *>(bar + stages);
    }
};

// Survivors of one tile held in registers until their base is known.
template <int U>
struct StepOut {
    float x[U], vx[U], vy[U], vz[U];
    uint32_t lane_off[U];
    uint32_t keep;  // bit u: the particle of row u is written by the tile
};

// True unless u certainly exceeds the collision probability of an electron
// with v.v = v2.  The exact test decides "no collision" whenever
// u >= B = fl(fl(fl(sigma(E) |v|) dt) + 5e-7), |v| = fl(sqrt(v2)); rounding
// is monotone, so with sigma_max the largest table entry
// u >= fl(fl(fl(sigma_max |v|) dt) + 5e-7) implies it.  The same bound
// without the square root: with k2 = fl(fl(sigma_max dt)^2 * 1.0001) and
// y = fl(u - 5.001e-7) >= 0, fl(y y) >= fl(k2 v2) gives
// y >= sigma_max dt sqrt(v2) (1 + 4.8e-5) (each rounding is within 2^-24
// relative), hence u - 5.001e-7 >= A (1 + 4.6e-5) with
// A = fl(fl(sigma_max |v|) dt) <= sigma_max dt sqrt(v2) (1 + 2e-7), and
// u >= A + 5e-7 + 1e-10 + 4.6e-5 A > fl(A + 5e-7): the decision is the
// exact test's, bit for bit; only u within 1e-4 relative of the bound
// takes the exact test in addition.
__device__ __forceinline__ bool may_collide(float u, float v2, float k2) {
    const float y = u - 5.001e-7f;
    return !(y >= 0.0f && y * y >= k2 * v2);
}

// Adds the CTA's per-thread counts v to *work (may be null): one atomic per warp.
__device__ __forceinline__ void add_work(unsigned long long *work, uint32_t v) {
    if (!work) return;
    const uint32_t s = __reduce_add_sync(0xffffffffu, v);
    if ((threadIdx.x & 31) == 0 && s) atomicAdd(work, (unsigned long long)s);
}

// Initialises the stage mbarriers (thread 0) and clears the deposit
// accumulators; the caller synchronises before the first segment.
template <int U, bool MCC>
__device__ __forceinline__ void step_smem_init(const StepSmem<U, MCC> &sm, int stages, int copies, uint32_t ef_pad) {
    if (threadIdx.x == 0) {
        for (int s = 0; s < stages; ++s) mbar_init(&sm.bar[s], 1);
        fence_mbar_init();
    }
    for (uint32_t k = threadIdx.x; k < (uint32_t)copies * ef_pad; k += ES_THREADS) sm.hist[k] = 0u;
    if (copies == 0) {
        float *hf = reinterpret_cast<float *>(sm.acc);
        for (uint32_t k = threadIdx.x; k < ef_pad; k += ES_THREADS) hf[k] = 0.0f;
        return;
    }
    for (uint32_t k = threadIdx.x; k < ef_pad; k += ES_THREADS) sm.acc[k] = 0ull;
}

// Processes the particles [beg, end) (discharge-local) of one species of
// one discharge whose planes start at element `off`.  On entry the
// histograms and the accumulator are zero; on return they are zero again
// (drained, the accumulator flushed into dc.dens and cleared).  `it` counts
// the tiles this CTA has run through the stage ring (it selects the stage
// and its mbarrier phase) and is advanced by the segment's tiles.  Returns
// false when a stage wait timed out (CUDAPIC_DEVERR_TIMEOUT set); the
// survivors held so far are still written and the deposits flushed.
// g: the grid constants as the tile loop reads them (a register copy in the
// batched kernels); gm: the same constants in memory, for the out-of-line
// scattering routine.
// SH: dc lives in shared memory; WALL: compile the electrode counters in
// (dc.wall may still be null at run time).
// live: incremented by every particle of [beg, end) that is pushed (slots
// emptied by an in-place step are skipped: not pushed, not kept, not counted).
template <int U, bool MCC, bool SH, bool WALL>
__device__ __forceinline__ bool step_segment(const StepPlanes &pl, const StepDisc &dc, const cudapic_grid &g,
                                             const cudapic_grid &gm, uint32_t off, uint32_t beg, uint32_t end,
                                             const StepSmem<U, MCC> &sm, int stages, int copies, uint32_t ef_pad,
                                             uint32_t epoch, uint32_t &it, uint32_t &live) {
    using S = StepShape<U, MCC>;
    constexpr int TILE = S::TILE;
    constexpr int PLANES = S::PLANES;
    constexpr int QCAP = S::QCAP;
    constexpr int NSEG = S::NSEG;
    const int tid = threadIdx.x;
    const int lane = tid & 31;
    const int warp = tid >> 5;
    const unsigned lt = lanemask_lt();
    // the push and test constants, read once (io may live in shared memory,
    // which the tile loop writes)
    const float factor = dc.factor, dt = dc.dt, sigma_max = dc.sigma_max;
    const float rej_k2 = sigma_max * dt * (sigma_max * dt) * 1.0001f;  // may_collide's bound
    const float inv_dx = g.inv_dx, gap = g.gap;
    const uint32_t n_g = g.n_g;
    const uint32_t it0 = it;
    const uint32_t ntiles = (end - beg + TILE - 1) / TILE;  // this segment's tiles

    auto issue = [&](uint32_t tile, int stage) {  // tile: index within the segment
        const uint32_t t0 = beg + tile * TILE;
        const uint32_t cnt = min((uint32_t)TILE, end - t0);
        const uint32_t bytes = ((cnt + 3u) & ~3u) * 4u;  // beg is a multiple of 4; so is the capacity
        mbar_arrive_expect_tx(&sm.bar[stage], PLANES * bytes);
        bulk_load(sm.in + (stage * PLANES + 0) * TILE, pl.sx + (off + t0), bytes, &sm.bar[stage]);
        bulk_load(sm.in + (stage * PLANES + 1) * TILE, pl.svx + (off + t0), bytes, &sm.bar[stage]);
        bulk_load(sm.in + (stage * PLANES + 2) * TILE, pl.svy + (off + t0), bytes, &sm.bar[stage]);
        bulk_load(sm.in + (stage * PLANES + 3) * TILE, pl.svz + (off + t0), bytes, &sm.bar[stage]);
        if (MCC) {
            bulk_load(sm.in + (stage * PLANES + 4) * TILE, pl.rng0 + (off + t0), bytes, &sm.bar[stage]);
            bulk_load(sm.in + (stage * PLANES + 5) * TILE, pl.rng1 + (off + t0), bytes, &sm.bar[stage]);
            bulk_load(sm.in + (stage * PLANES + 6) * TILE, pl.rng2 + (off + t0), bytes, &sm.bar[stage]);
            bulk_load(sm.in + (stage * PLANES + 7) * TILE, pl.rng3 + (off + t0), bytes, &sm.bar[stage]);
        }
    };

    for (uint32_t k = tid; k < g.n_g; k += ES_THREADS) sm.ef[k] = dcp<SH>(dc.efield)[k];
    uint32_t *h = copies ? sm.hist + (uint32_t)(warp % copies) * ef_pad : nullptr;
    float *hf = reinterpret_cast<float *>(sm.acc);  // the large-grid deposit (copies == 0)
    __syncthreads();
    if (tid == 0) {
        for (int s = 0; s < stages; ++s)
            if ((uint32_t)s < ntiles) issue((uint32_t)s, (int)((it0 + (uint32_t)s) % (uint32_t)stages));
    }

    // Scatters the queued colliders sm.queue[0, count), one per thread and
    // round: all the CTA's threads work the independent collision chains
    // together.  The caller has synchronised since the last queue write.
    auto drain = [&](uint32_t count) {
        unsigned long long *ncoll = dcp<SH>(dc.coll);
        if (ncoll && tid == 0) atomicAdd(ncoll, (unsigned long long)count);  // collision events (measurement)
        for (uint32_t q = tid; q < count; q += ES_THREADS) {
            const uint32_t i = off + sm.queue[q];
            const PushResult pr = push_one_c(pl.sx[i], pl.svx[i], sm.ef, factor, dt, inv_dx, n_g, gap, gm);
            const float vy = pl.svy[i], vz = pl.svz[i];
            Xoshiro128p rs{pl.rng0[i], pl.rng1[i], pl.rng2[i], pl.rng3[i]};
            // collides, as before
            const Test t = test_electron(pr.vx, vy, vz, rs, GlobalTable{dcp<SH>(dc.sigma_tot)}, gm);
            uint32_t slot;
            uint32_t *alive = dcp<SH>(dc.alive);
            if (claim_slot(alive, g.capacity, slot)) {
                pl.dx[off + slot] = pr.x;
                collide_electron_t<true>(off, slot, t.idx, pr.vx, vy, vz, rs, dcp<SH>(dc.cs), pl.dx, pl.dvx, pl.dvy,
                                         pl.dvz, pl.ix, pl.ivx, pl.ivy, pl.ivz, alive, dcp<SH>(dc.n_i), gm,
                                         dcp<SH>(dc.dens), dcp<SH>(dc.dens_i));
            } else {
                set_dev_err(gm.dev_err, CUDAPIC_DEVERR_SPAWN_E);
            }
            pl.rng0[i] = rs.s0;
            pl.rng1[i] = rs.s1;
            pl.rng2[i] = rs.s2;
            pl.rng3[i] = rs.s3;
        }
    };

    StepOut<U> prev;
    bool have_prev = false;
    bool ok = true;
    uint32_t pending_base = 0;  // warp 0 lane 31: atomicAdd result of the previous tile
    uint32_t qn = 0;            // queued colliders of the CTA (uniform: every thread counts the same)
    uint32_t tile = 0;
    for (; tile < ntiles; ++tile) {
        const uint32_t k = it0 + tile;  // position in the stage ring
        if (copies && tile != 0 && k % epoch == 0) {  // drain the deposit copies before they can overflow
            __syncthreads();
            dep_drain(sm.hist, copies, ef_pad, sm.acc, g.n_g);
            __syncthreads();
        }
        const int s = (int)(k % (uint32_t)stages);
        const uint32_t parity = (k / (uint32_t)stages) & 1u;
        const uint32_t r3 = k % 3u, p3 = (k + 2u) % 3u;  // buffers of this tile and of the previous one
        // every thread waits for the stage's bulk copies itself (bounded)
        ok = mbar_wait_bounded(&sm.bar[s], parity);
        if (!ok) set_dev_err(gm.dev_err, CUDAPIC_DEVERR_TIMEOUT);

        const uint32_t t0 = beg + tile * TILE;
        const uint32_t cnt = ok ? min((uint32_t)TILE, end - t0) : 0u;
        const uint32_t *b = sm.in + s * PLANES * TILE;
        // The rows of a tile are independent; the work is split into phases
        // over all rows so that the scheduler can interleave them.
        StepOut<U> cur;
        cur.keep = 0;
        uint32_t st[U][4];     // MCC: RNG states after the test draw
        uint32_t keep = 0, may = 0, coll = 0;  // bit u: row u survives / may collide / collides
        // (1) push (Rust-CUDA/src/main.rs:596-620); rows past the tile's end
        //     push a harmless stand-in and are masked
#pragma unroll
        for (int u = 0; u < U; ++u) {
            const uint32_t j = (uint32_t)u * ES_THREADS + tid;
            const bool valid = j < cnt && !slot_dead(__uint_as_float(b[j]));
            live += valid ? 1u : 0u;
            const float x0 = valid ? __uint_as_float(b[j]) : 0.5f * gap;
            const float v0 = valid ? __uint_as_float(b[TILE + j]) : 0.0f;
            const PushResult pr = push_one_c(x0, v0, sm.ef, factor, dt, inv_dx, n_g, gap, gm);
            if (valid && pr.keep) keep |= 1u << u;
            cur.x[u] = pr.x;
            cur.vx[u] = pr.vx;
            if (!MCC) {
                cur.vy[u] = __uint_as_float(b[2 * TILE + j]);
                cur.vz[u] = __uint_as_float(b[3 * TILE + j]);
                if (WALL) {
                    cudapic_wall_counters *wall = dcp<SH>(dc.wall);
                    if (wall) count_wall(wall, true, valid && !pr.keep, pr.x, pr.vx, cur.vy[u], cur.vz[u], gap);
                }
            } else if (WALL) {
                cudapic_wall_counters *wall = dcp<SH>(dc.wall);
                if (wall) count_wall(wall, false, valid && !pr.keep, pr.x, 0.0f, 0.0f, 0.0f, gap);
            }
        }
        if (MCC) {
            // (2) test_electron (mcc.cuh, Rust-CUDA/src/main.rs:992-1012) up to
            //     the certain rejection, which needs no table
#pragma unroll
            for (int u = 0; u < U; ++u) {
                const uint32_t j = (uint32_t)u * ES_THREADS + tid;
                cur.vy[u] = __uint_as_float(b[2 * TILE + j]);
                cur.vz[u] = __uint_as_float(b[3 * TILE + j]);
                Xoshiro128p rs{b[4 * TILE + j], b[5 * TILE + j], b[6 * TILE + j], b[7 * TILE + j]};
                const float v2 = cur.vx[u] * cur.vx[u] + cur.vy[u] * cur.vy[u] + cur.vz[u] * cur.vz[u];
                const float rnd = rs.uniform();
                if ((keep >> u & 1u) && may_collide(rnd, v2, rej_k2)) may |= 1u << u;
                st[u][0] = rs.s0;
                st[u][1] = rs.s1;
                st[u][2] = rs.s2;
                st[u][3] = rs.s3;
            }
            // (3) the exact test where the bound cannot decide (a few per cent)
            if (may) {
#pragma unroll
                for (int u = 0; u < U; ++u) {
                    if (may >> u & 1u) {
                        const uint32_t j = (uint32_t)u * ES_THREADS + tid;
                        Xoshiro128p rs{b[4 * TILE + j], b[5 * TILE + j], b[6 * TILE + j], b[7 * TILE + j]};
                        const float v2 = cur.vx[u] * cur.vx[u] + cur.vy[u] * cur.vy[u] + cur.vz[u] * cur.vz[u];
                        const float velocity = sqrtf(v2);
                        const float rnd = rs.uniform();
                        const uint32_t idx = energy_index(gm.half_me_over_e * v2);
                        if (collision_draw(rnd, __ldg(dcp<SH>(dc.sigma_tot) + idx) * velocity * dt)) coll |= 1u << u;
                    }
                }
            }
        }
        // (4) deposit every survivor; non-colliders (MCC: store their RNG
        //     state) are compacted, colliders are queued
#pragma unroll
        for (int u = 0; u < U; ++u) {
            const uint32_t j = (uint32_t)u * ES_THREADS + tid;
            const bool kept = keep >> u & 1u;
            const bool collide = MCC && (coll >> u & 1u);
            const bool stay = kept && !collide;
            if (kept) {  // CIC of the new position, Rust-CUDA/src/main.rs:377-387
                if (copies) dep_add(h, cur.x[u], g);
                else dep_add_f32(hf, cur.x[u], g);
            }
            if (MCC && stay) {
                const uint32_t i = off + t0 + j;
                pl.rng0[i] = st[u][0];
                pl.rng1[i] = st[u][1];
                pl.rng2[i] = st[u][2];
                pl.rng3[i] = st[u][3];
            }
            const unsigned m = __ballot_sync(0xffffffffu, stay);
            cur.lane_off[u] = __popc(m & lt);
            if (stay) cur.keep |= 1u << u;
            if (lane == 0) sm.offs[r3][u * ES_WARPS + warp] = __popc(m);
            if (MCC) {
                const unsigned cm = __ballot_sync(0xffffffffu, collide);
                if (lane == 0) sm.ccnt[r3][u * ES_WARPS + warp] = __popc(cm);
            }
        }
        // publish the previous tile's base (its atomic had this iteration to return)
        if (have_prev && warp == 0 && lane == 31) sm.s_base[p3] = pending_base;
        // the one block barrier of a tile: counts and previous base visible,
        // stage s consumed; a timeout anywhere ends the loop of every thread
        if (__syncthreads_or(!ok)) {
            ok = false;
            break;
        }
        if (tid == 0) {
            const uint32_t next = tile + (uint32_t)stages;
            if (next < ntiles) issue(next, s);
        }
        if (have_prev) {
            const uint32_t base = sm.s_base[p3];
#pragma unroll
            for (int u = 0; u < U; ++u) {
                if (prev.keep & (1u << u)) {
                    const uint32_t slot = base + sm.offs[p3][u * ES_WARPS + warp] + prev.lane_off[u];
                    if (slot < g.capacity) {
                        pl.dx[off + slot] = prev.x[u];
                        pl.dvx[off + slot] = prev.vx[u];
                        pl.dvy[off + slot] = prev.vy[u];
                        pl.dvz[off + slot] = prev.vz[u];
                    } else {
                        set_dev_err(gm.dev_err, MCC ? CUDAPIC_DEVERR_SPAWN_E : CUDAPIC_DEVERR_SPAWN_I);
                    }
                }
            }
        }
        if (warp == 0) {
            const uint32_t v = lane < NSEG ? sm.offs[r3][lane] : 0u;
            uint32_t incl = v;
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
                const uint32_t t = __shfl_up_sync(0xffffffffu, incl, o);
                if (lane >= o) incl += t;
            }
            if (lane < NSEG) sm.offs[r3][lane] = incl - v;
            if (lane == 31) pending_base = incl ? atomicAdd(dcp<SH>(dc.alive), incl) : 0u;
        }
        prev = cur;
        have_prev = true;
        if (MCC) {
            // queue this tile's colliders behind the earlier ones: every warp
            // scans the (row, warp) counts, which the tile barrier made visible
            // and which stay until the tile after next
            const uint32_t c = lane < NSEG ? sm.ccnt[r3][lane] : 0u;
            uint32_t cincl = c;
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
                const uint32_t t = __shfl_up_sync(0xffffffffu, cincl, o);
                if (lane >= o) cincl += t;
            }
            const uint32_t total = __shfl_sync(0xffffffffu, cincl, 31);
#pragma unroll
            for (int u = 0; u < U; ++u) {
                const bool collide = coll >> u & 1u;
                const unsigned cm = __ballot_sync(0xffffffffu, collide);
                const uint32_t seg = (uint32_t)(u * ES_WARPS + warp);
                const uint32_t before = __shfl_sync(0xffffffffu, cincl - c, (int)seg);
                if (collide) sm.queue[qn + before + __popc(cm & lt)] = t0 + (uint32_t)u * ES_THREADS + tid;
            }
            qn += total;
            if (qn >= (uint32_t)S::DRAIN_AT) {  // uniform: every thread holds the same qn
                __syncthreads();
                drain(qn);
                qn = 0;
            }
        }
    }
    const uint32_t lb = (it0 + tile + 2u) % 3u;  // buffers of the last tile with survivors held in registers
    if (have_prev && warp == 0 && lane == 31) sm.s_base[lb] = pending_base;
    __syncthreads();
    if (have_prev) {
        const uint32_t base = sm.s_base[lb];
#pragma unroll
        for (int u = 0; u < U; ++u) {
            if (prev.keep & (1u << u)) {
                const uint32_t slot = base + sm.offs[lb][u * ES_WARPS + warp] + prev.lane_off[u];
                if (slot < g.capacity) {
                    pl.dx[off + slot] = prev.x[u];
                    pl.dvx[off + slot] = prev.vx[u];
                    pl.dvy[off + slot] = prev.vy[u];
                    pl.dvz[off + slot] = prev.vz[u];
                } else {
                    set_dev_err(gm.dev_err, MCC ? CUDAPIC_DEVERR_SPAWN_E : CUDAPIC_DEVERR_SPAWN_I);
                }
            }
        }
    }
    if (MCC && qn) {
        __syncthreads();
        drain(qn);
    }
    __syncthreads();
    if (copies) {
        dep_drain(sm.hist, copies, ef_pad, sm.acc, g.n_g);
        __syncthreads();
        dep_flush(sm.acc, dcp<SH>(dc.dens), gm);  // clears the accumulator
    } else {
        dep_flush_f32(hf, dcp<SH>(dc.dens), gm);  // clears the histogram
    }
    it = it0 + tile;
    return ok;
}

}  // namespace cudapic
