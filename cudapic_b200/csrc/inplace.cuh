// inplace.cuh -- the in-place electron step, shared by the one-discharge
// kernels (kernels_inplace.cu) and the batched ones (kernels_batch.cu).
//
// The compacting fused step (step.cuh) writes every survivor into the other
// side, so each tile needs a block-wide scan and barrier before its stores.
// The in-place step keeps every electron in its slot instead:
//  * stream pass (inplace_segment): four consecutive slots per thread and
//    round, read with 16-byte loads from the eight SoA planes (x, vx, vy, vz,
//    rng0..3); push (Rust-CUDA/src/main.rs:596-620), electrode absorption,
//    collision test (:992-1012, the certain-rejection bound of step.cuh
//    first), CIC deposit of the new position into the next density
//    (push.cuh, 2^-20 fixed point); x, vx and the RNG state go back to the
//    same slots (vy, vz do not change in the push: 24 B written per electron
//    against 32 B read).  An absorbed electron leaves its slot with
//    x = DEAD_X; later passes skip it.  A collider's record (slot, vx, vy,
//    vz and the RNG state past the test draw) goes to its warp's queue in
//    shared memory and, 32 at a time, to the collider list (one atomicAdd
//    per 32 records, coalesced stores): eight planes of the other sides of
//    both species, which an in-place electron step does not otherwise use,
//    so the list holds one record for every slot (slots < 2^31: bit 31 of
//    the slot word marks an ionization).  The pass also makes the
//    scattering's event draw (the process entries are fetched with the
//    test's total) so that it knows how many draws the scattering takes (7
//    for an ionization, else 3) and writes every slot's final RNG state in
//    its coalesced store;
//  * scatter pass (inplace_scatter): one thread per listed collider reads
//    its record (coalesced, no gather from the slot), continues the RNG
//    stream from the record, scatters (collision_e, :1035-1165) and writes
//    the velocity back to the slot -- three scattered words per collider,
//    not seven; spawned electrons are appended after the live slots,
//    spawned ions to the ion side.
// The stream pass keeps the collision code out of its registers (the
// scattering needs ~110 per thread; the stream pass runs at 64 with four
// CTAs per SM), and no block barrier orders its stores.  The holes are
// closed by the compacting step, which the drivers run every N_SUB steps and
// as the last step of every run, so the particle planes are compact
// whenever a caller can see them.
// Every electron draws from the RNG stream of the slot it occupies, in the
// reference's order (test draw, then the scattering draws), as in the
// compacting fused step.
#pragma once
#include "step.cuh"

namespace cudapic {

constexpr float DEAD_X = -1.0f;     // x of a slot whose electron left through an electrode
constexpr int IP_THREADS = 256;
constexpr int IP_WARPS = IP_THREADS / 32;
constexpr int IP_ROW = 4;           // slots per thread and round (one 16-byte load per plane)
constexpr int IP_ROUND = IP_THREADS * IP_ROW;
constexpr int IP_QREC = 64;         // per-warp collider queue: < 32 left over + one row of a round
constexpr int IP_RECW = 8;          // words per record: slot, vx, vy, vz, rng0..3

// Dynamic shared memory: E[ef_pad] f32, the 64-bit deposit accumulator
// [ef_pad], [copies][ef_pad] fixed-point histograms, the collider records
// [IP_RECW][IP_WARPS][IP_QREC].  copies == 0 selects the large-grid deposit:
// one f32 histogram [ef_pad] in the accumulator's place and no copies (f32
// shared atomics: nothing to drain, and at thousands of nodes the lanes
// rarely meet on one), 8 B per node in all, so that four CTAs per SM still
// fit at N_G = 4096.
__host__ __device__ constexpr size_t inplace_smem_bytes(int copies, uint32_t ef_pad) {
    return (copies ? (size_t)ef_pad * (4 + 8) + (size_t)copies * ef_pad * 4 : (size_t)ef_pad * (4 + 4)) +
           (size_t)IP_RECW * IP_WARPS * IP_QREC * 4;
}

struct InplaceSmem {
    float *ef;
    unsigned long long *acc;
    uint32_t *hist;
    uint32_t *rec;
    __device__ __forceinline__ InplaceSmem(unsigned char *smem, int copies, uint32_t ef_pad) {
        ef = reinterpret_cast<float *>(smem);
        acc = reinterpret_cast<unsigned long long *>(ef + ef_pad);  // the f32 histogram when copies == 0
        hist = copies ? reinterpret_cast<uint32_t *>(acc + ef_pad) : reinterpret_cast<uint32_t *>(ef + 2u * ef_pad);
        rec = hist + (uint32_t)copies * ef_pad;
    }
    // word w of record j of warp `warp`
    __device__ __forceinline__ uint32_t &r(int w, int warp, uint32_t j) const {
        return rec[((uint32_t)w * IP_WARPS + (uint32_t)warp) * IP_QREC + j];
    }
    __device__ __forceinline__ unsigned char *end() const {
        return reinterpret_cast<unsigned char *>(rec + IP_RECW * IP_WARPS * IP_QREC);
    }
};

__device__ __forceinline__ void inplace_smem_init(const InplaceSmem &sm, int copies, uint32_t ef_pad) {
    for (uint32_t k = threadIdx.x; k < (uint32_t)copies * ef_pad; k += IP_THREADS) sm.hist[k] = 0u;
    if (copies == 0) {
        float *hf = reinterpret_cast<float *>(sm.acc);
        for (uint32_t k = threadIdx.x; k < ef_pad; k += IP_THREADS) hf[k] = 0.0f;
        return;
    }
    for (uint32_t k = threadIdx.x; k < ef_pad; k += IP_THREADS) sm.acc[k] = 0ull;
}

// Bulk prefetch of [p, p + bytes) into L2 (16-byte aligned, bytes a
// multiple of 16): no registers, no completion to wait for.
__device__ __forceinline__ void prefetch_l2(const void *p, uint32_t bytes) {
    asm volatile("cp.async.bulk.prefetch.L2.global [%0], %1;" ::"l"(p), "r"(bytes) : "memory");
}

// Prefetches round r's slots [beg + r IP_ROUND, end) of the eight planes
// (from element `off`) into L2; issued by one thread.
__device__ __forceinline__ void prefetch_round(const InplacePlanes &pl, uint32_t off, uint32_t beg, uint32_t end,
                                               uint32_t r) {
    const uint32_t s = beg + r * IP_ROUND;
    if (s >= end) return;
    // slots rounded up to a multiple of 4: within the planes (capacity is one)
    const uint32_t bytes = ((min(end - s, (uint32_t)IP_ROUND) + 3u) & ~3u) * 4u;
    const uint32_t i = off + s;
    prefetch_l2(pl.x + i, bytes);
    prefetch_l2(pl.vx + i, bytes);
    prefetch_l2(pl.vy + i, bytes);
    prefetch_l2(pl.vz + i, bytes);
    prefetch_l2(pl.rng0 + i, bytes);
    prefetch_l2(pl.rng1 + i, bytes);
    prefetch_l2(pl.rng2 + i, bytes);
    prefetch_l2(pl.rng3 + i, bytes);
}

// Moves whole groups of 32 queued records of the calling warp to the list
// (one atomicAdd per call), or all of them with `all`; the rest move to the
// front of the queue.  Every lane calls it with the same qn.
__device__ __forceinline__ void flush_records(const InplaceSmem &sm, uint32_t &qn, bool all, const CollList &list,
                                              uint32_t *count) {
    const int lane = threadIdx.x & 31;
    const int warp = threadIdx.x >> 5;
    const uint32_t n = all ? qn : (qn & ~31u);
    if (n == 0) return;
    uint32_t base = 0;
    if (lane == 0) base = atomicAdd(count, n);
    base = __shfl_sync(0xffffffffu, base, 0);
    // at most one record per slot: the list (capacity entries) cannot overflow
    for (uint32_t k = lane; k < n; k += 32) {
        list.slot[base + k] = sm.r(0, warp, k);
        list.vx[base + k] = __uint_as_float(sm.r(1, warp, k));
        list.vy[base + k] = __uint_as_float(sm.r(2, warp, k));
        list.vz[base + k] = __uint_as_float(sm.r(3, warp, k));
        list.r0[base + k] = sm.r(4, warp, k);
        list.r1[base + k] = sm.r(5, warp, k);
        list.r2[base + k] = sm.r(6, warp, k);
        list.r3[base + k] = sm.r(7, warp, k);
    }
    __syncwarp();
    const uint32_t rest = qn - n;
    uint32_t v[IP_RECW];
#pragma unroll
    for (int w = 0; w < IP_RECW; ++w) v[w] = lane < (int)rest ? sm.r(w, warp, n + lane) : 0u;
    __syncwarp();
    if (lane < (int)rest) {
#pragma unroll
        for (int w = 0; w < IP_RECW; ++w) sm.r(w, warp, lane) = v[w];
    }
    __syncwarp();
    qn = rest;
}

// The stream pass over slots [beg, end) (discharge-local, beg a multiple of
// 4) of one discharge whose planes start at element `off`.  Every thread of
// the CTA calls it with the same arguments; on entry the histograms and the
// accumulator are zero and the queues empty, and so they are on return (the
// deposits flushed into dc.dens, the colliders into `list` / `count`, both
// relative to the discharge).  The live electrons processed are added to
// `live` (per thread).  pf: rounds prefetched into L2 ahead of their loads
// (0: none), so that the CTA's next loads are in flight while it computes.
// SH: dc lives in shared memory; WALL: compile the electrode counters in.
template <bool SH, bool WALL>
__device__ __forceinline__ void inplace_segment(const InplacePlanes &pl, const StepDisc &dc, const cudapic_grid &g,
                                                const cudapic_grid &gm, uint32_t off, uint32_t beg, uint32_t end,
                                                const InplaceSmem &sm, int copies, uint32_t ef_pad, uint32_t epoch,
                                                const CollList &list, uint32_t *count, uint32_t &live,
                                                uint32_t pf) {
    const int tid = threadIdx.x;
    const int warp = tid >> 5;
    const unsigned lt = lanemask_lt();
    const float factor = dc.factor, dt = dc.dt, sigma_max = dc.sigma_max;
    const float rej_k2 = sigma_max * dt * (sigma_max * dt) * 1.0001f;  // may_collide's bound
    const float inv_dx = g.inv_dx, gap = g.gap;
    const uint32_t n_g = g.n_g;
    for (uint32_t k = tid; k < n_g; k += IP_THREADS) sm.ef[k] = dcp<SH>(dc.efield)[k];
    const bool f32dep = copies == 0;  // the large-grid deposit
    uint32_t *h = f32dep ? nullptr : sm.hist + (uint32_t)(warp % copies) * ef_pad;
    float *hf = reinterpret_cast<float *>(sm.acc);
    uint32_t qn = 0;  // records queued by this warp (uniform across its lanes), < 32 between rounds
    const uint32_t rounds = (end - beg + IP_ROUND - 1) / IP_ROUND;
    if (tid == 0)
        for (uint32_t r = 1; r < pf && r < rounds; ++r) prefetch_round(pl, off, beg, end, r);
    __syncthreads();
    for (uint32_t r = 0; r < rounds; ++r) {
        if (pf && tid == 0 && r + pf < rounds) prefetch_round(pl, off, beg, end, r + pf);
        if (!f32dep && r != 0 && r % epoch == 0) {  // drain the deposit copies before they can overflow
            __syncthreads();
            dep_drain(sm.hist, copies, ef_pad, sm.acc, n_g);
            __syncthreads();
        }
        const uint32_t s0 = beg + (r * IP_THREADS + (uint32_t)tid) * IP_ROW;  // first slot of this thread
        const bool any = s0 < end;
        const uint32_t i0 = off + s0;
        float4 X = make_float4(0.f, 0.f, 0.f, 0.f), VX = X, VY = X, VZ = X;
        uint4 R0 = make_uint4(0u, 0u, 0u, 0u), R1 = R0, R2 = R0, R3 = R0;
        if (any) {
            X = *reinterpret_cast<const float4 *>(pl.x + i0);
            VX = *reinterpret_cast<const float4 *>(pl.vx + i0);
            VY = *reinterpret_cast<const float4 *>(pl.vy + i0);
            VZ = *reinterpret_cast<const float4 *>(pl.vz + i0);
            R0 = *reinterpret_cast<const uint4 *>(pl.rng0 + i0);
            R1 = *reinterpret_cast<const uint4 *>(pl.rng1 + i0);
            R2 = *reinterpret_cast<const uint4 *>(pl.rng2 + i0);
            R3 = *reinterpret_cast<const uint4 *>(pl.rng3 + i0);
        }
        float x[IP_ROW] = {X.x, X.y, X.z, X.w};
        float vx[IP_ROW] = {VX.x, VX.y, VX.z, VX.w};
        const float vy[IP_ROW] = {VY.x, VY.y, VY.z, VY.w};
        const float vz[IP_ROW] = {VZ.x, VZ.y, VZ.z, VZ.w};
        uint32_t s[4][IP_ROW] = {{R0.x, R0.y, R0.z, R0.w}, {R1.x, R1.y, R1.z, R1.w}, {R2.x, R2.y, R2.z, R2.w},
                                 {R3.x, R3.y, R3.z, R3.w}};
        uint32_t kept = 0, coll = 0, ioniz = 0;  // bit u: slot s0 + u survives / collides / ionizes
        // (1) push; dead and past-the-end slots push a harmless stand-in and are masked
#pragma unroll
        for (int u = 0; u < IP_ROW; ++u) {
            const bool valid = s0 + (uint32_t)u < end && !slot_dead(x[u]);
            const PushResult pr = push_one_c(valid ? x[u] : 0.5f * gap, valid ? vx[u] : 0.0f, sm.ef, factor, dt,
                                             inv_dx, n_g, gap, gm);
            if (WALL) {
                cudapic_wall_counters *wall = dcp<SH>(dc.wall);
                if (wall) count_wall(wall, false, valid && !pr.keep, pr.x, 0.0f, 0.0f, 0.0f, gap);
            }
            if (valid) {
                ++live;
                if (pr.keep) {
                    kept |= 1u << u;
                    x[u] = pr.x;
                    vx[u] = pr.vx;
                } else {
                    x[u] = DEAD_X;
                }
            }
        }
        // (2) the collision test's draw and the certain rejection, which needs no table
#pragma unroll
        for (int u = 0; u < IP_ROW; ++u) {
            if (kept >> u & 1u) {
                Xoshiro128p rs{s[0][u], s[1][u], s[2][u], s[3][u]};
                const float v2 = vx[u] * vx[u] + vy[u] * vy[u] + vz[u] * vz[u];
                const float rnd = rs.uniform();
                if (may_collide(rnd, v2, rej_k2)) {
                    // (3) the exact test where the bound cannot decide (a few per cent),
                    //     with the scattering's three process entries fetched beside it
                    const float velocity = sqrtf(v2);
                    const uint32_t idx = energy_index(gm.half_me_over_e * v2);
                    const float *cs = dcp<SH>(dc.cs);
                    const float st = __ldg(dcp<SH>(dc.sigma_tot) + idx);
                    const float c0 = __ldg(cs + idx), c1 = __ldg(cs + CS_RANGES + idx);
                    const float c2 = __ldg(cs + 2 * CS_RANGES + idx);
                    if (collision_draw(rnd, st * velocity * dt)) {
                        coll |= 1u << u;
                        // collision_e's event draw (its first), from a copy of the
                        // state: an ionization takes 7 draws, the other events 3
                        Xoshiro128p re = rs;
                        const float t1 = c0 + c1, t2 = t1 + c2;
                        if (!(re.uniform() < t1 / t2)) ioniz |= 1u << u;
                    }
                }
                s[0][u] = rs.s0;
                s[1][u] = rs.s1;
                s[2][u] = rs.s2;
                s[3][u] = rs.s3;
                // CIC of the new position, Rust-CUDA/src/main.rs:377-387
                if (f32dep) dep_add_f32(hf, x[u], g);
                else dep_add(h, x[u], g);
            }
        }
        if (any) {
            *reinterpret_cast<float4 *>(pl.x + i0) = make_float4(x[0], x[1], x[2], x[3]);
            *reinterpret_cast<float4 *>(pl.vx + i0) = make_float4(vx[0], vx[1], vx[2], vx[3]);
        }
        // (4) queue this round's colliders as records (warp-synchronous), a
        //     flush after every row keeps the queue below 64
        if (__ballot_sync(0xffffffffu, coll != 0)) {
#pragma unroll
            for (int u = 0; u < IP_ROW; ++u) {
                const bool c = coll >> u & 1u;
                const unsigned cm = __ballot_sync(0xffffffffu, c);
                if (c) {
                    const uint32_t pos = qn + __popc(cm & lt);
                    sm.r(0, warp, pos) = (s0 + (uint32_t)u) | (ioniz >> u & 1u) << 31;  // bit 31: ionization
                    sm.r(1, warp, pos) = __float_as_uint(vx[u]);
                    sm.r(2, warp, pos) = __float_as_uint(vy[u]);
                    sm.r(3, warp, pos) = __float_as_uint(vz[u]);
                    sm.r(4, warp, pos) = s[0][u];
                    sm.r(5, warp, pos) = s[1][u];
                    sm.r(6, warp, pos) = s[2][u];
                    sm.r(7, warp, pos) = s[3][u];
                }
                qn += __popc(cm);
                __syncwarp();
                if (qn >= 32) flush_records(sm, qn, false, list, count);
            }
        }
        // (5) the RNG state of every slot; a collider's goes past all of its
        //     scattering's draws (the record keeps the state the scattering starts from)
#pragma unroll
        for (int u = 0; u < IP_ROW; ++u) {
            if (coll >> u & 1u) {
                Xoshiro128p rs{s[0][u], s[1][u], s[2][u], s[3][u]};
                rs.next();  // the event draw
                rs.next();
                rs.next();
                if (ioniz >> u & 1u) {  // an ionization's four more
                    rs.next();
                    rs.next();
                    rs.next();
                    rs.next();
                }
                s[0][u] = rs.s0;
                s[1][u] = rs.s1;
                s[2][u] = rs.s2;
                s[3][u] = rs.s3;
            }
        }
        if (any) {
            *reinterpret_cast<uint4 *>(pl.rng0 + i0) = make_uint4(s[0][0], s[0][1], s[0][2], s[0][3]);
            *reinterpret_cast<uint4 *>(pl.rng1 + i0) = make_uint4(s[1][0], s[1][1], s[1][2], s[1][3]);
            *reinterpret_cast<uint4 *>(pl.rng2 + i0) = make_uint4(s[2][0], s[2][1], s[2][2], s[2][3]);
            *reinterpret_cast<uint4 *>(pl.rng3 + i0) = make_uint4(s[3][0], s[3][1], s[3][2], s[3][3]);
        }
    }
    flush_records(sm, qn, true, list, count);
    __syncthreads();
    if (f32dep) {
        dep_flush_f32(hf, dcp<SH>(dc.dens), gm);  // each node cleared by the thread that flushed it
        return;
    }
    dep_drain(sm.hist, copies, ef_pad, sm.acc, n_g);
    __syncthreads();
    dep_flush(sm.acc, dcp<SH>(dc.dens), gm);  // clears the accumulator
}

// The scatter pass for record k of a discharge's collider list (its planes
// at element `off`), the collision code inlined so that the loads of the
// record, the table entries and the slot's position overlap: the recorded
// RNG state (the slot's final state is already written by the stream pass)
// continues past the test draw
// (collision_e, Rust-CUDA/src/main.rs:1035-1165, with the fused step's
// algebraic sines and cosines); the velocity goes back to the slot,
// a spawned electron takes the next slot of n_e, a spawned ion the next slot
// of n_i.
__device__ __forceinline__ void inplace_scatter(const InplacePlanes &pl, const CollList &list, uint32_t off,
                                                uint32_t k, const float *cs, uint32_t *n_e, uint32_t *n_i,
                                                const cudapic_grid &g, float *dens_e, float *dens_i) {
    const uint32_t w = list.slot[off + k];
    const uint32_t i = w & 0x7fffffffu;  // bit 31: the stream pass's event draw said ionization
    const float vxi = list.vx[off + k], vyi = list.vy[off + k], vzi = list.vz[off + k];
    const uint32_t j = off + i;
    Xoshiro128p rs{list.r0[off + k], list.r1[off + k], list.r2[off + k], list.r3[off + k]};
    const float xi = (w >> 31) ? pl.x[j] : 0.0f;  // an ionization's birthplace, fetched beside the table lookups
    const float v2 = vxi * vxi + vyi * vyi + vzi * vzi;
    const uint32_t idx = energy_index(g.half_me_over_e * v2);
    collide_electron_body<true, true>(off, i, idx, vxi, vyi, vzi, rs, cs, pl.x, pl.vx, pl.vy, pl.vz, pl.ix, pl.ivx,
                                      pl.ivy, pl.ivz, n_e, n_i, g, dens_e, dens_i, xi);
}

}  // namespace cudapic
