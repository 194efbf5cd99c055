"""Autotuner of the kernel launch shapes (cudapic_tuning).

Sweeps, on the live GPU and a given population, the CTA size / CTAs per SM /
warp-private histogram copies / cluster size of get_density, the bulk-copy
pipeline depth and CTAs per SM of move_and_compact (timed with the fused
deposit of the driver step), those of check_collisions_e and those of the
fused electron step; each candidate is timed with CUDA events (median of
`reps` launches, L2 flushed before each launch) and the fastest is kept.

    python -m cudapic_b200.autotune [--particles N] [--n-g 400] [--out tuning.json]

tune_batch() does the same for the batched kernels on a live batch of
discharges (their shapes depend on the mix of grids and particle counts).

The built-in defaults of libcudapic (host.cpp kDefaultTuning) are the
values this tool picks on B200 for the 4 M + 4 M steady-state population.
"""
import argparse
import itertools
import json
import statistics

import numpy as np

E_MASS = 9.10938356e-31
AR_MASS = 6.63352090e-26


def _timer(stream, flush, reps):
    from cudapic_b200.timing import time_launch

    def run(fn, pre=None):
        return time_launch(fn, stream, reps, flush=flush, pre=pre) * 1e6
    return run


def make_state(particles, n_g=400, seed=1):
    import cudapic_b200 as cp
    from cudapic_b200.sim import GpuSimState, ParticlesSoA
    from cudapic_b200.workloads import steady_state
    params = cp.default_params(n_g=n_g, capacity=2 * particles, weight=7.0e4 * 120000 / particles)
    st = GpuSimState(params)
    g = st.grid
    st.upload_electrons(ParticlesSoA(*steady_state(particles, E_MASS, 3.0, dt=g.dt_e, seed=seed)))
    st.upload_ions(ParticlesSoA(*steady_state(particles, AR_MASS, 0.03, dt=g.dt_i, seed=seed + 1)))
    st.seed()
    st.run_steps(40)   # a field, densities and a realistic population
    st.synchronize()
    return st


def tune(st, reps=5, verbose=True):
    """Returns (best tuning dict, {kernel: [(config, us), ...]})."""
    import torch

    import cudapic_b200 as cp
    K = cp.kernels
    stream = torch.cuda.Stream()
    st.set_stream(stream)
    torch.cuda.set_stream(stream)
    from cudapic_b200.timing import L2Flusher
    timed = _timer(stream, L2Flusher(), reps)
    b = st.buffers()
    g = st.grid
    n_e, n_i = st.counts()
    s = stream.cuda_stream

    def u32(v):
        return torch.tensor([v], dtype=torch.int32, device="cuda")

    ne_c = u32(n_e)
    dens = torch.zeros(g.n_g, dtype=torch.float32, device="cuda")
    alive = u32(0)
    alive_e, alive_i = u32(n_e), u32(n_i)
    base = cp.get_tuning()
    results = {"get_density": [], "move_and_compact": [], "check_collisions_e": [], "step_electrons": []}

    def density():
        K.get_density(b.x[0], dens, ne_c, g, stream=s)

    def push():  # the fused driver's push: move_and_compact + deposit of the next density
        K.move_and_compact_deposit(b.efield, b.x[0], b.vx[0], b.vy[0], b.vz[0], b.tmp_x[0], b.tmp_vx[0],
                                   b.tmp_vy[0], b.tmp_vz[0], alive, ne_c, g.factor_e, g.dt_e, dens, g, stream=s)

    def reset_push():
        alive.zero_()
        dens.zero_()

    def mcc():
        K.check_collisions_e(b.sigma_tot_e, b.cs, ne_c, b.x[0], b.vx[0], b.vy[0], b.vz[0], *b.rng[0], b.x[1],
                             b.vx[1], b.vy[1], b.vz[1], alive_e, alive_i, g, stream=s)

    def reset_alive():
        alive_e.fill_(n_e)
        alive_i.fill_(n_i)

    dens_i = torch.zeros(g.n_g, dtype=torch.float32, device="cuda")

    def step_e():  # the fused driver's electron kernel
        K.step_electrons(b.efield, b.x[0], b.vx[0], b.vy[0], b.vz[0], b.tmp_x[0], b.tmp_vx[0], b.tmp_vy[0],
                         b.tmp_vz[0], *b.rng[0], b.sigma_tot_e, b.cs, b.sigma_max_e, b.x[1], b.vx[1], b.vy[1],
                         b.vz[1], alive, ne_c, alive_i, dens, dens_i, g, stream=s)

    def reset_step():
        alive.zero_()
        alive_i.fill_(n_i)
        dens.zero_()

    sweeps = [
        ("get_density", density, None,
         [dict(density_threads=t, density_ctas_per_sm=c, density_copies=k, density_cluster=cl)
          for t, c, k, cl in itertools.product((256, 512, 1024), (1, 2, 4), (2, 4, 8, 16, 32), (1, 2, 4, 8))
          if k <= t // 32]),
        ("move_and_compact", push, reset_push,
         [dict(push_stages=st_, push_ctas_per_sm=c) for st_, c in itertools.product((2, 3, 4, 5, 6), (1, 2, 3, 4))]),
        ("check_collisions_e", mcc, reset_alive,
         [dict(mcc_variant=1)] +
         [dict(mcc_variant=2, mcc_stages=st_, mcc_ctas_per_sm=c) for st_, c in itertools.product((2, 3, 4), (2, 3, 4))]),
        ("step_electrons", step_e, reset_step,
         [dict(step_rows=r, step_stages=st_, step_ctas_per_sm=c)
          for r, st_, c in itertools.product((2, 4), (2, 3, 4, 5, 6), (1, 2, 3, 4))]),
    ]
    best = dict(base)
    for name, fn, pre, configs in sweeps:
        for cfg in configs:
            cp.set_tuning(**{**best, **cfg})
            us = timed(fn, pre)
            results[name].append((cfg, us))
        cfg, us = min(results[name], key=lambda r: r[1])
        best.update(cfg)
        if verbose:
            print("%-20s best %s  %.2f us (worst %.2f us)" % (name, cfg, us, max(r[1] for r in results[name])))
    cp.set_tuning(**best)
    return best, results


# Launch shapes of the batched particle kernels (kernels_batch.cu): the
# in-place electron step's resident CTAs per SM and histogram copies (it runs
# all but one step in N_SUB), and the compacting step's rows per thread and
# resident CTAs per SM.
BATCH_CANDIDATES = [dict(inplace_ctas_per_sm=ic, inplace_copies=ik, step_rows=r, step_stages=2, step_ctas_per_sm=c,
                         density_copies=4)
                    for ic, ik, (r, c) in itertools.product((3, 4), (4, 8), ((4, 2), (2, 3)))]
# the same sweep with every electron step compacting (no in-place steps)
BATCH_CANDIDATES_COMPACTING = [dict(step_rows=r, step_stages=st_, step_ctas_per_sm=c, density_copies=k)
                               for r, st_, c, k in itertools.product((1, 2, 4), (2, 4), (2, 3), (4, 8))]


def tune_batch(batch, candidates=None, rounds=2, verbose=False):
    """Times every candidate shape of the batched particle kernels on a live
    ``cudapic_b200.batch.Batch`` (one captured period of 2 N_SUB steps each,
    after an untimed period that captures the graph with the new shapes),
    `rounds` interleaved passes; keeps and returns the shape with the best
    median particle-steps/s: (best dict, {shape: [rates]})."""
    import cudapic_b200 as cp
    if candidates is None:
        candidates = BATCH_CANDIDATES if batch.batch.inplace else BATCH_CANDIDATES_COMPACTING
    cands = list(candidates)
    period = 2 * batch.states[0].params.n_sub
    rates = {}
    for _ in range(rounds):
        for cand in cands:
            cp.set_tuning(**cand)
            batch.run_steps(period)
            t, w = batch.timed_steps(period)
            key = tuple(sorted(cand.items()))
            rates.setdefault(key, []).append(w / t)
            if verbose:
                print("  batch %s %.2f G particle-steps/s" % (cand, w / t / 1e9), flush=True)
    best = max(rates, key=lambda k: statistics.median(rates[k]))
    cp.set_tuning(**dict(best))
    return dict(best), {str(dict(k)): v for k, v in rates.items()}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--particles", type=int, default=1 << 22)
    ap.add_argument("--n-g", type=int, default=400)
    ap.add_argument("--reps", type=int, default=5)
    ap.add_argument("--out", default=None)
    a = ap.parse_args()
    st = make_state(a.particles, a.n_g)
    best, results = tune(st, reps=a.reps)
    out = {"best": best, "particles": a.particles, "n_g": a.n_g,
           "results": {k: [[c, us] for c, us in v] for k, v in results.items()}}
    print(json.dumps({"best": best}))
    if a.out:
        with open(a.out, "w") as f:
            json.dump(out, f, indent=1)
    st.close()


if __name__ == "__main__":
    main()
