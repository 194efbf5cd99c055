"""Runs one drop-in kernel on the steady-state population (CUDA-event timed,
L2 flushed before each launch): the target of the committed ncu captures.

    python -m cudapic_b200.microbench --kernel check_collisions_e [--particles N] [--reps 3] [--tuning k=v ...]

Kernels: get_density, solve_poisson, move_and_compact, move_and_compact_deposit,
check_collisions_e, check_collisions_e_deposit, check_collisions_i (and
check_collisions_i_bounded, the drivers' entry given max(sigma_tot_i)) and
step_electrons (the *_deposit variants also deposit the next step's density;
step_electrons is the fused driver's compacting electron kernel,
step_electrons_inplace the stream pass of its in-place step).  Prints one JSON line with the median time, the particle
count and the algorithmic bytes per launch.
"""
import argparse
import json
import statistics

BYTES = {"get_density": 4, "move_and_compact": 32, "move_and_compact_deposit": 32, "check_collisions_e": 44,
         "check_collisions_e_deposit": 44, "check_collisions_i": 44, "check_collisions_i_bounded": 44,
         "solve_poisson": 0, "step_electrons": 64,
         "step_electrons_inplace": 56}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--kernel", required=True, choices=sorted(BYTES))
    ap.add_argument("--particles", type=int, default=1 << 22)
    ap.add_argument("--n-g", type=int, default=400)
    ap.add_argument("--reps", type=int, default=3)
    ap.add_argument("--tuning", nargs="*", default=[], metavar="FIELD=VALUE",
                    help="launch-shape overrides (cudapic_tuning fields) for the timed launches")
    a = ap.parse_args()

    import torch

    import cudapic_b200 as cp
    from cudapic_b200.autotune import make_state
    st = make_state(a.particles, a.n_g)
    stream = torch.cuda.Stream()
    st.set_stream(stream)
    torch.cuda.set_stream(stream)
    K = cp.kernels
    b = st.buffers()
    g = st.grid
    n_e, n_i = st.counts()
    s = stream.cuda_stream

    def u32(v):
        return torch.tensor([v], dtype=torch.int32, device="cuda")

    ne_c, ni_c = u32(n_e), u32(n_i)
    alive_e, alive_i = u32(n_e), u32(n_i)
    dens = torch.zeros(g.n_g, dtype=torch.float32, device="cuda")
    pot = torch.zeros(g.n_g, dtype=torch.float32, device="cuda")
    ef = torch.zeros(g.n_g, dtype=torch.float32, device="cuda")
    alive = u32(0)
    ccount = u32(0)
    sigma_max_i = float(K.init_cross_sections(g.gas_density)[2].max())  # the ion table's largest entry
    fns = {
        "get_density": (lambda: K.get_density(b.x[0], dens, ne_c, g, stream=s), lambda: dens.zero_(), n_e),
        "solve_poisson": (lambda: K.solve_poisson_scan_f32(b.e_density, b.i_density, pot, ef, 250.0, g, stream=s),
                          None, g.n_g),
        "move_and_compact": (lambda: K.move_and_compact(b.efield, b.x[0], b.vx[0], b.vy[0], b.vz[0], b.tmp_x[0],
                                                        b.tmp_vx[0], b.tmp_vy[0], b.tmp_vz[0], alive, ne_c,
                                                        g.factor_e, g.dt_e, g, stream=s), alive.zero_, n_e),
        "check_collisions_e": (lambda: K.check_collisions_e(b.sigma_tot_e, b.cs, ne_c, b.x[0], b.vx[0], b.vy[0],
                                                            b.vz[0], *b.rng[0], b.x[1], b.vx[1], b.vy[1], b.vz[1],
                                                            alive_e, alive_i, g, stream=s),
                               lambda: (alive_e.fill_(n_e), alive_i.fill_(n_i)), n_e),
        "move_and_compact_deposit": (lambda: K.move_and_compact_deposit(
            b.efield, b.x[0], b.vx[0], b.vy[0], b.vz[0], b.tmp_x[0], b.tmp_vx[0], b.tmp_vy[0], b.tmp_vz[0], alive,
            ne_c, g.factor_e, g.dt_e, dens, g, stream=s), lambda: (alive.zero_(), dens.zero_()), n_e),
        "check_collisions_e_deposit": (lambda: K.check_collisions_e_deposit(
            b.sigma_tot_e, b.cs, ne_c, b.x[0], b.vx[0], b.vy[0], b.vz[0], *b.rng[0], b.x[1], b.vx[1], b.vy[1],
            b.vz[1], alive_e, alive_i, dens, pot, g, stream=s), lambda: (alive_e.fill_(n_e), alive_i.fill_(n_i)),
            n_e),
        "step_electrons": (lambda: K.step_electrons(
            b.efield, b.x[0], b.vx[0], b.vy[0], b.vz[0], b.tmp_x[0], b.tmp_vx[0], b.tmp_vy[0], b.tmp_vz[0], *b.rng[0],
            b.sigma_tot_e, b.cs, b.sigma_max_e, b.x[1], b.vx[1], b.vy[1], b.vz[1], alive, ne_c, alive_i, dens, pot, g,
            stream=s), lambda: (alive.zero_(), alive_i.fill_(n_i), dens.zero_()), n_e),
        "check_collisions_i": (lambda: K.check_collisions_i(b.sigma_tot_i, b.cs, ni_c, b.vx[1], b.vy[1], b.vz[1],
                                                            *b.rng[1], g, stream=s), None, n_i),
        "check_collisions_i_bounded": (lambda: K.check_collisions_i(
            b.sigma_tot_i, b.cs, ni_c, b.vx[1], b.vy[1], b.vz[1], *b.rng[1], g, stream=s,
            sigma_max_i=sigma_max_i), None, n_i),
        # the in-place step's stream pass (each launch advances the live planes by one step)
        "step_electrons_inplace": (lambda: K.step_electrons_inplace(
            b.efield, b.x[0], b.vx[0], b.vy[0], b.vz[0], *b.rng[0], b.sigma_tot_e, b.cs, b.sigma_max_e, ne_c,
            (b.tmp_x[0], b.tmp_vx[0], b.tmp_vy[0], b.tmp_vz[0], b.tmp_x[1], b.tmp_vx[1], b.tmp_vy[1], b.tmp_vz[1]),
            ccount, dens, g, stream=s), lambda: (ccount.zero_(), dens.zero_()), n_e),
    }
    fn, pre, n = fns[a.kernel]
    if a.tuning:
        cp.set_tuning(**{k: int(v) for k, v in (f.split("=", 1) for f in a.tuning)})
    from cudapic_b200.timing import L2Flusher, time_launch
    t = time_launch(fn, stream, a.reps, flush=L2Flusher(), pre=pre)
    out = {"kernel": a.kernel, "us": t * 1e6, "n": n, "algo_bytes": BYTES[a.kernel] * n,
           "gbs": BYTES[a.kernel] * n / t / 1e9 if BYTES[a.kernel] else None, "tuning": cp.get_tuning()}
    print(json.dumps(out))
    st.close()


if __name__ == "__main__":
    main()
