"""Runs against eduPIC's reference case and reports the end-to-end error.

eduPIC (C/eduPIC.cc, FP64) ships a converged reference case
(C/ReferenceCase_RawData: argon, 25 mm, 250 V, 13.56 MHz, 10 Pa, ~107 k
electrons after ~7900 RF cycles).  This module starts discharges near that
steady state -- electrons and ions sampled from the reference's
time-averaged density profiles with 3 eV / 0.03 eV Maxwellians -- lets them
relax, measures a window, and compares with eduPIC's outputs normalised as
eduPIC normalises them:

  * n_e, n_i: cycle-averaged densities (save_density, C/eduPIC.cc:787-798);
  * potential: the XT potential map averaged over the RF period (Fig. 11c);
  * EEPF: save_eepf (:804-818), compared below 15 eV;
  * <j E> electron power density (:1011-1026, the mean of Fig. 11g);
  * the electron count (the mean of the last 100 cycles of Fig. 9).

Errors are relative L2 norms (relative differences for the scalars); each
mode runs two seeds side by side, and their difference is the statistical
noise floor.  Arithmetic modes:

  * ``mixed``: the fused driver -- f32 particles, 2^-20 fixed-point deposits
    summed exactly in 64-bit integers, FP64 Poisson scans and FP64 time
    averages (the default path);
  * ``f32_poisson``: the same with the reference's f32 Poisson scans;
  * ``reference_f32``: the reference's launch sequence with f32 atomic
    deposits and f32 Poisson scans (the arithmetic of the reference's GPU path);
  * ``fp64``: the all-FP64 GPU twin (cudapic_b200.fp64): the reference's
    launch sequence with particles, fields, densities and collisions in double.

    python -m cudapic_b200.refcase --reference DIR [--modes mixed,f32_poisson,reference_f32,fp64]
                                   [--relax 300] [--measure 100] [--cross mixed,fp64]

``--cross a,b`` compares two modes with each other (same model, same starts)
instead of with eduPIC: mixed against fp64 is the f32 path's error against
an FP64 computation of the same model.

DIR holds eduPIC's reference outputs under the names of tests/golden
(edupic_ref_density.txt, edupic_ref_eepf.txt, edupic_ref_xt_means.txt,
edupic_ref_conv_tail.txt).
"""
import json
import os

import numpy as np

E_MASS = 9.10938356e-31
AR_MASS = 6.63352090e-26
E_CHARGE = 1.60217662e-19
DE_EEPF = 0.05
EEPF_BAND_EV = 15.0

MODES = ("mixed", "f32_poisson", "reference_f32", "fp64")


def load_reference(directory):
    """eduPIC's reference-case outputs: density [N_G, 3] (x, n_e, n_i), EEPF
    [2000, 2], RF-period means of the XT maps [N_G, 9] (pot, efield, je, ji,
    heate, heati, meanee, meanei, ioniz), the last 100 cycles of the counts."""
    def f(name):
        return np.loadtxt(os.path.join(directory, name))
    return {"density": f("edupic_ref_density.txt"), "eepf": f("edupic_ref_eepf.txt"),
            "xt_means": f("edupic_ref_xt_means.txt"), "conv_tail": f("edupic_ref_conv_tail.txt")}


def sample_profile(dens, dx, weight, area, mass, t_ev, rng):
    """Superparticles distributed like a nodal density profile (each cell at
    the mean of its nodes, uniform inside), Maxwellian velocities at t_ev."""
    cell = 0.5 * (dens[:-1] + dens[1:])
    n = int(round(cell.sum() * dx * area / weight))
    k = rng.choice(len(cell), size=n, p=cell / cell.sum())
    x = ((k + rng.random(n)) * dx).astype(np.float32)
    s = np.sqrt(t_ev * E_CHARGE / mass)
    v = rng.normal(0.0, s, (3, n)).astype(np.float32)
    return x, v[0], v[1], v[2]


def start_particles(ref, seed, weight=7.0e4, gap=0.025, n_g=400, area=1.0e-4):
    """The start of one seed: electrons, then ions, each (x, vx, vy, vz) f32,
    sampled from the reference profiles with numpy's default_rng(seed).  The
    same arrays start the GPU runs (start_states) and the eduPIC runs of
    tests/golden/make_samestart.py."""
    dx = gap / (n_g - 1)
    rng = np.random.default_rng(seed)
    d = ref["density"]
    e = sample_profile(d[:, 1], dx, weight, area, E_MASS, 3.0, rng)
    i = sample_profile(d[:, 2], dx, weight, area, AR_MASS, 0.03, rng)
    return e, i


def start_states(ref, mode, seeds=(1, 2), capacity=400_000, weight=7.0e4, options=None):
    """One state per seed at the reference parameters, particles from the
    reference profiles, in the arithmetic of `mode`.  options: driver
    switches applied to every state (e.g. {"spawn_collide": True})."""
    import cudapic_b200 as cp
    from cudapic_b200.sim import GpuSimState, ParticlesSoA
    flags = 0
    if mode in ("f32_poisson", "reference_f32"):
        flags |= cp.FLAG_POISSON_F32_SCAN
    if mode == "reference_f32":
        flags |= cp.FLAG_DEPOSIT_F32
    states = []
    try:
        for seed in seeds:
            p = cp.default_params(capacity=capacity, flags=flags, weight=weight)
            st = GpuSimState(p)
            states.append(st)
            if mode == "reference_f32":
                st.set_fused(False)
            for name, on in (options or {}).items():
                getattr(st, "set_" + name)(on)
            e, i = start_particles(ref, seed, p.weight, p.gap, p.n_g, p.electrode_area)
            st.upload_electrons(ParticlesSoA(*e))
            st.upload_ions(ParticlesSoA(*i))
            st.seed(e_master=(0x12345678 + seed, 0x11112222, 0x22223333, 0x33334444),
                    i_master=(0x44445555 + seed, 0x55556666, 0x66667777, 0x77778888))
    except Exception:
        for st in states:
            st.close()
        raise
    return states


def run(states, relax, measure, batched=True):
    """relax cycles, then a measurement window of `measure` cycles; fused
    states step together in one batch (unless batched is False), others one
    after another."""
    from cudapic_b200.sim import GpuBatch
    if batched and all(st.fused for st in states):
        with GpuBatch(states) as b:
            b.run_cycles(relax)
            b.synchronize()
            for st in states:
                st.set_measure(True)
            b.run_cycles(measure)
            b.synchronize()
    else:
        for st in states:
            st.run_cycles(relax)
            st.set_measure(True)
            st.run_cycles(measure)
            st.synchronize()


def outputs(st, measure):
    """A state's measurement window normalised as eduPIC's outputs."""
    steps = measure * st.params.n_t
    ce, ci, eepf = st.download_measurements()
    # the ion density is summed on ion steps only (Rust-CUDA/src/main.rs:1752,
    # averaged over them at :1586); eduPIC sums the held density every step
    ion_steps = steps // st.params.n_sub
    counts = eepf.astype(np.float64)
    energy = (np.arange(len(counts)) + 0.5) * DE_EEPF
    r = st.report()
    return {"ne": ce / steps, "ni": ci / ion_steps, "pot": st.download_xt("pot").mean(axis=1),
            "eepf": counts / (counts.sum() * DE_EEPF) / np.sqrt(energy), "power_e": r["power_e"],
            "count_e": float(st.counts()[0]), "device_error": st.device_error()}


def compare(got, ref):
    """(errors, seed-to-seed spread) of the outputs of two or more seeds
    against the reference: the largest error over the seeds, the spread
    between the first two."""
    band = (np.arange(len(ref["eepf"])) + 0.5) * DE_EEPF < EEPF_BAND_EV
    want = {"ne": ref["density"][:, 1], "ni": ref["density"][:, 2], "pot": ref["xt_means"][:, 0],
            "eepf": ref["eepf"][:, 1], "power_e": float(ref["xt_means"][:, 4].mean()),
            "count_e": float(ref["conv_tail"][:, 1].mean())}

    def rel_l2(a, b):
        return float(np.linalg.norm(a - b) / np.linalg.norm(b))

    errors, spread = {}, {}
    for key in ("ne", "ni", "pot", "eepf", "power_e", "count_e"):
        if key in ("power_e", "count_e"):
            errors[key] = max(abs(g[key] / want[key] - 1.0) for g in got)
            spread[key] = abs(got[0][key] / got[1][key] - 1.0)
        else:
            sel = band if key == "eepf" else slice(None)
            errors[key] = max(rel_l2(g[key][sel], want[key][sel]) for g in got)
            spread[key] = rel_l2(got[0][key][sel], got[1][key][sel])
    return errors, spread


def load_samestart(directory, tag="ss", seeds=(1, 2, 3, 4)):
    """eduPIC's outputs of runs from the same starts as start_states
    (tests/golden/make_samestart.py), one dict per seed, shaped like
    outputs(): n_e, n_i, potential, EEPF, <j E> power and the final electron
    count."""
    out = []
    for s in seeds:
        base = os.path.join(directory, "edupic_%s_s%d" % (tag, s))
        dens = np.loadtxt(base + "_density.txt")
        eepf = np.loadtxt(base + "_eepf.txt")
        xt = np.loadtxt(base + "_xt_means.txt")
        conv = np.loadtxt(base + "_conv.txt")
        out.append({"ne": dens[:, 1], "ni": dens[:, 2], "pot": xt[:, 0], "eepf": eepf[:, 1],
                    "power_e": float(xt[:, 4].mean()), "count_e": float(conv[-1, 1])})
    return out


def compare_samples(got, want):
    """Two independent samples of runs (seeds) from the same starts: per
    quantity, the relative L2 norm (relative difference for the scalars) of
    the difference of the seed means, and its noise -- the same norm of the
    standard error of that difference from the seeds' variances.  Profiles
    are compared over all nodes, the EEPF below EEPF_BAND_EV."""
    band = (np.arange(len(want[0]["eepf"])) + 0.5) * DE_EEPF < EEPF_BAND_EV
    diff, noise = {}, {}
    for key in ("ne", "ni", "pot", "eepf", "power_e", "count_e"):
        G = np.array([g[key] for g in got], np.float64)
        W = np.array([w[key] for w in want], np.float64)
        d = G.mean(axis=0) - W.mean(axis=0)
        se2 = G.var(axis=0, ddof=1) / len(G) + W.var(axis=0, ddof=1) / len(W)
        ref = W.mean(axis=0)
        if key in ("power_e", "count_e"):
            diff[key] = float(abs(d) / abs(ref))
            noise[key] = float(np.sqrt(se2) / abs(ref))
        else:
            sel = band if key == "eepf" else slice(None)
            diff[key] = float(np.linalg.norm(d[sel]) / np.linalg.norm(ref[sel]))
            noise[key] = float(np.sqrt(se2[sel].sum()) / np.linalg.norm(ref[sel]))
    return diff, noise


def samestart(ref, directory, mode="mixed", tag="ss", seeds=(1, 2, 3, 4), relax=300, measure=100, weight=7.0e4,
              options=None):
    """This library's runs against eduPIC's runs from the same starts."""
    got = mode_outputs(ref, mode, relax, measure, seeds, weight=weight, options=options)
    want = load_samestart(directory, tag, seeds)
    diff, noise = compare_samples(got, want)
    return {"mode": mode, "options": options or {}, "tag": tag, "seeds": list(seeds), "relax_cycles": relax,
            "measured_cycles": measure, "weight": weight, "difference": diff, "noise": noise,
            "device_errors": [g["device_error"] for g in got],
            "gpu_count_e": [g["count_e"] for g in got], "edupic_count_e": [w["count_e"] for w in want]}


def run_fp64(twins, relax, measure):
    """relax, then measure, cycles of all-FP64 twins (each on its state's
    stream, side by side)."""
    for tw in twins:
        tw.run_cycles(relax)
    for tw in twins:
        tw.set_measure(True)
        tw.run_cycles(measure)


def outputs_fp64(tw):
    """A twin's measurement window normalised as eduPIC's outputs."""
    m = tw.measurements()
    counts = m["eepf"].astype(np.float64)
    energy = (np.arange(len(counts)) + 0.5) * DE_EEPF
    return {"ne": m["ne"], "ni": m["ni"], "pot": m["pot"],
            "eepf": counts / (counts.sum() * DE_EEPF) / np.sqrt(energy), "power_e": m["power_e"],
            "count_e": float(m["counts"][0]), "device_error": m["device_error"]}


def mode_outputs(ref, mode, relax=300, measure=100, seeds=(1, 2), weight=7.0e4, options=None, capacity=None):
    """Per seed, the outputs of one arithmetic mode (normalised as eduPIC's).
    options: driver switches (e.g. {"spawn_collide": True}); states with
    switches the batch driver does not take run one after another."""
    from .fp64 import Fp64Discharge
    cap = capacity or int(400_000 * 7.0e4 / weight)
    states = start_states(ref, mode, seeds, capacity=cap, weight=weight, options=options)
    twins = []
    try:
        if mode == "fp64":
            twins = [Fp64Discharge(st) for st in states]
            run_fp64(twins, relax, measure)
            got = [outputs_fp64(tw) for tw in twins]
        else:
            run(states, relax, measure, batched=not options)
            got = [outputs(st, measure) for st in states]
    finally:
        for tw in twins:
            tw.close()
        for st in states:
            st.close()
    return got


def study(ref, mode, relax=300, measure=100, seeds=(1, 2)):
    got = mode_outputs(ref, mode, relax, measure, seeds)
    errors, spread = compare(got, ref)
    return {"mode": mode, "relax_cycles": relax, "measured_cycles": measure, "seeds": list(seeds),
            "errors": errors, "seed_spread": spread, "device_errors": [g["device_error"] for g in got]}


def cross(ref, a="mixed", b="fp64", relax=300, measure=100, seeds=(1, 2), weight=7.0e4):
    """Mode a against mode b of the same model from the same starts: the
    relative L2 (relative difference for the scalars) of the seed means, and
    each mode's seed-to-seed spread (the noise floor of the comparison)."""
    ga = mode_outputs(ref, a, relax, measure, seeds, weight=weight)
    gb = mode_outputs(ref, b, relax, measure, seeds, weight=weight)
    band = (np.arange(len(ref["eepf"])) + 0.5) * DE_EEPF < EEPF_BAND_EV
    diff, spread = {}, {}
    for key in ("ne", "ni", "pot", "eepf", "power_e", "count_e"):
        ma = np.mean([g[key] for g in ga], axis=0)
        mb = np.mean([g[key] for g in gb], axis=0)
        if key in ("power_e", "count_e"):
            diff[key] = abs(ma / mb - 1.0)
            spread[key] = [abs(g[0][key] / g[1][key] - 1.0) for g in (ga, gb)]
        else:
            sel = band if key == "eepf" else slice(None)
            diff[key] = float(np.linalg.norm(ma[sel] - mb[sel]) / np.linalg.norm(mb[sel]))
            spread[key] = [float(np.linalg.norm(g[0][key][sel] - g[1][key][sel]) / np.linalg.norm(g[1][key][sel]))
                           for g in (ga, gb)]
    return {"modes": [a, b], "relax_cycles": relax, "measured_cycles": measure, "seeds": list(seeds),
            "weight": weight, "particles_e": [g["count_e"] for g in ga], "difference": diff, "seed_spread": spread,
            "device_errors": [g["device_error"] for g in ga + gb]}


def main(argv=None):
    import argparse
    ap = argparse.ArgumentParser()
    ap.add_argument("--reference", required=True, help="directory of eduPIC's reference-case outputs")
    ap.add_argument("--modes", default=",".join(MODES))
    ap.add_argument("--relax", type=int, default=300)
    ap.add_argument("--measure", type=int, default=100)
    ap.add_argument("--cross", help="two modes a,b compared with each other instead of with eduPIC")
    ap.add_argument("--samestart", metavar="TAG",
                    help="compare with eduPIC's runs from the same starts (fixtures edupic_TAG_s<seed>_*)")
    ap.add_argument("--seeds", default="1,2,3,4")
    ap.add_argument("--weight", type=float, default=7.0e4)
    ap.add_argument("--spawn-collide", action="store_true",
                    help="eduPIC's same-step collisions of new electrons (in-place steps)")
    a = ap.parse_args(argv)
    ref = load_reference(a.reference)
    if a.samestart:
        opts = {"spawn_collide": True} if a.spawn_collide else None
        seeds = tuple(int(v) for v in a.seeds.split(","))
        for mode in a.modes.split(","):
            print(json.dumps(samestart(ref, a.reference, mode, a.samestart, seeds, a.relax, a.measure, a.weight, opts)),
                  flush=True)
        return 0
    if a.cross:
        ma, mb = a.cross.split(",")
        seeds = tuple(int(v) for v in a.seeds.split(","))
        print(json.dumps(cross(ref, ma, mb, a.relax, a.measure, seeds, a.weight)), flush=True)
        return 0
    for mode in a.modes.split(","):
        print(json.dumps(study(ref, mode, a.relax, a.measure)), flush=True)
    return 0


if __name__ == "__main__":
    raise SystemExit(main())
