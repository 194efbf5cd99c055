"""Voltage sensitivities of one discharge by a pathwise adjoint
(``cudapic_sens_*`` in include/cudapic.h).

The reference has no differentiation.  This differentiates its step loop
(Rust-CUDA/src/main.rs:1725-1808) in slot form -- the same kernels in the
same order, absorbed particles marked dead instead of compacted, spawns in
the slot order of their parents -- so a run is a deterministic function of
the initial state and the RF amplitude V0, and the derivative is taken with
collision events and random draws frozen:

  * ``forward(V0)``: the window of K steps from the state's snapshot, a
    checkpoint every ``checkpoint_every`` steps; returns the observables
    ``power_e`` (<j E> electron power averaged over the gap, W/m^3,
    C/eduPIC.cc:1011-1026) and ``ion_flux_gnd`` (ion flux to the grounded
    electrode, 1/(m^2 s), as the CIC flux density at the electrode node);
  * ``backward()``: d(observable)/dV0 -- each checkpoint interval recomputed
    with a tape and swept in reverse by the adjoint kernels (push, collision
    Jacobians, spawns, Poisson, deposit gather).  ``horizon`` > 0 restarts
    the adjoint every ``horizon`` steps: the sensitivity with the voltage's
    influence truncated to that horizon.  Over long windows the full
    pathwise derivative of this chaotic particle system grows exponentially
    and is meaningless; the truncated one stays bounded;
  * ``central_difference(dv)``: (J(V0 + dv) - J(V0 - dv)) / 2 dv from the
    same snapshot and RNG streams (common random numbers).

    python -m cudapic_b200.sensitivity [--particles 1000000] [--window 8000]
        [--checkpoint 200] [--horizons 0,200,1000] [--dv 0.5] [--relax-cycles 10]
        [--seeds 1,2,3,4]
"""
import ctypes as C
import json
import time

import numpy as np

from . import check, lib

OBSERVABLES = ("power_e", "ion_flux_gnd")


class VoltageSensitivity:
    """Snapshot of a GpuSimState's particles and RNG streams with the
    sensitivity machinery around it (the state itself is not changed)."""

    def __init__(self, state, window_steps=8000, checkpoint_every=200, horizon=0):
        h = C.c_void_p()
        check(lib.cudapic_sens_create(state.handle, int(window_steps), int(checkpoint_every), int(horizon),
                                      C.byref(h)))
        self._h = h
        self.state = state
        self.window_steps = window_steps
        self.checkpoint_every = checkpoint_every
        self.horizon = horizon
        self.voltage = None

    def close(self):
        if getattr(self, "_h", None):
            lib.cudapic_sens_destroy(self._h)
            self._h = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        self.close()

    def forward(self, voltage):
        o = (C.c_double * 2)()
        check(lib.cudapic_sens_forward(self._h, float(voltage), o))
        self.voltage = float(voltage)
        return dict(zip(OBSERVABLES, o))

    def backward(self):
        g = (C.c_double * 2)()
        check(lib.cudapic_sens_backward(self._h, g))
        return dict(zip(OBSERVABLES, g))

    def info(self):
        c = (C.c_uint32 * 2)()
        err = C.c_uint32()
        nbytes = C.c_uint64()
        check(lib.cudapic_sens_info(self._h, c, C.byref(err), C.byref(nbytes)))
        return {"slots": (c[0], c[1]), "device_error": err.value, "device_bytes": nbytes.value}

    def download(self, species):
        """(x, vx, vy, vz, rng[4, capacity]) of all slots after the last run."""
        cap = self.state.capacity
        planes = [np.empty(cap, np.float32) for _ in range(4)]
        rng = np.empty((4, cap), np.uint32)
        check(lib.cudapic_sens_download(self._h, int(species), *[a.ctypes.data for a in planes], rng.ctypes.data,
                                        cap))
        return planes[0], planes[1], planes[2], planes[3], rng

    def central_difference(self, voltage, dv=0.5):
        """d obs / dV0 by central differences with common random numbers."""
        up = self.forward(voltage + dv)
        dn = self.forward(voltage - dv)
        self.forward(voltage)
        return {k: (up[k] - dn[k]) / (2.0 * dv) for k in OBSERVABLES}


def steady_state(particles=1_000_000, relax_cycles=10, seed=1, reference=None):
    """The reference-case discharge (argon, 25 mm, 250 V, 13.56 MHz, 10 Pa,
    N_G = 400) with about `particles` electrons: both species sampled from
    eduPIC's converged density profiles (the weight scaled to the count),
    relaxed `relax_cycles` RF cycles by the fused driver."""
    import os
    from . import default_params
    from .refcase import E_MASS, AR_MASS, load_reference, sample_profile
    from .sim import GpuSimState, ParticlesSoA
    if reference is None:
        reference = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "tests", "golden")
    ref = load_reference(reference)
    p0 = default_params()
    dx = p0.gap / (p0.n_g - 1)
    d = ref["density"]
    n_ref = 0.5 * (d[:-1, 1] + d[1:, 1]).sum() * dx * p0.electrode_area / p0.weight
    weight = p0.weight * n_ref / particles
    p = default_params(weight=weight, capacity=int(2 * particles * 1.2) // 4 * 4)
    st = GpuSimState(p)
    rng = np.random.default_rng(seed)
    st.upload_electrons(ParticlesSoA(*sample_profile(d[:, 1], dx, weight, p.electrode_area, E_MASS, 3.0, rng)))
    st.upload_ions(ParticlesSoA(*sample_profile(d[:, 2], dx, weight, p.electrode_area, AR_MASS, 0.03, rng)))
    st.seed(e_master=(0x12345678 + seed, 0x11112222, 0x22223333, 0x33334444),
            i_master=(0x44445555 + seed, 0x55556666, 0x66667777, 0x77778888))
    if relax_cycles:
        st.run_cycles(relax_cycles)
    st.synchronize()
    return st


def one_start(particles=1_000_000, window=8000, checkpoint=200, horizons=(0, 200, 1000), dv=0.5, voltage=250.0,
              relax_cycles=10, seed=1):
    """Adjoint sensitivities for each horizon against central differences
    with common random numbers, from one relaxed start, with timings."""
    import torch
    st = steady_state(particles, relax_cycles, seed)
    out = {"seed": seed, "counts": st.counts(), "horizons": []}
    try:
        with VoltageSensitivity(st, window, checkpoint, 0) as s:
            torch.cuda.synchronize()
            t = time.perf_counter()
            out["observables"] = s.forward(voltage)
            out["forward_s"] = time.perf_counter() - t
            out["central_difference"] = s.central_difference(voltage, dv)
            out["device_bytes"] = s.info()["device_bytes"]
        for h in horizons:
            with VoltageSensitivity(st, window, checkpoint, h) as s:
                s.forward(voltage)
                t = time.perf_counter()
                g = s.backward()
                el = time.perf_counter() - t
            rel = {k: abs(g[k] / out["central_difference"][k] - 1.0) if out["central_difference"][k] else None
                   for k in g}
            out["horizons"].append({"horizon": h, "adjoint": g, "backward_s": el, "rel_to_fd": rel})
    finally:
        st.close()
    return out


def mean_and_error(values):
    """(mean, standard error of the mean) of per-start values."""
    a = np.asarray(values, np.float64)
    if a.size < 2:
        return float(a.mean()), float("nan")
    return float(a.mean()), float(a.std(ddof=1) / np.sqrt(a.size))


def study(particles=1_000_000, window=8000, checkpoint=200, horizons=(0, 200, 1000), dv=0.5, voltage=250.0,
          relax_cycles=10, seeds=(1,)):
    """one_start for every seed, and over the starts the mean and standard
    error of the central differences and of each horizon's adjoint (the
    difference of one start is noise-dominated over long windows)."""
    starts = [one_start(particles, window, checkpoint, horizons, dv, voltage, relax_cycles, sd) for sd in seeds]
    out = {"particles": particles, "window_steps": window, "checkpoint_every": checkpoint, "dv": dv,
           "voltage": voltage, "relax_cycles": relax_cycles, "starts": starts, "summary": {}}
    for k in OBSERVABLES:
        sm = {"central_difference": mean_and_error([r["central_difference"][k] for r in starts])}
        for j, h in enumerate(horizons):
            sm["adjoint_h%d" % h] = mean_and_error([r["horizons"][j]["adjoint"][k] for r in starts])
        out["summary"][k] = sm
    return out


def main(argv=None):
    import argparse
    ap = argparse.ArgumentParser()
    ap.add_argument("--particles", type=int, default=1_000_000)
    ap.add_argument("--window", type=int, default=8000)
    ap.add_argument("--checkpoint", type=int, default=200)
    ap.add_argument("--horizons", default="0,200,1000")
    ap.add_argument("--dv", type=float, default=0.5)
    ap.add_argument("--voltage", type=float, default=250.0)
    ap.add_argument("--relax-cycles", type=int, default=10)
    ap.add_argument("--seeds", default="1", help="relaxed starts, e.g. 1,2,3,4: mean and standard error over them")
    a = ap.parse_args(argv)
    r = study(a.particles, a.window, a.checkpoint, [int(h) for h in a.horizons.split(",")], a.dv, a.voltage,
              a.relax_cycles, [int(x) for x in a.seeds.split(",")])
    print(json.dumps(r), flush=True)
    return 0



if __name__ == "__main__":
    raise SystemExit(main())
