"""Seeded synthetic inputs of the benchmark and parity configurations.

* ``edupic_initial``  -- the plain eduPIC case: N uniform positions in
  [0, L], zero velocities (C/eduPIC.cc:283-294; the GPU reference draws
  Maxwellian velocities instead, Rust-CUDA/src/main.rs:1361-1376).
* ``steady_state``    -- the single-step microbenchmark population: electrons
  Maxwellian at 3 eV, ions at 0.03 eV, positions uniform in [0, L], about
  0.1 % placed within one step of an electrode moving outward so that they
  are absorbed this step.
* ``field_profile``   -- E(x) = E0 cos(pi x / L) on the grid nodes.
* ``sweep_params``    -- 256 seeded discharge parameter sets (voltage
  U(100, 500) V, pressure logU(5, 50) Pa, gap U(15, 40) mm, N_G in
  {200, 400, 800}, particles per species logU(1e4, 1e6)).
* ``c2_specs`` / ``DischargeSpec`` / ``initial_population`` -- the batched
  sweep's discharges and their seeded starting populations.

Plain numpy: nothing here loads the CUDA library, so CPU-side tools (the
eduPIC baseline runner, fixture scripts) can load this file on its own.
"""
import math
from dataclasses import dataclass

import numpy as np

DT_E_REFERENCE = 1.0 / 13.56e6 / 4000   # electron time step of the 13.56 MHz, N_T = 4000 discharges
N_SUB = 20

E_CHARGE = 1.60217662e-19
E_MASS = 9.10938356e-31
AR_MASS = 6.63352090e-26


def edupic_initial(n, gap=0.025, seed=0):
    rng = np.random.default_rng(seed)
    x = (rng.random(n) * gap).astype(np.float32)
    z = np.zeros(n, np.float32)
    return x, z.copy(), z.copy(), z.copy()


def steady_state(n, mass, temperature_ev, gap=0.025, dt=1.8436578171091445e-11, edge_fraction=1e-3, seed=0):
    """Maxwellian population with `edge_fraction` placed to leave this step."""
    rng = np.random.default_rng(seed)
    sigma = math.sqrt(temperature_ev * E_CHARGE / mass)
    vx = rng.normal(0.0, sigma, n)
    vy = rng.normal(0.0, sigma, n).astype(np.float32)
    vz = rng.normal(0.0, sigma, n).astype(np.float32)
    x = rng.random(n) * gap
    k = int(round(n * edge_fraction))
    if k:
        idx = rng.choice(n, size=k, replace=False)
        left = rng.random(k) < 0.5
        u = rng.random(k)
        speed = np.abs(vx[idx])
        # distance u * |v| dt from the electrode, moving towards it
        x[idx] = np.where(left, u * speed * dt, gap - u * speed * dt)
        vx[idx] = np.where(left, -speed, speed)
    x = np.clip(x, 0.0, gap).astype(np.float32)
    return x, vx.astype(np.float32), vy, vz


def field_profile(n_g, e0=2.0e4):
    xs = np.arange(n_g, dtype=np.float64) / (n_g - 1)
    return (e0 * np.cos(math.pi * xs)).astype(np.float32)


def sweep_params(n_discharges=256, seed=0x5EED):
    rng = np.random.default_rng(seed)
    out = []
    for _ in range(n_discharges):
        out.append({
            "voltage": float(rng.uniform(100.0, 500.0)),
            "pressure": float(math.exp(rng.uniform(math.log(5.0), math.log(50.0)))),
            "gap": float(rng.uniform(0.015, 0.040)),
            "n_g": int(rng.choice([200, 400, 800])),
            "particles": int(round(math.exp(rng.uniform(math.log(1e4), math.log(1e6))))),
        })
    return out


@dataclass
class DischargeSpec:
    """One discharge of a sweep (argon CCP, eduPIC physics)."""
    voltage: float      # RF amplitude [V]
    pressure: float     # [Pa]
    gap: float          # electrode gap [m]
    n_g: int            # grid points
    particles: int      # initial electrons (and ions)
    seed: int

    @property
    def weight(self):
        """Superparticle weight of the reference steady state (7e4 at ~1.2e5
        particles) scaled to the particle count."""
        return 7.0e4 * 120000 / self.particles

    def params(self, capacity_factor=2.0):
        import cudapic_b200 as cp
        cap = int(math.ceil(self.particles * capacity_factor / 4.0)) * 4
        return cp.default_params(voltage=self.voltage, pressure=self.pressure, gap=self.gap, n_g=self.n_g,
                                 capacity=cap, weight=self.weight)


def c2_specs(n=256, seed=0x5EED):
    """The C2 sweep: V ~ U(100, 500) V, p ~ logU(5, 50) Pa, L ~ U(15, 40) mm,
    N_G in {200, 400, 800}, particles per species ~ logU(1e4, 1e6)."""
    rng = np.random.default_rng(seed)
    specs = []
    for k in range(n):
        specs.append(DischargeSpec(
            voltage=float(rng.uniform(100.0, 500.0)),
            pressure=float(math.exp(rng.uniform(math.log(5.0), math.log(50.0)))),
            gap=float(rng.uniform(0.015, 0.040)),
            n_g=int(rng.choice([200, 400, 800])),
            particles=int(round(math.exp(rng.uniform(math.log(1e4), math.log(1e6))))),
            seed=int(seed) * 1000 + k))
    return specs


def initial_population(spec, dt_e=DT_E_REFERENCE, dt_i=N_SUB * DT_E_REFERENCE):
    """Maxwellian electrons (3 eV) and ions (0.03 eV) uniform in the gap."""
    e = steady_state(spec.particles, E_MASS, 3.0, gap=spec.gap, dt=dt_e, seed=spec.seed)
    i = steady_state(spec.particles, AR_MASS, 0.03, gap=spec.gap, dt=dt_i, seed=spec.seed + 1)
    return e, i
