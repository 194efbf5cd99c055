"""Benchmark of the cudaPIC per-timestep PIC/MCC cycle on B200.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                    [--workload c2|c1|c0]

Metric: particle-steps/s (one electron advanced by one electron step, or one
ion by one ion step, counts 1), counted on the device.

--workload c2 (default): the configuration the metric "batched+mixed vs
plain GPU path" is quoted on.  256 independent argon CCP discharges,
seeded: V ~ U(100, 500) V, p ~ logU(5, 50) Pa, L ~ U(15, 40) mm,
N_G in {200, 400, 800}, 1e4..1e6 particles per species (Maxwellian 3 eV
electrons, 0.03 eV ions, x ~ U[0, L]); seeded synthetic data.  Every kernel
of a step is one launch over all discharges of a rank (libcudapic's batch
driver), 2 N_SUB steps per captured CUDA graph; discharges are sharded over
the ranks of an N-GPU job with no collective.  One benchmark step = 40 PIC
time steps of every discharge (the reference loop
Rust-CUDA/src/main.rs:1725-1808).  Phases:
  1. untimed: warm-up, autotuning of the batched kernels' launch shapes;
  2. every discharge reset to its initial population (RNG re-seeded), W
     warm-up steps, K steps timed with CUDA events on the batch's stream
     (inputs resident in HBM; ~3.7 GB of electron planes per PIC step, far above
     the 126 MB L2, so no flush);
  3. e2e: every discharge re-uploaded from pinned host memory, K steps, every
     discharge's counts read back, all inside a wall-clock region;
  4. per-kernel device times of 40 uncaptured batched steps (roofline);
  5. the same discharges one at a time, each reset first, W + K steps
     (K timed): (a) the plain path -- the reference's launch sequence,
     every kernel launched from the host each step -- and (b) the
     one-discharge fused driver.  speedup_vs_plain = batched / plain.
A discharge whose device error word is set in any phase (spawns beyond its
capacity) is excluded from every sum and counted in the line.

--workload c1: the fused one-discharge driver on one 4 194 304 + 4 194 304
steady-state discharge (argon CCP, 25 mm, N_G = 400, 250 V, 10 Pa).

--workload c0: the plain eduPIC case, 1000 + 1000 particles at rest, one
initialising RF cycle then 10 RF cycles timed: the fused graph driver, the
reference launch sequence and eduPIC on one core.

--impl reference times the reference's own CPU implementation of the path,
eduPIC 1.0 (C/eduPIC.cc, built from the reference tree into oracle/_ref/),
on the selected workload: c2 a sample of the sweep's discharges stratified
by particle count, one full-size discharge per host core; c1 equal shares of
the 4 M + 4 M population, one per core; c0 the case itself on one core (the
program is single-threaded).  Processes start together behind a barrier;
one reference step is --cpu-step-s seconds of all-core work, the value the
particle-steps all cores did inside the K-step window divided by it.  The
GPU arm's cpu_baseline runs the same function with the same window.  For
N > 1 ranks other than 0 exit without work.
"""
import argparse
import importlib.util
import json
import os
import statistics
import subprocess
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

METRIC = "particle-steps/sec on 1 B200: batched+mixed vs plain GPU path at stated error"
UNIT = "particle-steps/s"
STEP = 40               # PIC time steps per benchmark step (graph period 2 * N_SUB)
N_PARTICLES = 1 << 22
E_MASS = 9.10938356e-31
AR_MASS = 6.63352090e-26
FALLBACK_HBM_GBS = 6650.0
C0_CYCLES = 10


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--workload", choices=["c2", "c1", "c0"], default="c2",
                    help="c2: the 256-discharge sweep (batched path, default); c1: one 4M+4M discharge "
                         "(fused one-discharge driver); c0: the plain eduPIC case")
    ap.add_argument("--n-g", type=int, default=400, help="c1: grid points")
    ap.add_argument("--particles", type=int, default=N_PARTICLES, help="c1: particles per species")
    ap.add_argument("--discharges", type=int, default=256, help="c2: discharges of the sweep")
    ap.add_argument("--capacity-factor", type=float, default=3.0, help="c2: slots per initial particle")
    ap.add_argument("--no-tune", dest="tune", action="store_false",
                    help="c2: skip the autotuning of the batched kernels' launch shapes")
    ap.add_argument("--plain-sample", type=int, default=0,
                    help="c2: discharges also timed one at a time for the plain comparisons (0: all of them)")
    ap.add_argument("--cpu-step-s", type=float, default=1.0,
                    help="seconds of all-core eduPIC work per reference step")
    ap.add_argument("--no-inplace", dest="inplace", action="store_false",
                    help="c1/c2: every electron step compacts (no in-place steps between)")
    ap.add_argument("--no-solve-ahead", dest="solve_ahead", action="store_false",
                    help="c1/c0: a Poisson kernel every step (the in-place steps do not solve the next step's "
                         "field in their scatter pass)")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-breakdown", action="store_true")
    a = ap.parse_args()
    a.warmup = max(a.warmup, 3)
    return a


def load_workloads():
    """cudapic_b200/workloads.py loaded by path: plain numpy, so that the CPU
    reference arm never maps the CUDA library."""
    spec = importlib.util.spec_from_file_location("cudapic_workloads", os.path.join(ROOT, "cudapic_b200",
                                                                                     "workloads.py"))
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


def population(args, rank=0):
    """c1: the 4M + 4M steady-state population."""
    W = load_workloads()
    dt_e = 1.0 / 13.56e6 / 4000
    e = W.steady_state(args.particles, E_MASS, 3.0, dt=dt_e, seed=11 + 2 * rank)
    i = W.steady_state(args.particles, AR_MASS, 0.03, dt=20 * dt_e, seed=12 + 2 * rank)
    return e, i


def measured_peaks():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(path):
        with open(path) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    return FALLBACK_HBM_GBS, "fallback"


def workload_config(args):
    if args.workload == "c2":
        return {"workload": "C2 batched sweep: %d argon CCP discharges (V ~ U(100,500) V, p ~ logU(5,50) Pa, "
                            "L ~ U(15,40) mm, N_G in {200,400,800}, 1e4..1e6 particles per species, seeded); "
                            "1 step = %d PIC steps of every discharge" % (args.discharges, STEP),
                "discharges": args.discharges, "pic_steps_per_step": STEP,
                "l2": "inputs larger than L2 (~3.7 GB of electron planes read and written per PIC step), no flush"}
    if args.workload == "c1":
        return {"workload": "C1 fused one-discharge driver: %d e + %d Ar+ steady state, argon CCP L=25mm, N_G=%d, "
                            "250V, 10Pa, 13.56MHz, N_T=4000, N_SUB=20; 1 step = %d PIC steps"
                            % (args.particles, args.particles, args.n_g, STEP),
                "particles_per_species": args.particles, "n_g": args.n_g, "pic_steps_per_step": STEP,
                "weight": 7.0e4 * 120000 / args.particles,
                "l2": "inputs larger than L2 (>190 MB touched per PIC step), no flush",
                "parallelism": "replicas (one independent discharge per GPU)"}
    return {"workload": "C0 plain eduPIC case: 1000 e + 1000 Ar+ at rest, argon CCP L=25mm, N_G=400, 250V, 10Pa; "
                        "one initialising RF cycle, then %d RF cycles timed (1 step = 1 RF cycle)" % C0_CYCLES,
            "rf_cycles": C0_CYCLES, "l2": "population fits in L2 (launch-bound case)",
            "parallelism": "one discharge"}


# ---------------------------------------------------------------- clocks

class ClockSampler:
    """nvidia-smi clocks and throttle reasons every 20 ms; only the samples
    taken between __enter__ (which returns once the sampler is running) and
    __exit__ -- the timed region -- are summarised."""
    FIELDS = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.hw_slowdown,"
              "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
              "clocks_event_reasons.sw_power_cap")

    def __init__(self, device_index):
        self.dev = device_index
        self.proc = None
        self.lines = []
        self.out = ""

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append((time.perf_counter(), line))

    def __enter__(self):
        import threading
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.dev), "--query-gpu=" + self.FIELDS, "--format=csv,noheader,nounits",
                 "-lms", "20"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except (OSError, FileNotFoundError):
            self.proc = None
            return self
        self.reader = threading.Thread(target=self._read, daemon=True)
        self.reader.start()
        deadline = time.perf_counter() + 5.0
        while not self.lines and time.perf_counter() < deadline and self.proc.poll() is None:
            time.sleep(0.005)
        self.t0 = time.perf_counter()
        return self

    def __exit__(self, *exc):
        if self.proc is None:
            return
        t1 = time.perf_counter() + 0.025  # the sample in flight at the end of the region
        time.sleep(0.03)
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
            self.proc.wait()
        self.reader.join(timeout=5)
        self.out = "".join(line for t, line in self.lines if self.t0 <= t <= t1)

    def summary(self):
        sm, mx, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in (self.out or "").splitlines():
            parts = [p.strip() for p in line.split(",")]
            if len(parts) < 7:
                continue
            try:
                sm.append(float(parts[0]))
                mx.append(float(parts[1]))
            except ValueError:
                continue
            for name, v in zip(names, parts[3:7]):
                if v.lower().startswith("active"):
                    reasons.add(name)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": max(mx), "reasons": sorted(reasons),
                "samples": len(sm)}


# ---------------------------------------------------------------- distributed

def dist_setup(args):
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1 and args.impl == "ours":
        import datetime
        import torch
        import torch.distributed as dist
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
    return world, rank, local


def reduce_max_sum(world, elapsed, work):
    from cudapic_b200.batch import reduce_max_sum as rms
    return rms(world, elapsed, work)


def barrier(world):
    if world > 1:
        import torch.distributed as dist
        dist.barrier()


# ---------------------------------------------------------------- CPU (reference program)

def cpu_jobs(args, cores):
    """The eduPIC processes of the selected workload, and a description."""
    W = load_workloads()
    if args.workload == "c2":
        specs = W.c2_specs(n=args.discharges)
        order = sorted(range(len(specs)), key=lambda k: specs[k].particles)
        n = min(cores, len(specs))
        pick = [order[int((j + 0.5) * len(order) / n)] for j in range(n)]
        jobs = []
        for k in pick:
            s = specs[k]
            e, i = W.initial_population(s)
            jobs.append({"electrons": e, "ions": i, "weight": s.weight, "n_g": s.n_g,
                         "env": {"EDUPIC_VOLTAGE": repr(s.voltage), "EDUPIC_L": repr(s.gap),
                                 "EDUPIC_PRESSURE": repr(s.pressure)}})
        parts = sorted(specs[k].particles for k in pick)
        what = ("%d of the %d sweep discharges (stratified by particle count: %d..%d per species, median %d), "
                "each at full size in its own process" % (n, len(specs), parts[0], parts[-1], parts[len(parts) // 2]))
        return jobs, what
    if args.workload == "c1":
        e, i = population(args)
        jobs = []
        for k in range(cores):
            ek = tuple(np.asarray(a[k::cores]) for a in e)
            ik = tuple(np.asarray(a[k::cores]) for a in i)
            jobs.append({"electrons": ek, "ions": ik, "weight": 7.0e4 * 120000 / len(ek[0]), "n_g": args.n_g})
        what = ("the %d + %d population dealt into %d equal shares (%d e + %d Ar+ each, weight scaled to the same "
                "density), one per process" % (args.particles, args.particles, cores, len(jobs[0]["electrons"][0]),
                                                len(jobs[0]["ions"][0])))
        return jobs, what
    raise ValueError(args.workload)


def cpu_reference(args):
    """eduPIC on all host cores over the common window of the selected
    workload (c2, c1), plus one of its processes alone on one core."""
    from oracle import edupic_runner as R
    cores = R.host_cores()
    jobs, what = cpu_jobs(args, cores)
    warm_s, window_s = args.warmup * args.cpu_step_s, args.steps * args.cpu_step_s
    value, rates, window, per_job = R.run_window(jobs, warm_s, window_s)
    mid = sorted(range(len(jobs)), key=lambda k: len(jobs[k]["electrons"][0]))[len(jobs) // 2]
    one = R.run_window([jobs[mid]], warm_s, min(window_s, 10.0))[0]
    sample = ("eduPIC 1.0 (C/eduPIC.cc, g++ -O3) x %d processes on %d host cores: %s; all started together, "
              "%.0f s warm-up, particle-steps inside a %.0f s window (%d steps of %.1f s); "
              "single_core_value: the median process alone on one core"
              % (len(jobs), cores, what, warm_s, window, args.steps, args.cpu_step_s))
    return {"value": value, "unit": UNIT, "cores": len(jobs), "kind": "reference", "sample": sample,
            "single_core_value": one, "window_s": window}


def edupic_c0():
    """The plain eduPIC case (1000 + 1000 particles at rest) on the reference
    CPU program: the initialising cycle (eduPIC 0), then C0_CYCLES RF cycles
    (eduPIC 10) timed from its marks (set-up excluded)."""
    import shutil
    import tempfile
    from oracle import edupic_runner as R
    exe = os.path.join(R.REF_DIR, "eduPIC")
    d = tempfile.mkdtemp(prefix="edupic_c0_")
    try:
        subprocess.run([exe, "0"], cwd=d, check=True, capture_output=True)
        t0 = time.perf_counter()
        r = subprocess.run([exe, str(C0_CYCLES)], cwd=d, check=True, capture_output=True, text=True)
        wall = time.perf_counter() - t0
        marks = [(int(a), int(b), int(c)) for a, b, c in R._MARK.findall(r.stderr)]
        work = marks[-1][1] - marks[0][1]
        secs = (marks[-1][2] - marks[0][2]) * 1e-9
        return {"value": work / secs, "unit": UNIT, "cores": 1, "kind": "reference",
                "sample": "eduPIC 1.0 on one core: the init cycle from 1000 + 1000 particles at rest, then %d RF "
                          "cycles timed (%d particle-steps, %.2f s; %.2f s with set-up)" % (C0_CYCLES, work, secs,
                                                                                         wall),
                "work": work, "seconds": secs}
    finally:
        shutil.rmtree(d, ignore_errors=True)


def run_reference(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    from oracle import edupic_runner as R
    if not all(R.available(g) for g in (200, 400, 800)) or (args.workload == "c1" and not R.available(args.n_g)):
        print(json.dumps({"impl": "reference", "unavailable": "eduPIC reference build missing (oracle/_ref)"}))
        return 0
    if args.workload == "c0":
        cpu = edupic_c0()
        ms = 1e3 * cpu["seconds"] / C0_CYCLES
        steps, warm = C0_CYCLES, 1
    else:
        cpu = cpu_reference(args)
        ms = 1e3 * cpu["window_s"] / args.steps
        steps, warm = args.steps, args.warmup
    line = {
        "metric": METRIC, "value": cpu["value"], "unit": UNIT, "n_gpus": args.gpus, "steps": steps,
        "warmup": warm, "ms_per_step": ms, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": workload_config(args), "impl": "reference", "cpu_baseline": cpu,
        "e2e": {"value": cpu["value"], "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line))
    return 0


def cpu_baseline(args, rank, world):
    """The reference arm's measurement, on rank 0 of a 1-GPU run only."""
    if rank != 0 or world != 1 or args.no_cpu_baseline:
        return None
    try:
        from oracle import edupic_runner as R
        if not all(R.available(g) for g in (200, 400, 800)):
            return None
        return edupic_c0() if args.workload == "c0" else cpu_reference(args)
    except Exception as ex:  # the baseline is reported, never the measured product
        return {"value": None, "unit": UNIT, "error": str(ex)[:200]}


# ---------------------------------------------------------------- GPU arm: one discharge (c1)

ALGO_BYTES = {  # algorithmic bytes per particle per launch
    "get_density": 4,            # read x
    "move_and_compact": 32,      # read x, vx, vy, vz; write them for survivors
    "check_collisions_e": 44,    # read v (12) + RNG (16), write RNG (16); colliders' v writes not counted
    "check_collisions_i": 44,
    "check_collisions_i_bounded": 44,
    "step_electrons": 64,        # read x, v, RNG (32); write x, v, RNG of survivors (32)
    "step_electrons_inplace": 56,  # read x, v, RNG (32); write x, vx, RNG in place (24)
}


def kernel_breakdown(st, K, reps, flush):
    """Times every drop-in kernel of one PIC step on the state's live buffers
    with CUDA events on the state's stream; L2 flushed before each launch."""
    import torch

    def dev_u32(v):
        return torch.tensor([v], dtype=torch.int32, device="cuda")

    b = st.buffers()
    g = st.grid
    stream = torch.cuda.current_stream()
    n_e, n_i = st.counts()
    res = {}

    from cudapic_b200.timing import time_launch

    def timed(name, fn, n, bytes_per, pre=None):
        t = time_launch(fn, stream, reps, flush=flush, pre=pre)
        d = {"us": t * 1e6, "n": n}
        if bytes_per:
            d["bytes_per_particle"] = bytes_per
            d["algo_bytes"] = bytes_per * n
            d["gbs"] = bytes_per * n / t / 1e9
        res[name] = d

    ne_c, ni_c = dev_u32(n_e), dev_u32(n_i)
    dens = torch.zeros(g.n_g, dtype=torch.float32, device="cuda")
    pot = torch.zeros(g.n_g, dtype=torch.float32, device="cuda")
    ef = torch.zeros(g.n_g, dtype=torch.float32, device="cuda")
    alive = dev_u32(0)
    timed("get_density_e", lambda: K.get_density(b.x[0], dens, ne_c, g, stream=stream.cuda_stream), n_e, 4)
    timed("get_density_i", lambda: K.get_density(b.x[1], dens, ni_c, g, stream=stream.cuda_stream), n_i, 4)
    timed("solve_poisson", lambda: K.solve_poisson_scan_f32(b.e_density, b.i_density, pot, ef, 250.0, g,
                                                            stream=stream.cuda_stream), g.n_g, 0)

    def mac(sp, n_c, factor, dt, dep=None):
        args = (b.efield, b.x[sp], b.vx[sp], b.vy[sp], b.vz[sp], b.tmp_x[sp], b.tmp_vx[sp], b.tmp_vy[sp],
                b.tmp_vz[sp], alive, n_c, factor, dt)
        if dep is None:
            K.move_and_compact(*args, g, stream=stream.cuda_stream)
        else:
            K.move_and_compact_deposit(*args, dep, g, stream=stream.cuda_stream)
    timed("move_and_compact_e", lambda: mac(0, ne_c, g.factor_e, g.dt_e), n_e, 32, pre=alive.zero_)
    timed("move_and_compact_i", lambda: mac(1, ni_c, g.factor_i, g.dt_i), n_i, 32, pre=alive.zero_)
    # the fused driver's kernels: the push also deposits the next step's density
    timed("move_and_compact_deposit_e", lambda: mac(0, ne_c, g.factor_e, g.dt_e, dens), n_e, 32,
          pre=lambda: (alive.zero_(), dens.zero_()))
    timed("move_and_compact_deposit_i", lambda: mac(1, ni_c, g.factor_i, g.dt_i, dens), n_i, 32,
          pre=lambda: (alive.zero_(), dens.zero_()))
    alive_e, alive_i = dev_u32(n_e), dev_u32(n_i)
    dens_i = torch.zeros(g.n_g, dtype=torch.float32, device="cuda")

    def reset_alive():
        alive_e.fill_(n_e)
        alive_i.fill_(n_i)

    def ce():
        K.check_collisions_e(b.sigma_tot_e, b.cs, ne_c, b.x[0], b.vx[0], b.vy[0], b.vz[0], *b.rng[0], b.x[1],
                             b.vx[1], b.vy[1], b.vz[1], alive_e, alive_i, g, stream=stream.cuda_stream)

    def ce_dep():
        K.check_collisions_e_deposit(b.sigma_tot_e, b.cs, ne_c, b.x[0], b.vx[0], b.vy[0], b.vz[0], *b.rng[0],
                                     b.x[1], b.vx[1], b.vy[1], b.vz[1], alive_e, alive_i, dens, dens_i, g,
                                     stream=stream.cuda_stream)
    timed("check_collisions_e", ce, n_e, 44, pre=reset_alive)
    timed("check_collisions_e_deposit", ce_dep, n_e, 44, pre=reset_alive)
    # the fused driver's electron kernel: push + collisions + compaction + deposit
    n_i_c = dev_u32(n_i)

    def step_e():
        K.step_electrons(b.efield, b.x[0], b.vx[0], b.vy[0], b.vz[0], b.tmp_x[0], b.tmp_vx[0], b.tmp_vy[0],
                         b.tmp_vz[0], *b.rng[0], b.sigma_tot_e, b.cs, b.sigma_max_e, b.x[1], b.vx[1], b.vy[1],
                         b.vz[1], alive, ne_c, n_i_c, dens, dens_i, g, stream=stream.cuda_stream)

    def reset_step():
        alive.zero_()
        n_i_c.fill_(n_i)
        dens.zero_()
    timed("step_electrons", step_e, n_e, 64, pre=reset_step)
    # the in-place step's two passes (on the live planes: each launch advances them by one step);
    # the collider records go to the other sides' planes, as in the driver
    rec = (b.tmp_x[0], b.tmp_vx[0], b.tmp_vy[0], b.tmp_vz[0], b.tmp_x[1], b.tmp_vx[1], b.tmp_vy[1], b.tmp_vz[1])
    cnt, ticket = dev_u32(0), dev_u32(0)

    def stream_pass():
        K.step_electrons_inplace(b.efield, b.x[0], b.vx[0], b.vy[0], b.vz[0], *b.rng[0], b.sigma_tot_e, b.cs,
                                 b.sigma_max_e, ne_c, rec, cnt, dens, g, stream=stream.cuda_stream)

    def scatter_pass():
        K.scatter_colliders_e(b.x[0], b.vx[0], b.vy[0], b.vz[0], *b.rng[0], b.cs, rec, cnt, ticket, b.x[1], b.vx[1],
                              b.vy[1], b.vz[1], ne_c, n_i_c, dens, dens_i, g, stream=stream.cuda_stream)
    timed("step_electrons_inplace", stream_pass, n_e, 56, pre=lambda: (cnt.zero_(), ne_c.fill_(n_e), dens.zero_()))
    n_coll = int(cnt.item())
    timed("scatter_colliders_e", scatter_pass, n_coll, 0,
          pre=lambda: (cnt.zero_(), ne_c.fill_(n_e), n_i_c.fill_(n_i), stream_pass()))
    res["scatter_colliders_e"]["colliders_per_step"] = n_coll
    timed("check_collisions_i", lambda: K.check_collisions_i(b.sigma_tot_i, b.cs, ni_c, b.vx[1], b.vy[1], b.vz[1],
                                                             *b.rng[1], g, stream=stream.cuda_stream), n_i, 44)
    # the drivers' ion MCC: the same entry given max(sigma_tot_i), same results
    sigma_max_i = float(K.init_cross_sections(g.gas_density)[2].max())
    timed("check_collisions_i_bounded", lambda: K.check_collisions_i(
        b.sigma_tot_i, b.cs, ni_c, b.vx[1], b.vy[1], b.vz[1], *b.rng[1], g, stream=stream.cuda_stream,
        sigma_max_i=sigma_max_i), n_i, 44)
    return res


def run_one_discharge(args):
    import torch
    world, rank, local = dist_setup(args)
    torch.cuda.set_device(local)
    import cudapic_b200 as cp
    from cudapic_b200.sim import GpuSimState, ParticlesSoA

    n = args.particles
    params = cp.default_params(n_g=args.n_g, capacity=2 * n, weight=7.0e4 * 120000 / n)
    st = GpuSimState(params, device=local)
    st.set_inplace(args.inplace)
    st.set_solve_ahead(args.solve_ahead)
    stream = torch.cuda.Stream()
    st.set_stream(stream)
    (e, i) = population(args, rank)
    st.upload_electrons(ParticlesSoA(*e))
    st.upload_ions(ParticlesSoA(*i))
    st.seed()
    torch.cuda.set_stream(stream)

    # ---------------- device-timed region (inputs resident in HBM)
    st.run_steps(STEP * args.warmup)
    st.synchronize()
    barrier(world)
    w0 = st.work()
    ev0 = torch.cuda.Event(enable_timing=True)
    ev1 = torch.cuda.Event(enable_timing=True)
    with ClockSampler(local) as clk:
        torch.cuda.synchronize()
        ev0.record(stream)
        st.run_steps(STEP * args.steps)
        ev1.record(stream)
        torch.cuda.synchronize()
    barrier(world)
    elapsed = ev0.elapsed_time(ev1) * 1e-3
    work = st.work() - w0
    n_e_end, n_i_end = st.counts()
    dev_err = st.device_error()
    elapsed_max, work_sum = reduce_max_sum(world, elapsed, work)
    value = work_sum / elapsed_max
    ion_steps = sum(1 for k in range(STEP) if k % 20 == 0)
    # fused driver: the electron step (in place: stream + scatter pass, two launches; compacting: one)
    # every step; ion push and MCC on ion steps; a Poisson kernel after every compacting step (the
    # in-place steps' scatter passes solve the next step's field), or every step
    compacting = STEP // 20 if args.inplace else STEP
    poisson = compacting if args.inplace and args.solve_ahead else STEP
    launches = args.steps * (poisson + compacting + 2 * (STEP - compacting) + ion_steps * 2)

    # ---------------- end to end through the C ABI with host buffers
    pinned = {}
    for name, arrs in (("e", e), ("i", i)):
        pinned[name] = []
        for a in arrs:
            t = torch.empty(len(a), dtype=torch.float32, pin_memory=True)
            t.numpy()[:] = a
            pinned[name].append(t)
    out = {name: [torch.empty(params.capacity, dtype=torch.float32, pin_memory=True) for _ in range(4)]
           for name in ("e", "i")}
    lib = cp.lib
    import ctypes as C
    n_out = C.c_uint32()
    w_before = st.work()
    barrier(world)
    torch.cuda.synchronize()
    q0 = torch.cuda.Event(enable_timing=True)
    q1 = torch.cuda.Event(enable_timing=True)
    t_wall = time.perf_counter()
    q0.record(stream)
    h2d = 0
    for sp, name in ((0, "e"), (1, "i")):     # H2D of the step inputs from pinned host memory
        cp.check(lib.cudapic_state_upload(st.handle, sp, *(t.data_ptr() for t in pinned[name]), n))
        h2d += 4 * 4 * n
    d2h = 0
    for _ in range(args.steps):
        st.run_steps(STEP)                    # cudapic_state_run_steps
        st.counts()                           # D2H of the step's result (n_e, n_i)
        d2h += 8
    for sp, name in ((0, "e"), (1, "i")):     # D2H of the final particle state
        cp.check(lib.cudapic_state_download(st.handle, sp, *(t.data_ptr() for t in out[name]), params.capacity,
                                            C.byref(n_out)))
        d2h += 4 * 4 * n_out.value
    q1.record(stream)
    torch.cuda.synchronize()
    e2e_wall = time.perf_counter() - t_wall
    e2e_elapsed = q0.elapsed_time(q1) * 1e-3
    e2e_work = st.work() - w_before
    e2e_elapsed_max, e2e_work_sum = reduce_max_sum(world, e2e_elapsed, e2e_work)
    e2e_value = e2e_work_sum / e2e_elapsed_max

    # ---------------- per-kernel breakdown (rank 0 prints)
    breakdown = None
    roofline = None
    peak, peak_kind = measured_peaks()
    if not args.no_breakdown:
        from cudapic_b200.timing import L2Flusher
        breakdown = kernel_breakdown(st, cp.kernels, reps=7, flush=L2Flusher())
        # launches of each kernel in one bench step of the fused driver (the plain
        # get_density / move_and_compact / check_collisions_e lines are for comparison)
        # the driver's schedule: in place except the step before every N_SUB-th one
        compacting = STEP // 20 if args.inplace else STEP
        # (the solve counts every step: in the scatter pass or in a kernel of its own)
        share_w = {"solve_poisson": STEP, "step_electrons": compacting, "move_and_compact_deposit_i": ion_steps,
                   "check_collisions_i_bounded": ion_steps}
        if args.inplace:
            share_w.update({"step_electrons_inplace": STEP - compacting, "scatter_colliders_e": STEP - compacting})
        tot = sum(breakdown[k]["us"] * w for k, w in share_w.items())
        for k in breakdown:
            breakdown[k]["share"] = breakdown[k]["us"] * share_w.get(k, 0) / tot
        dom = max((k for k in breakdown if "gbs" in breakdown[k]), key=lambda k: breakdown[k]["share"])
        d = breakdown[dom]
        traffic = ncu_traffic(dom, d["n"])
        roofline = {"bound": "hbm", "kernel": dom, "achieved": d["gbs"], "peak": peak, "unit": "GB/s",
                    "frac": d["gbs"] / peak, "traffic": traffic, "peak_source": peak_kind,
                    "algo_bytes_per_particle": d["bytes_per_particle"]}

    cpu = cpu_baseline(args, rank, world)
    st.close()
    if world > 1:
        import torch.distributed as dist
        dist.destroy_process_group()
    if rank != 0:
        return 0
    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": 1e3 * elapsed_max / args.steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": workload_config(args),
        "e2e": {"value": e2e_value, "unit": UNIT, "h2d_bytes_per_step": h2d // args.steps,
                "d2h_bytes_per_step": d2h // args.steps, "wall_s": e2e_wall},
        "roofline": roofline, "cpu_baseline": cpu, "stated_error": STATED_ERROR, "clocks": clk.summary(),
        "gpu_launches": launches,
        "kernels": breakdown, "population_end": [n_e_end, n_i_end], "device_error_bits": dev_err,
    }
    print(json.dumps(line))
    return 0


def ncu_traffic(kernel, n):
    """DRAM bytes per launch of `kernel` from the committed ncu summary,
    scaled to n particles; None without a capture."""
    path = os.path.join(ROOT, "profiles", "ncu_traffic.json")
    if not os.path.exists(path):
        return None
    with open(path) as f:
        d = json.load(f)
    k = d.get(kernel)
    if not k:
        return None
    return k["dram_bytes"] * n / k["n"]


STATED_ERROR = {"kernels": "RNG, push/compaction, collisions bit-exact with the CPU restatement of the reference",
                "deposit": "relative L2 <= 2e-5 vs FP64", "poisson": "relative L2 <= 1e-6 vs FP64 Thomas (FP64 sums)",
                "end_to_end": "vs eduPIC 1.0 (FP64, built from the reference) from the same starting particles, "
                              "4 seeds per side, 300 relaxation + 100 measured RF cycles at the reference case: "
                              "relative differences n_e 0.2-0.5 %, n_i 0.3-0.6 %, potential 0.03 %, EEPF 0.4-0.6 %, "
                              "<j E> power 0.1-0.2 %, final N_e 0.1-0.5 %, within 1-3 standard errors of the seed "
                              "noise; with eduPIC's birth-step collisions of new electrons (spawn_collide) every "
                              "quantity within 1 standard error; FP64 twin and reference f32 launch sequence the same",
                "precision": "1000 RF cycles at ~2e5 particles per species: every cycle-averaged profile of the "
                             "mixed path within 0.3 % relative L2 of the all-FP64 GPU twin (seed spread "
                             "0.3-0.9 %); <j E> power 0.29 %; from the same starts at that size, mixed, FP64 twin and "
                             "reference arithmetic within 0.1-0.6 % of eduPIC after 300 + 100 cycles"}


# ---------------------------------------------------------------- GPU arm: the batched sweep (c2)

def run_batched(args):
    import torch
    world, rank, local = dist_setup(args)
    torch.cuda.set_device(local)
    import cudapic_b200 as cp
    from cudapic_b200.autotune import tune_batch
    from cudapic_b200.batch import Batch, c2_specs, gather, initial_population, shard
    specs = c2_specs(n=args.discharges)
    mine = [specs[k] for k in shard(specs, world)[rank]]
    batch = Batch(mine, device=local, capacity_factor=args.capacity_factor)
    for st in batch.states:
        st.set_inplace(args.inplace)
    flagged = set()

    def note_errors():
        for k, e in enumerate(batch.device_errors()):
            if e:
                flagged.add(k)

    # 1. untimed: warm-up and the launch shapes of the batched kernels for this
    #    mix of discharges (every rank tunes on its own shard)
    batch.run_steps(STEP * args.warmup)
    batch.synchronize()
    defaults = cp.get_tuning()
    tuned, _ = tune_batch(batch) if args.tune else (None, None)

    # the initial populations in pinned host memory: every reset below and the
    # end-to-end phase upload them from there
    pinned = []
    for st, spec in zip(batch.states, mine):
        e, i = initial_population(spec, st.grid.dt_e, st.grid.dt_i)
        pinned.append([torch.from_numpy(np.ascontiguousarray(a)).pin_memory() for a in (*e, *i)])

    # 2. device-timed: from the initial populations, W warm-up steps, K timed
    batch.reset(pinned=pinned)
    batch.run_steps(STEP * args.warmup)
    batch.synchronize()
    barrier(world)
    works0 = batch.works()
    with ClockSampler(local) as clk:
        elapsed, _ = batch.timed_steps(STEP * args.steps)
    barrier(world)
    works_timed = [b - a for a, b in zip(works0, batch.works())]
    note_errors()

    # 3. end to end through the public API: every discharge re-uploaded from
    #    pinned host memory, the steps, every discharge's counts read back
    h2d = 16 * sum(2 * p[0].numel() for p in pinned)
    barrier(world)
    batch.synchronize()
    w0 = batch.works()
    t0 = time.perf_counter()
    batch.reset(pinned=pinned, reseed=False)
    batch.run_steps(STEP * args.steps)
    batch.counts()
    e2e_wall = time.perf_counter() - t0
    works_e2e = [b - a for a, b in zip(w0, batch.works())]
    d2h = 8 * len(batch.states)
    note_errors()

    # 4. per-kernel device times of 40 uncaptured steps (roofline)
    breakdown = None
    if not args.no_breakdown:
        c_before = np.array(batch.counts(), np.float64).sum(axis=0)
        prof = batch.profile_steps(STEP)
        c_after = np.array(batch.counts(), np.float64).sum(axis=0)
        n_e_mean, n_i_mean = 0.5 * (c_before + c_after)
        breakdown = {}
        for k, (ms, n) in prof.items():
            if not n:
                continue
            us = 1e3 * ms / n
            d = {"us": us, "launches": int(n), "share": None}
            per = {"electron_step": (64, n_e_mean), "electron_inplace": (56, n_e_mean), "ion_push": (32, n_i_mean),
                   "ion_collisions": (44, n_i_mean)}
            if k in per:
                b, cnt = per[k]
                d.update({"bytes_per_particle": b, "n": cnt, "algo_bytes": b * cnt, "gbs": b * cnt / (us * 1e3)})
            breakdown[k] = d
        tot = sum(v["us"] * v["launches"] for v in breakdown.values())
        for v in breakdown.values():
            v["share"] = v["us"] * v["launches"] / tot
        note_errors()

    # 5. the single-simulation comparisons, rank 0's discharges one at a time,
    #    each from its initial population
    plain = fused = None
    sums = {"plain": [0.0, []], "fused": [0.0, []]}
    order = []
    if rank == 0:
        order = sorted(range(len(mine)), key=lambda k: mine[k].particles)
        if 0 < args.plain_sample < len(order):
            order = [order[int(j * (len(order) - 1) / max(1, args.plain_sample - 1))] for j in range(args.plain_sample)]
        batch.synchronize()

        def alone(st, k_steps):
            ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            s = torch.cuda.ExternalStream(st.stream)
            w0 = st.work()
            ev0.record(s)
            st.run_steps(k_steps)
            ev1.record(s)
            ev1.synchronize()
            return ev0.elapsed_time(ev1) * 1e-3, st.work() - w0

        cp.set_tuning(**defaults)  # the one-discharge kernels' own shapes
        for k in order:
            st = batch.states[k]
            for mode in ("plain", "fused"):
                on = mode == "fused"
                batch.reset_one(k, pinned[k])
                st.set_fused(on)
                st.set_graphs(on)
                st.set_overlap(on)
                st.run_steps(STEP * args.warmup)
                st.synchronize()
                t, w = alone(st, STEP * args.steps)
                sums[mode][0] += t
                sums[mode][1].append((k, w))
                if st.device_error():
                    flagged.add(k)

    # every sum leaves out the discharges flagged in any phase
    flagged_all = set().union(*gather(sorted(flagged), world)) if world > 1 else flagged
    per_rank_flagged = gather(len(flagged), world)
    work_timed = sum(w for k, w in enumerate(works_timed) if k not in flagged)
    work_e2e = sum(w for k, w in enumerate(works_e2e) if k not in flagged)
    elapsed_max, work_sum = reduce_max_sum(world, elapsed, work_timed)
    e2e_max, e2e_sum = reduce_max_sum(world, e2e_wall, work_e2e)
    value = work_sum / elapsed_max
    if rank == 0:
        what = "%d of the %d discharges, each alone in turn from its initial population, %d warm-up + %d timed " \
               "PIC steps each" % (len(order), len(specs), STEP * args.warmup, STEP * args.steps)
        for mode in ("plain", "fused"):
            w = sum(x for k, x in sums[mode][1] if k not in flagged)
            sums[mode].append(w / sums[mode][0] if sums[mode][0] else None)
        plain = {"value": sums["plain"][2], "unit": UNIT,
                 "path": "reference launch sequence (get_density, Poisson, move_and_compact, check_collisions), "
                         "every step launched from the host", "sample": what}
        fused = {"value": sums["fused"][2], "unit": UNIT,
                 "path": "one-discharge fused driver (fused electron step, CUDA graph of 2 N_SUB steps, PDL)",
                 "sample": what}
    n_clean = sum(1 for k in range(len(mine)) if k not in flagged)
    batch.close()
    cpu = cpu_baseline(args, rank, world)
    if world > 1:
        import torch.distributed as dist
        dist.destroy_process_group()
    if rank != 0:
        return 0
    peak, peak_kind = measured_peaks()
    ion_steps = sum(1 for k in range(STEP) if k % 20 == 0)
    roofline = None
    if breakdown:
        dom = max((k for k in breakdown if "gbs" in breakdown[k]), key=lambda k: breakdown[k]["share"])
        d = breakdown[dom]
        names = {"electron_inplace": ("batch_inplace_kernel (in-place electron step of all discharges, stream pass)",
                                      "batch_electron_inplace"),
                 "electron_step": ("batch_step_kernel<MCC> (compacting fused electron step of all discharges)",
                                   "batch_electron_step")}
        label, key = names.get(dom, (dom, dom))
        roofline = {"bound": "hbm", "kernel": label, "achieved": d["gbs"], "peak": peak, "unit": "GB/s",
                    "frac": d["gbs"] / peak, "traffic": ncu_traffic(key, d["n"]), "peak_source": peak_kind,
                    "algo_bytes_per_particle": d["bytes_per_particle"],
                    "aggregate_gbs_64B": 64.0 * work_sum / elapsed_max / 1e9}
    cfg = workload_config(args)
    cfg.update({"precision": "f32 particles and push, 2^-20 fixed-point deposits summed exactly in 64-bit integers, "
                             "FP64 Poisson scans and time averages",
                "launch_shapes": tuned or "library defaults",
                "particles_total": int(sum(s.particles for s in specs)),
                "capacity_factor": args.capacity_factor,
                "parallelism": "discharges sharded over %d rank(s), no collective" % world})
    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": 1e3 * elapsed_max / args.steps, "higher_is_better": True,
        "scaling": "strong", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": cfg,
        "plain_sequential": plain,
        "fused_sequential": fused,
        "speedup_vs_plain": value / plain["value"] if plain and plain["value"] else None,
        "speedup_vs_fused_single": value / fused["value"] if fused and fused["value"] else None,
        "e2e": {"value": e2e_sum / e2e_max, "unit": UNIT, "h2d_bytes_per_step": h2d // args.steps,
                "d2h_bytes_per_step": d2h // args.steps, "wall_s": e2e_max},
        "roofline": roofline, "kernels": breakdown, "cpu_baseline": cpu,
        "stated_error": STATED_ERROR, "clocks": clk.summary(),
        "gpu_launches": args.steps * (STEP + (STEP // 20) + 2 * (STEP - STEP // 20) + ion_steps * 2
                                      if args.inplace else STEP * 2 + ion_steps * 2),
        "discharges_counted": n_clean if world == 1 else None,
        "discharges_excluded": len(flagged_all),
        "excluded_why": "device error word set in some phase (spawns beyond the capacity of %.1fx the initial "
                        "population); their particle-steps are not counted, their time is" % args.capacity_factor,
        "excluded_per_rank": per_rank_flagged,
    }
    print(json.dumps(line))
    return 0


# ---------------------------------------------------------------- GPU arm: the plain eduPIC case (c0)

def run_c0(args):
    import torch
    world, rank, local = dist_setup(args)
    torch.cuda.set_device(local)
    import cudapic_b200 as cp
    from cudapic_b200.sim import GpuSimState, ParticlesSoA
    W = load_workloads()
    e0 = W.edupic_initial(1000, seed=0)
    i0 = W.edupic_initial(1000, seed=1)
    res = {}
    for mode in ("fused", "plain"):
        st = GpuSimState(capacity=40_000, device=local)
        on = mode == "fused"
        st.set_fused(on)
        st.set_graphs(on)
        st.set_overlap(on)
        st.set_solve_ahead(on and args.solve_ahead)
        st.upload_electrons(ParticlesSoA(*e0))
        st.upload_ions(ParticlesSoA(*i0))
        st.seed()
        st.run_cycles(1)          # the initialising cycle (eduPIC 0), graphs captured
        st.synchronize()
        s = torch.cuda.ExternalStream(st.stream)
        ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        w0 = st.work()
        if on:
            clk = ClockSampler(local)
            clk.__enter__()
        ev0.record(s)
        st.run_cycles(C0_CYCLES)
        ev1.record(s)
        ev1.synchronize()
        if on:
            clk.__exit__(None, None, None)
        t = ev0.elapsed_time(ev1) * 1e-3
        res[mode] = {"seconds": t, "work": st.work() - w0, "counts": st.counts(), "dev_err": st.device_error()}
        if on:
            # end to end: upload from pinned memory, the init cycle and 10 cycles, counts read back per cycle
            pin = [torch.from_numpy(np.ascontiguousarray(a)).pin_memory() for a in (*e0, *i0)]
            st.seed()
            torch.cuda.synchronize()
            w1 = st.work()
            t0 = time.perf_counter()
            for sp in (0, 1):
                cp.check(cp.lib.cudapic_state_upload(st.handle, sp, *(p.data_ptr() for p in pin[4 * sp:4 * sp + 4]),
                                                     1000))
            for _ in range(C0_CYCLES + 1):
                st.run_cycles(1)
                st.counts()
            e2e_t = time.perf_counter() - t0
            res["e2e"] = {"value": (st.work() - w1) / e2e_t, "unit": UNIT, "h2d_bytes_per_step": 2 * 16 * 1000,
                          "d2h_bytes_per_step": 8, "wall_s": e2e_t}
        st.close()
    cpu = cpu_baseline(args, rank, world)
    f, p = res["fused"], res["plain"]
    line = {
        "metric": METRIC, "value": f["work"] / f["seconds"], "unit": UNIT, "n_gpus": 1, "steps": C0_CYCLES,
        "warmup": 1, "ms_per_step": 1e3 * f["seconds"] / C0_CYCLES, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic", "config": workload_config(args),
        "plain_path": {"value": p["work"] / p["seconds"], "unit": UNIT, "seconds": p["seconds"],
                       "path": "reference launch sequence, every kernel launched from the host"},
        "fused_seconds": f["seconds"], "particle_steps": f["work"], "counts_end": f["counts"],
        "e2e": res["e2e"], "cpu_baseline": cpu, "clocks": clk.summary(), "roofline": None,
        # per 40 steps: 2 Poisson kernels (40 with --no-solve-ahead; the other solves run in the scatter
        # passes), 38 in-place steps of two kernels, 2 compacting steps, 2 ion pushes + MCC
        "gpu_launches": C0_CYCLES * (4000 // STEP) * ((2 if args.solve_ahead else STEP) + 2 * (STEP - 2) + 2
                                                      + 2 * 2),
        "device_error_bits": [f["dev_err"], p["dev_err"]],
    }
    if rank == 0:
        print(json.dumps(line))
    return 0


if __name__ == "__main__":
    a = parse()
    if a.workload == "c2":
        # one hardware work queue per stream up to the maximum, so that the
        # discharges' streams do not share (and serialise on) the default 8
        os.environ.setdefault("CUDA_DEVICE_MAX_CONNECTIONS", "32")
    if a.impl == "reference":
        sys.exit(run_reference(a))
    sys.exit({"c2": run_batched, "c1": run_one_discharge, "c0": run_c0}[a.workload](a))
