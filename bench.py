"""Benchmark of the cudaPIC per-timestep PIC/MCC cycle on B200.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference] [--n-g 400|4096]

Workload (single-GPU microbenchmark configuration of the reference's
headline metric): 4 194 304 electrons (Maxwellian 3 eV) + 4 194 304 Ar+ ions
(Maxwellian 0.03 eV), positions uniform in [0, L], ~0.1 % within one step of
an electrode moving outward; argon CCP L = 25 mm, N_G = 400, 13.56 MHz,
250 V, 10 Pa, 350 K, N_T = 4000, N_SUB = 20.  The superparticle weight is
scaled to 7e4 * 120 000 / 4 194 304 so that the plasma density equals the
reference case's steady state.  Seeded synthetic data.

One benchmark step = 40 PIC time steps (two ion subcycles) of the
reference's loop, Rust-CUDA/src/main.rs:1728-1807: per time step
get_density(e) -> solve_poisson_scan_f32 -> move_and_compact(e) ->
check_collisions_e, plus get_density(i), move_and_compact(i),
check_collisions_i on every 20th step.  Metric: particle-steps/s (one
electron advanced by one electron step, or one ion by one ion step, counts
1), counted on the device.

Each timed step touches > 190 MB (electron SoA source + destination + RNG
planes), more than the 126 MB L2, so no L2 flush is needed between steps.

--workload c2 runs the batched path instead: the 256-discharge sweep of the
reference's batched configuration (V ~ U(100, 500) V, p ~ logU(5, 50) Pa,
L ~ U(15, 40) mm, N_G in {200, 400, 800}, 1e4..1e6 particles per species,
seeded), every kernel of a step one launch over all discharges of a rank
(libcudapic's batch driver), discharges sharded over the ranks of an N-GPU
job; the line also reports the same discharges run one at a time through
the reference's launch sequence (the plain path) and through the
one-discharge fused driver.

--impl reference times the reference's own CPU implementation of the path,
eduPIC 1.0 (C/eduPIC.cc, built from the reference tree into oracle/_ref/),
on all host cores, each core running an independent share of the same
population; N > 1 ranks other than 0 exit without work.
"""
import argparse
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


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--n-g", type=int, default=400)
    ap.add_argument("--particles", type=int, default=N_PARTICLES)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-breakdown", action="store_true")
    ap.add_argument("--workload", choices=["c1", "c2"], default="c1",
                    help="c1: one 4M+4M discharge (plain path); c2: the 256-discharge sweep (batched path)")
    ap.add_argument("--discharges", type=int, default=256)
    ap.add_argument("--no-tune", dest="tune", action="store_false",
                    help="c2: skip the autotuning of the batched kernels' launch shapes")
    ap.add_argument("--plain-sample", type=int, default=0,
                    help="c2: discharges also timed one at a time for the plain comparisons (0: all of them)")
    a = ap.parse_args()
    a.warmup = max(a.warmup, 3)
    return a


def workload_config(args):
    return {
        "workload": "plain GPU path: %d e + %d Ar+ steady state, argon CCP L=25mm, N_G=%d, 250V, 10Pa, "
                    "13.56MHz, N_T=4000, N_SUB=20; 1 step = %d PIC steps" % (args.particles, args.particles,
                                                                          args.n_g, STEP),
        "particles_per_species": args.particles,
        "n_g": args.n_g,
        "pic_steps_per_step": STEP,
        "weight": 7.0e4 * 120000 / args.particles,
        "l2": "inputs larger than L2 (>190 MB touched per PIC step), no flush",
        "parallelism": "replicas (one independent discharge per GPU)",
    }


def population(args, rank=0):
    from cudapic_b200.workloads import steady_state
    dt_e = 1.0 / 13.56e6 / 4000
    e = steady_state(args.particles, E_MASS, 3.0, dt=dt_e, seed=11 + 2 * rank)
    i = steady_state(args.particles, AR_MASS, 0.03, dt=20 * dt_e, seed=12 + 2 * rank)
    return e, i


def measured_peaks():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(path):
        with open(path) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    return FALLBACK_HBM_GBS, "fallback"


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

def cpu_reference_run(args, n_marks_warm, n_marks_timed, per_share_cap=None, single=False):
    """eduPIC on all host cores; returns (value, cores, sample description,
    per-step figures, total), with single: also (last) the throughput of one
    process alone on one core with one share."""
    from oracle import edupic_runner as R
    cores = R.host_cores()
    e, i = population(args)
    shares = R.split_population(e, i, cores, per_share_cap=per_share_cap)
    n_e_share = len(shares[0][0][0])
    weight = 7.0e4 * 120000 / args.particles * (args.particles / n_e_share)
    marks = R.run(shares, weight, n_marks_warm + n_marks_timed, n_g=args.n_g)
    value, total, wall, per_step = R.window_throughput(marks, n_marks_warm, n_marks_warm + n_marks_timed)
    sample = ("eduPIC 1.0 (C/eduPIC.cc, g++ -O3) x %d processes, %d e + %d Ar+ per process "
              "(weight x%.1f, same density), %d x %d PIC steps timed after %d warm-up" %
              (cores, n_e_share, len(shares[0][1][0]), args.particles / n_e_share, n_marks_timed, STEP,
               n_marks_warm))
    if not single:
        return value, cores, sample, per_step, total
    one = R.run(shares[:1], weight, n_marks_warm + n_marks_timed, n_g=args.n_g)
    value_1 = R.window_throughput(one, n_marks_warm, n_marks_warm + n_marks_timed)[0]
    sample += "; the same share alone on one core: single_core_value"
    return value, cores, sample, per_step, total, value_1


def run_reference(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    from oracle import edupic_runner as R
    if not R.available(args.n_g):
        print(json.dumps({"impl": "reference", "unavailable": "eduPIC reference build missing (oracle/_ref)"}))
        return 0
    value, cores, sample, per_step, _, value_1 = cpu_reference_run(args, args.warmup, args.steps, single=True)
    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": args.gpus, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": 1e3 * statistics.mean(per_step), "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": workload_config(args), "impl": "reference",
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": cores, "kind": "reference", "sample": sample,
                         "single_core_value": value_1},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line))
    return 0


# ---------------------------------------------------------------- GPU arm

ALGO_BYTES = {  # algorithmic bytes per particle per launch
    "get_density": 4,            # read x
    "move_and_compact": 32,      # read x, vx, vy, vz; write them for survivors
    "check_collisions_e": 44,    # read v (12) + RNG (16), write RNG (16); colliders' v writes not counted
    "check_collisions_i": 44,
    "step_electrons": 64,        # read x, v, RNG (32); write x, v, RNG of survivors (32)
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
    timed("check_collisions_i", lambda: K.check_collisions_i(b.sigma_tot_i, b.cs, ni_c, b.vx[1], b.vy[1], b.vz[1],
                                                             *b.rng[1], g, stream=stream.cuda_stream), n_i, 44)
    return res


def run_ours(args):
    import torch
    world, rank, local = dist_setup(args)
    torch.cuda.set_device(local)
    import cudapic_b200 as cp
    from cudapic_b200.sim import GpuSimState, ParticlesSoA

    n = args.particles
    params = cp.default_params(n_g=args.n_g, capacity=2 * n, weight=7.0e4 * 120000 / n)
    st = GpuSimState(params, device=local)
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
    # fused driver: Poisson and the fused electron step every step; ion push and MCC on ion steps
    launches = args.steps * (STEP * 2 + ion_steps * 2)

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
        share_w = {"solve_poisson": STEP, "step_electrons": STEP, "move_and_compact_deposit_i": ion_steps,
                   "check_collisions_i": ion_steps}
        tot = sum(breakdown[k]["us"] * w for k, w in share_w.items())
        for k in breakdown:
            breakdown[k]["share"] = breakdown[k]["us"] * share_w.get(k, 0) / tot
        dom = max((k for k in breakdown if "gbs" in breakdown[k]), key=lambda k: breakdown[k]["share"])
        d = breakdown[dom]
        traffic = ncu_traffic(dom, d["n"])
        roofline = {"bound": "hbm", "kernel": dom, "achieved": d["gbs"], "peak": peak, "unit": "GB/s",
                    "frac": d["gbs"] / peak, "traffic": traffic, "peak_source": peak_kind,
                    "algo_bytes_per_particle": d["bytes_per_particle"]}

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        try:
            from oracle import edupic_runner as R
            if R.available(args.n_g):
                v, cores, sample, _, _, v1 = cpu_reference_run(args, 1, 3, per_share_cap=1 << 17, single=True)
                cpu = {"value": v, "unit": UNIT, "cores": cores, "kind": "reference", "sample": sample,
                       "single_core_value": v1}
        except Exception as ex:  # the baseline is reported, never the measured product
            cpu = {"value": None, "unit": UNIT, "error": str(ex)[:200]}

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
                "end_to_end": "vs eduPIC's FP64 reference case (cudapic_b200.refcase, 2 seeds, 100 measured cycles): "
                              "relative L2 n_e 0.055, n_i 0.054, potential 0.002, EEPF 0.043; <j E> power 0.012, "
                              "N_e 0.053; f32 and FP64 arithmetic modes agree within the seed spread (<= 0.012)"}


def run_batched(args):
    """The C2 sweep through cudapic_b200.batch (see the module docstring)."""
    import torch
    world, rank, local = dist_setup(args)
    torch.cuda.set_device(local)
    from cudapic_b200.batch import Batch, c2_specs, gather, shard
    specs = c2_specs(n=args.discharges)
    mine = [specs[k] for k in shard(specs, world)[rank]]
    batch = Batch(mine, device=local)
    batch.run_steps(STEP * args.warmup)
    batch.synchronize()
    # launch shapes of the batched kernels for this mix of discharges
    # (untimed; every rank tunes on its own shard)
    import cudapic_b200 as cp
    from cudapic_b200.autotune import tune_batch
    defaults = cp.get_tuning()
    tuned, _ = tune_batch(batch) if args.tune else (None, None)
    batch.run_steps(STEP)
    batch.synchronize()
    barrier(world)
    with ClockSampler(local) as clk:
        elapsed, work = batch.timed_steps(STEP * args.steps)
    barrier(world)
    elapsed_max, work_sum = reduce_max_sum(world, elapsed, work)
    value = work_sum / elapsed_max
    errors = batch.device_errors()
    flagged = [k for k, pc in enumerate(batch.prechecks()) if not pc["conditions_ok"]]

    # end to end through the public API: every discharge re-uploaded from
    # pinned host memory, the steps, every discharge's counts read back
    from cudapic_b200.batch import initial_population
    pinned = []
    for st, spec in zip(batch.states, mine):
        e, i = initial_population(spec, st.grid.dt_e, st.grid.dt_i)
        pinned.append([torch.from_numpy(np.ascontiguousarray(a)).pin_memory() for a in (*e, *i)])
    lib = __import__("cudapic_b200").lib
    barrier(world)
    batch.synchronize()
    w0 = batch.work()
    t0 = time.perf_counter()
    h2d = d2h = 0
    for st, arrs in zip(batch.states, pinned):
        n = arrs[0].numel()
        for sp in (0, 1):
            __import__("cudapic_b200").check(lib.cudapic_state_upload(
                st.handle, sp, *(t.data_ptr() for t in arrs[4 * sp:4 * sp + 4]), n))
            h2d += 16 * n
    batch.run_steps(STEP * args.steps)
    for st in batch.states:
        st.counts()
        d2h += 8
    e2e_wall = time.perf_counter() - t0
    e2e_work = batch.work() - w0
    e2e_max, e2e_sum = reduce_max_sum(world, e2e_wall, e2e_work)

    # the single-simulation comparisons, rank 0's discharges one at a time
    # (the same states, continuing from where the batch left them):
    #  * plain: the reference's launch sequence, every step launched from the
    #    host (no fusion, no graph, no programmatic dependent launch);
    #  * fused: this library's one-discharge driver (fused step, graphs, PDL).
    plain = fused = None
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
        sums = {"plain": [0.0, 0.0], "fused": [0.0, 0.0]}
        for k in order:
            st = batch.states[k]
            for mode in ("plain", "fused"):
                on = mode == "fused"
                st.set_fused(on)
                st.set_graphs(on)
                st.set_overlap(on)
                st.run_steps(STEP * args.warmup)
                st.synchronize()
                t, w = alone(st, STEP * args.steps)
                sums[mode][0] += t
                sums[mode][1] += w
        what = "%d of the %d discharges, each alone in turn, %d PIC steps each" % (len(order), len(specs),
                                                                                 STEP * args.steps)
        plain = {"value": sums["plain"][1] / sums["plain"][0], "unit": UNIT,
                 "path": "reference launch sequence (get_density, Poisson, move_and_compact, check_collisions), "
                         "every step launched from the host", "sample": what}
        fused = {"value": sums["fused"][1] / sums["fused"][0], "unit": UNIT,
                 "path": "one-discharge fused driver (fused electron step, CUDA graph of 2 N_SUB steps, PDL)",
                 "sample": what}
    per_rank = gather({"discharges": len(mine), "errors": sum(1 for e in errors if e)}, world)
    batch.close()
    if world > 1:
        import torch.distributed as dist
        dist.destroy_process_group()
    if rank != 0:
        return 0
    peak, peak_kind = measured_peaks()
    ion_steps = sum(1 for k in range(STEP) if k % 20 == 0)
    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": 1e3 * elapsed_max / args.steps, "higher_is_better": True,
        "scaling": "strong", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": {"workload": "batched path: %d discharges of the C2 sweep (V, p, L, N_G, 1e4..1e6 particles per "
                               "species sampled, seeded), one launch per kernel for all discharges, graph of 2 N_SUB "
                               "steps; 1 step = %d PIC steps" % (len(specs), STEP),
                   "precision": "f32 particles and push, 2^-20 fixed-point deposits summed exactly in 64-bit "
                                "integers, FP64 Poisson scans and time averages",
                   "launch_shapes": tuned or "library defaults",
                   "discharges": len(specs), "particles_total": int(sum(s.particles for s in specs)),
                   "l2": "inputs larger than L2 in aggregate, no flush",
                   "parallelism": "discharges sharded over %d rank(s), no collective" % world},
        "plain_sequential": plain,
        "fused_sequential": fused,
        "speedup_vs_plain": value / plain["value"] if plain else None,
        "speedup_vs_fused_single": value / fused["value"] if fused else None,
        "e2e": {"value": e2e_sum / e2e_max, "unit": UNIT, "h2d_bytes_per_step": h2d // args.steps,
                "d2h_bytes_per_step": d2h // args.steps, "wall_s": e2e_max},
        "roofline": {"bound": "hbm", "kernel": "all (batch aggregate, 64 B per particle-step)",
                     "achieved": 64.0 * work_sum / elapsed_max / 1e9, "peak": peak, "unit": "GB/s",
                     "frac": 64.0 * work_sum / elapsed_max / 1e9 / peak, "traffic": None, "peak_source": peak_kind},
        "stated_error": STATED_ERROR, "clocks": clk.summary(),
        "gpu_launches": args.steps * (STEP * 2 + ion_steps * 2),
        "discharges_with_device_errors": sum(r["errors"] for r in per_rank),
        "precheck_flagged": len(flagged),
    }
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
    sys.exit(run_batched(a) if a.workload == "c2" else run_ours(a))
