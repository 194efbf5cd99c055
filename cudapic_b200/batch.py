"""Batched discharges: many independent discharges stepped concurrently.

A parameter sweep (the C2 workload: 256 argon CCP discharges with sampled
voltage, pressure, gap, grid and particle count) leaves most of a B200 idle
when its small discharges run one after another: a discharge of 1e4
particles fills a few of the 148 SMs for a few microseconds per step.
``Batch`` gives every discharge its own ``GpuSimState`` and steps them all
through one ``GpuBatch``: each kernel of a step is ONE persistent launch over
the concatenated particles of every discharge (libcudapic's batch driver,
kernels_batch.cu), 2 N_SUB steps per captured CUDA graph.  Throughput is
timed on the device with events on the batch's stream.

``shard`` spreads discharges over the ranks of a multi-GPU job (no
collective during the run: the discharges are independent); ``gather``
collects per-rank results on every rank through ``torch.distributed``.

    python -m cudapic_b200.batch [--discharges 256 | --one-discharge N] [--steps 40]
                                 [--tune | --rows R --ctas C --stages S --copies K]
                                 [--pressure P] [--voltage V]

times a batch (the C2 sweep, optionally with every discharge at one
pressure or voltage, or one argon CCP of N particles per species at the
reference parameters) and prints one JSON line: the target of the
committed ncu captures of the batched kernels.
"""
from dataclasses import asdict

from .workloads import DischargeSpec, c2_specs, initial_population  # noqa: F401  (the sweep's definitions)


def shard(specs, world):
    """Indices of the discharges of each rank: largest first onto the rank
    with the fewest particles so far (balanced by particle count)."""
    order = sorted(range(len(specs)), key=lambda k: -specs[k].particles)
    load = [0] * world
    parts = [[] for _ in range(world)]
    for k in order:
        r = min(range(world), key=lambda q: (load[q], q))
        parts[r].append(k)
        load[r] += specs[k].particles
    return [sorted(p) for p in parts]


def gather(local, world):
    """All ranks' results (any picklable object) on every rank, rank order."""
    if world == 1:
        return [local]
    import torch.distributed as dist
    out = [None] * world
    dist.all_gather_object(out, local)
    return out


def reduce_max_sum(world, elapsed, work):
    """(max over ranks of elapsed, sum over ranks of work): the job's time and
    its total work.  Tensors live on the GPU for NCCL, on the host for gloo."""
    if world == 1:
        return elapsed, work
    import torch
    import torch.distributed as dist
    dev = "cuda" if dist.get_backend() == "nccl" else "cpu"
    t = torch.tensor([elapsed], dtype=torch.float64, device=dev)
    w = torch.tensor([float(work)], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    dist.all_reduce(w, op=dist.ReduceOp.SUM)
    return t.item(), w.item()


class Batch:
    """Every discharge of ``specs`` as a GpuSimState, stepped by one GpuBatch."""

    def __init__(self, specs, device=0, capacity_factor=2.0):
        from cudapic_b200.sim import GpuBatch, GpuSimState, ParticlesSoA
        self.specs = list(specs)
        self.states = []
        self.batch = None
        try:
            for spec in self.specs:
                st = GpuSimState(spec.params(capacity_factor), device=device)
                self.states.append(st)
                g = st.grid
                e, i = initial_population(spec, g.dt_e, g.dt_i)
                st.upload_electrons(ParticlesSoA(*e))
                st.upload_ions(ParticlesSoA(*i))
                self._seed(st, spec)
            self.batch = GpuBatch(self.states)
        except Exception:
            self.close()
            raise

    def run_steps(self, n_steps):
        """Enqueues n_steps of every discharge (asynchronous)."""
        self.batch.run_steps(n_steps)

    def run_cycles(self, n_cycles):
        self.batch.run_cycles(n_cycles)

    def synchronize(self):
        self.batch.synchronize()
        for st in self.states:
            st.synchronize()

    def work(self):
        return sum(st.work() for st in self.states)

    def timed_steps(self, n_steps):
        """Runs n_steps on every discharge; returns (device seconds, particle-steps)."""
        import torch
        w0 = self.work()
        self.synchronize()
        s = torch.cuda.ExternalStream(self.batch.stream)
        start = torch.cuda.Event(enable_timing=True)
        end = torch.cuda.Event(enable_timing=True)
        with torch.cuda.stream(s):
            # a bounded sleep holds the start while the host enqueues, so the
            # device clock measures the batch, not the host
            torch.cuda._sleep(int(5e7))
        start.record(s)
        self.run_steps(n_steps)
        end.record(s)
        end.synchronize()
        return start.elapsed_time(end) * 1e-3, self.work() - w0

    def profile_steps(self, n_steps):
        """Per-kernel device time of n_steps uncaptured batched steps."""
        return self.batch.profile_steps(n_steps)

    def reset(self, pinned=None, reseed=True):
        """Every discharge back to its initial population (from `pinned`
        host tensors when given: per discharge e x, vx, vy, vz, i x, vx, vy,
        vz), RNG streams re-seeded unless reseed is False, device error words
        cleared; enqueued on each state's stream."""
        for k in range(len(self.states)):
            self.reset_one(k, None if pinned is None else pinned[k], reseed)

    def reset_one(self, k, pinned=None, reseed=True):
        import cudapic_b200 as cp
        from cudapic_b200.sim import ParticlesSoA
        st, spec = self.states[k], self.specs[k]
        if pinned is None:
            e, i = initial_population(spec, st.grid.dt_e, st.grid.dt_i)
            st.upload_electrons(ParticlesSoA(*e))
            st.upload_ions(ParticlesSoA(*i))
        else:
            n = pinned[0].numel()
            for sp in (0, 1):
                cp.check(cp.lib.cudapic_state_upload(st.handle, sp, *(t.data_ptr() for t in pinned[4 * sp:4 * sp + 4]),
                                                     n))
        if reseed:
            self._seed(st, spec)
        st.clear_device_error()

    @staticmethod
    def _seed(st, spec):
        st.seed(e_master=(0x12345678 ^ spec.seed, 0x11112222, 0x22223333, 0x33334444),
                i_master=(0x44445555 ^ spec.seed, 0x55556666, 0x66667777, 0x77778888))

    def works(self):
        """Particle-steps counted so far, per discharge."""
        return [st.work() for st in self.states]

    def counts(self):
        return [st.counts() for st in self.states]

    def device_errors(self):
        return [st.device_error() for st in self.states]

    def prechecks(self):
        import cudapic_b200 as cp
        return [cp.stability_precheck(st.params) for st in self.states]

    def describe(self):
        return [asdict(s) for s in self.specs]

    def close(self):
        if self.batch is not None:
            self.batch.close()
            self.batch = None
        for st in self.states:
            st.close()
        self.states = []

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()


def main(argv=None):
    import argparse
    import json
    ap = argparse.ArgumentParser()
    ap.add_argument("--discharges", type=int, default=256)
    ap.add_argument("--one-discharge", type=int, default=0,
                    help="one discharge of N particles per species at the reference parameters instead of the sweep")
    ap.add_argument("--steps", type=int, default=40)
    ap.add_argument("--warmup", type=int, default=40)
    ap.add_argument("--tune", action="store_true", help="autotune the batched kernels' launch shapes first")
    ap.add_argument("--pressure", type=float, help="every discharge of the sweep at this pressure [Pa]")
    ap.add_argument("--voltage", type=float, help="every discharge of the sweep at this RF amplitude [V]")
    ap.add_argument("--rows", type=int)
    ap.add_argument("--ctas", type=int)
    ap.add_argument("--stages", type=int)
    ap.add_argument("--copies", type=int)
    ap.add_argument("--tuning", nargs="*", default=[], metavar="FIELD=VALUE",
                    help="other launch-shape overrides (cudapic_tuning fields)")
    a = ap.parse_args(argv)
    import cudapic_b200 as cp
    if a.one_discharge:
        specs = [DischargeSpec(voltage=250.0, pressure=10.0, gap=0.025, n_g=400, particles=a.one_discharge, seed=17)]
    else:
        specs = c2_specs(n=a.discharges)
        for s in specs:
            if a.pressure:
                s.pressure = a.pressure
            if a.voltage:
                s.voltage = a.voltage
    shape = {k: v for k, v in (("step_rows", a.rows), ("step_ctas_per_sm", a.ctas), ("step_stages", a.stages),
                               ("density_copies", a.copies)) if v}
    shape.update({k: int(v) for k, v in (f.split("=", 1) for f in a.tuning)})
    if shape:
        cp.set_tuning(**shape)
    with Batch(specs) as b:
        b.run_steps(a.warmup)
        b.synchronize()
        if a.tune:
            from cudapic_b200.autotune import tune_batch
            tune_batch(b)
            b.run_steps(a.warmup)
        t, w = b.timed_steps(a.steps)
        tu = cp.get_tuning()
        print(json.dumps({"discharges": len(specs), "steps": a.steps, "particle_steps_per_s": w / t,
                          "ms_per_step": 1e3 * t / a.steps, "device_errors": sum(1 for e in b.device_errors() if e),
                          "shape": tu}))
    return 0


if __name__ == "__main__":
    raise SystemExit(main())
