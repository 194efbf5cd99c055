"""Runs the reference CPU program (eduPIC 1.0 built from C/eduPIC.cc into
oracle/_ref/ by oracle/Makefile) as the timed CPU baseline.

Test and baseline infrastructure only: used by bench.py's CPU-baseline leg
and its reference arm, never by the product.

The workload is split into one independent eduPIC process per host core.
Each process resumes from a picdata.bin holding its share of the particles
(eduPIC's own checkpoint format, C/eduPIC.cc:726-781) with the
superparticle weight scaled by the number of shares, so every process
simulates the same discharge density as the whole population.  The
benchmark builds count particle-steps with the GPU metric (every electron
each step, every ion on steps t % N_SUB == 0) and print a timestamped mark
every 40 steps; the aggregate throughput over a window of marks is
sum(particle-steps) / (last end - first start) across processes.
"""
import os
import re
import shutil
import subprocess
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REF_DIR = os.path.join(HERE, "_ref")
STEPS_PER_MARK = 40
_MARK = re.compile(r"^EDUPIC_MARK (\d+) (\d+) (\d+)$", re.M)


def binary(n_g=400):
    name = "eduPIC_bench" if n_g == 400 else "eduPIC_bench_g%d" % n_g
    path = os.path.join(REF_DIR, name)
    if not os.path.exists(path):
        raise FileNotFoundError("%s not built (make -C oracle ref, needs the reference tree)" % path)
    return path


def available(n_g=400):
    try:
        binary(n_g)
        return True
    except FileNotFoundError:
        return False


def host_cores():
    try:
        return len(os.sched_getaffinity(0))
    except AttributeError:
        return os.cpu_count() or 1


def write_picdata(path, electrons, ions, time=0.0, cycles_done=1):
    """eduPIC checkpoint: doubles [Time, cycles, N_e, x..., vx..., vy..., vz..., N_i, ...]."""
    with open(path, "wb") as f:
        np.array([time, float(cycles_done), float(len(electrons[0]))], np.float64).tofile(f)
        for a in electrons:
            np.asarray(a, np.float64).tofile(f)
        np.array([float(len(ions[0]))], np.float64).tofile(f)
        for a in ions:
            np.asarray(a, np.float64).tofile(f)


def run(shares, weight, n_marks, n_g=400, env=None, timeout=900):
    """Starts one eduPIC process per share and waits for all.

    shares: list of (electrons, ions), each a tuple of 4 arrays (x, vx, vy, vz).
    n_marks: number of 40-step benchmark steps each process runs.
    Returns one list of marks (steps, particle_steps, t_ns) per process.
    """
    exe = binary(n_g)
    base_env = dict(os.environ)
    base_env["EDUPIC_WEIGHT"] = repr(float(weight))
    if env:
        base_env.update({k: str(v) for k, v in env.items()})
    tmp = tempfile.mkdtemp(prefix="edupic_")
    procs = []
    try:
        for k, (e, i) in enumerate(shares):
            d = os.path.join(tmp, "p%d" % k)
            os.makedirs(d)
            write_picdata(os.path.join(d, "picdata.bin"), e, i)
            err = open(os.path.join(d, "stderr.txt"), "w")
            p = subprocess.Popen([exe, str(n_marks)], cwd=d, env=base_env, stdout=subprocess.DEVNULL, stderr=err)
            procs.append((p, err, d))
        marks = []
        for p, err, d in procs:
            rc = p.wait(timeout=timeout)
            err.close()
            if rc != 0:
                raise RuntimeError("eduPIC exited with %d" % rc)
            text = open(os.path.join(d, "stderr.txt")).read()
            marks.append([(int(a), int(b), int(c)) for a, b, c in _MARK.findall(text)])
        return marks
    finally:
        for p, err, _ in procs:
            if p.poll() is None:
                p.kill()
        shutil.rmtree(tmp, ignore_errors=True)


def window_throughput(marks, first, last):
    """Aggregate particle-steps/s between marks `first` and `last` (indices of
    40-step marks) over all processes, and the per-mark wall times (s)."""
    total = 0
    t0 = min(m[first][2] for m in marks)
    t1 = max(m[last][2] for m in marks)
    for m in marks:
        total += m[last][1] - m[first][1]
    per_step = []
    for k in range(first, last):
        a = min(m[k][2] for m in marks)
        b = max(m[k + 1][2] for m in marks)
        per_step.append((b - a) * 1e-9)
    return total / ((t1 - t0) * 1e-9), total, (t1 - t0) * 1e-9, per_step


def split_population(electrons, ions, shares, per_share_cap=None, seed=0):
    """Deals particles round-robin into `shares` parts (optionally capped)."""
    out = []
    for k in range(shares):
        e = tuple(np.asarray(a[k::shares]) for a in electrons)
        i = tuple(np.asarray(a[k::shares]) for a in ions)
        if per_share_cap:
            e = tuple(a[:per_share_cap] for a in e)
            i = tuple(a[:per_share_cap] for a in i)
        out.append((e, i))
    return out
