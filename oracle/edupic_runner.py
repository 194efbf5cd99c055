"""Runs the reference CPU program (eduPIC 1.0 built from C/eduPIC.cc into
oracle/_ref/ by oracle/Makefile) as the timed CPU baseline.

Test and baseline infrastructure only: used by bench.py's CPU-baseline leg
and its reference arm, never by the product.

A workload is a list of jobs, one independent eduPIC process per host core.
Each process resumes from a picdata.bin holding its particles (eduPIC's own
checkpoint format, C/eduPIC.cc:726-781) with its own voltage, gap, pressure,
superparticle weight and grid size.  The benchmark builds count
particle-steps with the GPU metric (every electron each step, every ion on
steps t % N_SUB == 0) and print a timestamped mark every 40 steps.

run_window() times all processes over one common wall-clock window: every
process sets itself up (cross sections, picdata.bin), reports ready and
waits at a start barrier; once all are ready they start together, run
through a warm-up and the window, and are stopped after it.  Each process's
particle-steps inside the window are read from its marks (linear between
two marks), so the aggregate is the work all cores did while all of them
were busy, divided by the window.
"""
import os
import re
import shutil
import subprocess
import tempfile
import time

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


def _work_at(marks, t_ns):
    """Particle-steps a process had done at time t_ns (linear between marks)."""
    for (s0, w0, a), (s1, w1, b) in zip(marks, marks[1:]):
        if a <= t_ns <= b:
            return w0 + (w1 - w0) * (t_ns - a) / max(1, b - a)
    raise RuntimeError("eduPIC marks do not cover the timing window")


def run_window(jobs, warm_s, window_s, timeout=900):
    """Times `jobs` as concurrent eduPIC processes over a common window.

    jobs: list of dicts with "electrons", "ions" (tuples of x, vx, vy, vz),
    "weight", "n_g" and optional "env" (EDUPIC_VOLTAGE, EDUPIC_L,
    EDUPIC_PRESSURE, ...) and "marks" (40-step marks the process may run;
    it is stopped once the window has passed).
    Returns (aggregate particle-steps/s, per-job particle-steps/s, window
    seconds, per-job particle-steps in the window).
    """
    tmp = tempfile.mkdtemp(prefix="edupic_")
    start_file = os.path.join(tmp, "start")
    procs = []
    try:
        for k, job in enumerate(jobs):
            d = os.path.join(tmp, "p%d" % k)
            os.makedirs(d)
            write_picdata(os.path.join(d, "picdata.bin"), job["electrons"], job["ions"])
            env = dict(os.environ)
            env.update({kk: str(v) for kk, v in (job.get("env") or {}).items()})
            env["EDUPIC_WEIGHT"] = repr(float(job["weight"]))
            env["EDUPIC_READY_FILE"] = os.path.join(d, "ready")
            env["EDUPIC_START_FILE"] = start_file
            err = open(os.path.join(d, "stderr.txt"), "w")
            p = subprocess.Popen([binary(job["n_g"]), str(int(job.get("marks", 100000)))], cwd=d, env=env,
                                 stdout=subprocess.DEVNULL, stderr=err)
            procs.append((p, err, d))
        deadline = time.monotonic() + timeout
        while not all(os.path.exists(os.path.join(d, "ready")) for _, _, d in procs):
            if time.monotonic() > deadline or any(p.poll() is not None for p, _, _ in procs):
                raise RuntimeError("eduPIC processes did not reach the start barrier")
            time.sleep(0.01)
        t_start = time.monotonic_ns()   # CLOCK_MONOTONIC, the clock of the marks
        with open(start_file, "w"):
            pass
        a = t_start + int(warm_s * 1e9)
        b = a + int(window_s * 1e9)
        # stop once every process has printed a mark after the window
        while True:
            time.sleep(0.05)
            if time.monotonic_ns() > b + int(1e9 * max(5.0, 0.5 * window_s)):
                break
            done = True
            for p, _, d in procs:
                text = open(os.path.join(d, "stderr.txt")).read()
                m = _MARK.findall(text)
                if p.poll() is None and (not m or int(m[-1][2]) < b):
                    done = False
                    break
            if done:
                break
        for p, _, _ in procs:
            if p.poll() is None:
                p.kill()
        per_job, rates = [], []
        for p, err, d in procs:
            p.wait(timeout=30)
            err.close()
            text = open(os.path.join(d, "stderr.txt")).read()
            marks = [(int(x), int(y), int(z)) for x, y, z in _MARK.findall(text)]
            w = _work_at(marks, b) - _work_at(marks, a)
            per_job.append(w)
            rates.append(w / window_s)
        return sum(per_job) / window_s, rates, window_s, per_job
    finally:
        for p, err, _ in procs:
            if p.poll() is None:
                p.kill()
                p.wait()
            if not err.closed:
                err.close()
        shutil.rmtree(tmp, ignore_errors=True)
