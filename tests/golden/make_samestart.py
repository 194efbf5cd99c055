"""Runs eduPIC (the reference CPU program) from exactly the starts that the
GPU end-to-end runs use, and writes its outputs as fixtures.

The GPU runs against the eduPIC reference case (cudapic_b200/refcase.py)
start from electrons and ions sampled from the converged reference profiles
(`refcase.start_particles`, numpy default_rng(seed)).  This script writes
the same arrays into eduPIC's own checkpoint format (picdata.bin,
C/eduPIC.cc:726-781, time 0), lets eduPIC 1.0 (built from C/eduPIC.cc by
oracle/Makefile into oracle/_ref/, Mersenne-Twister seed = the start seed)
relax them for RELAX cycles (`eduPIC RELAX`) and measure MEASURE cycles
(`eduPIC MEASURE m`), and keeps what eduPIC writes, normalised by eduPIC
itself:

  edupic_<tag>_s<seed>_density.txt  -- density.dat (x, n_e, n_i)
  edupic_<tag>_s<seed>_eepf.txt     -- eepf.dat (energy, EEPF)
  edupic_<tag>_s<seed>_xt_means.txt -- RF-period means per node of the XT
      maps pot, efield, je, ji, powere, poweri, meanee, meanei, ioniz
  edupic_<tag>_s<seed>_conv.txt     -- conv.dat: cycle, N_e, N_i after
      every cycle of both runs

Both runs together take about 10 s per RF cycle per seed on one core at the
reference weight (7e4, ~1.1e5 particles per species); seeds run as parallel
processes.

    python tests/golden/make_samestart.py [--seeds 1,2,3,4] [--relax 300] [--measure 100]
                                          [--weight 7e4] [--tag ss]

Needs oracle/_ref/eduPIC (make -C oracle ref, which needs the reference
tree; CUDAPIC_REFERENCE names it).
"""
import argparse
import concurrent.futures as cf
import os
import shutil
import subprocess
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

XT_NAMES = ("pot", "efield", "je", "ji", "powere", "poweri", "meanee", "meanei", "ioniz")


def _load_refcase_module():
    """cudapic_b200/refcase.py by path: the sampling is plain numpy, and the
    package itself (which loads the CUDA library) is not needed here."""
    import importlib.util
    spec = importlib.util.spec_from_file_location("refcase", os.path.join(ROOT, "cudapic_b200", "refcase.py"))
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


def run_seed(seed, relax, measure, weight, tag, keep=None):
    from oracle.edupic_runner import write_picdata
    refcase = _load_refcase_module()
    ref = refcase.load_reference(HERE)
    e, i = refcase.start_particles(ref, seed, weight)
    exe = os.path.join(ROOT, "oracle", "_ref", "eduPIC")
    env = dict(os.environ, EDUPIC_SEED=str(seed), EDUPIC_WEIGHT=repr(float(weight)))
    d = keep or tempfile.mkdtemp(prefix="edupic_ss%d_" % seed)
    os.makedirs(d, exist_ok=True)
    try:
        write_picdata(os.path.join(d, "picdata.bin"), e, i, time=0.0, cycles_done=0)
        with open(os.path.join(d, "stdout.txt"), "w") as log:
            subprocess.run([exe, str(relax)], cwd=d, env=env, check=True, stdout=log, stderr=subprocess.DEVNULL)
            subprocess.run([exe, str(measure), "m"], cwd=d, env=env, check=True, stdout=log,
                           stderr=subprocess.DEVNULL)
        out = os.path.join(HERE, "edupic_%s_s%d" % (tag, seed))
        head = "# eduPIC 1.0 from refcase.start_particles(seed=%d, weight=%g): %d relax + %d measured cycles\n" % (
            seed, weight, relax, measure)
        for src, dst in (("density.dat", "_density.txt"), ("eepf.dat", "_eepf.txt"), ("conv.dat", "_conv.txt")):
            with open(os.path.join(d, src)) as f:
                body = f.read()
            with open(out + dst, "w") as f:
                f.write(head + body)
        cols = [np.loadtxt(os.path.join(d, "%s_xt.dat" % n)).mean(axis=1) for n in XT_NAMES]
        np.savetxt(out + "_xt_means.txt", np.stack(cols, 1), fmt="%.6e",
                   header=head.strip("# \n") + "\n" + " ".join(XT_NAMES) + " (RF-period averages per node)")
        return seed, len(e[0]), len(i[0])
    finally:
        if keep is None:
            shutil.rmtree(d, ignore_errors=True)


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--seeds", default="1,2,3,4")
    ap.add_argument("--relax", type=int, default=300)
    ap.add_argument("--measure", type=int, default=100)
    ap.add_argument("--weight", type=float, default=7.0e4)
    ap.add_argument("--tag", default="ss")
    a = ap.parse_args(argv)
    seeds = [int(s) for s in a.seeds.split(",")]
    with cf.ProcessPoolExecutor(max_workers=len(seeds), mp_context=__import__("multiprocessing").get_context(
            "spawn")) as ex:
        futs = [ex.submit(run_seed, s, a.relax, a.measure, a.weight, a.tag) for s in seeds]
        for f in futs:
            seed, ne, ni = f.result()
            print("seed %d: started from %d e + %d Ar+, fixtures written" % (seed, ne, ni), flush=True)


if __name__ == "__main__":
    main()
