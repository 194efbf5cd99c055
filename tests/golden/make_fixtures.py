"""Regenerates the golden fixtures of tests/golden/ from the reference tree.

Run where the reference checkout is present (CUDAPIC_REFERENCE, default a
sibling of this repository named "reference"):

    python tests/golden/make_fixtures.py

It writes:
  xoshiro128p_10000.txt  -- 10 000 xoshiro128+ outputs from state {1,1,1,1},
      produced by the reference's own generator
      (Rust-CUDA/xorshiro128c/xoshiro128p.c, built by oracle/Makefile into
      oracle/_ref/) and checked byte-identical to the file the reference
      ships (Rust-CUDA/xorshiro128c/10000-c.txt).
  edupic_ref_density.txt -- converged cycle-averaged n_e, n_i of the
      eduPIC reference case (C/ReferenceCase_RawData/Figure10_density.dat).
  edupic_ref_eepf.txt    -- its EEPF (Figure12_eepf.dat).
  edupic_ref_conv_tail.txt -- last 100 cycles of its particle counts
      (Figure9_conv.dat).
  edupic_ref_xt_means.txt -- its XT maps (Figure11*_xt.dat) averaged over
      the RF period: one row per node, columns pot, efield, je, ji, heate,
      heati, meanee, meanei, ioniz.
  edupic_ref_ifed.txt    -- its IFEDs at both electrodes (Figure13_ifed.dat).
  edupic_c0_conv.txt     -- cycle, N_e, N_i of the reference CPU program
      (eduPIC 1.0 built from C/eduPIC.cc by oracle/Makefile, Mersenne
      Twister seed 5489) for the init cycle plus 10 cycles from 1000 + 1000
      particles.
  edupic_c0_conv_seeds.txt -- the same run for Mersenne-Twister seeds
      1 .. 16 (EDUPIC_SEED): one row per seed and cycle, columns seed,
      cycle, N_e, N_i (the spread of the growth between seeds).

The same-start fixtures (edupic_ss_*, edupic_c3_*) come from
make_samestart.py.
"""
import filecmp
import os
import shutil
import subprocess
import sys
import tempfile

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
ORACLE = os.path.join(ROOT, "oracle")
REF = os.environ.get("CUDAPIC_REFERENCE", os.path.join(os.path.dirname(ROOT), "reference"))


def main():
    subprocess.run(["make", "-s", "-C", ORACLE, "ref", "REF=" + REF], check=True)
    gen = os.path.join(ORACLE, "_ref", "10000-c.txt")
    shipped = os.path.join(REF, "Rust-CUDA", "xorshiro128c", "10000-c.txt")
    if not filecmp.cmp(gen, shipped, shallow=False):
        sys.exit("xoshiro128p.c output differs from the shipped 10000-c.txt")
    shutil.copyfile(gen, os.path.join(HERE, "xoshiro128p_10000.txt"))

    raw = os.path.join(REF, "C", "ReferenceCase_RawData")
    shutil.copyfile(os.path.join(raw, "Figure10_density.dat"), os.path.join(HERE, "edupic_ref_density.txt"))
    shutil.copyfile(os.path.join(raw, "Figure12_eepf.dat"), os.path.join(HERE, "edupic_ref_eepf.txt"))
    shutil.copyfile(os.path.join(raw, "Figure13_ifed.dat"), os.path.join(HERE, "edupic_ref_ifed.txt"))
    cols = []
    for name in ("c)_pot", "d)_efield", "e)_je", "f)_ji", "g)_heate", "h)_heati", "i)_meanee", "j)_meanei",
                 "k)_ioniz"):
        with open(os.path.join(raw, "Figure11%s_xt.dat" % name)) as f:
            rows = [[float(v) for v in ln.split()] for ln in f if ln.strip()]
        cols.append([sum(r) / len(r) for r in rows])
    with open(os.path.join(HERE, "edupic_ref_xt_means.txt"), "w") as f:
        f.write("# pot efield je ji heate heati meanee meanei ioniz (RF-period averages per node)\n")
        for k in range(len(cols[0])):
            f.write("  ".join("%.6e" % c[k] for c in cols) + "\n")
    with open(os.path.join(raw, "Figure9_conv.dat")) as f:
        lines = [ln for ln in f if ln.strip()]
    with open(os.path.join(HERE, "edupic_ref_conv_tail.txt"), "w") as f:
        f.writelines(lines[-100:])

    exe = os.path.join(ORACLE, "_ref", "eduPIC")
    with tempfile.TemporaryDirectory() as d:
        subprocess.run([exe, "0"], cwd=d, check=True, capture_output=True)
        subprocess.run([exe, "10"], cwd=d, check=True, capture_output=True)
        shutil.copyfile(os.path.join(d, "conv.dat"), os.path.join(HERE, "edupic_c0_conv.txt"))
    write_c0_seeds(exe, range(1, 17))
    print("fixtures written to", HERE)


def _c0_run(exe, seed):
    env = dict(os.environ, EDUPIC_SEED=str(seed))
    with tempfile.TemporaryDirectory() as d:
        subprocess.run([exe, "0"], cwd=d, check=True, capture_output=True, env=env)
        subprocess.run([exe, "10"], cwd=d, check=True, capture_output=True, env=env)
        with open(os.path.join(d, "conv.dat")) as f:
            return [(seed,) + tuple(int(v) for v in ln.split()) for ln in f if ln.strip()]


def write_c0_seeds(exe, seeds):
    import concurrent.futures as cf
    with cf.ThreadPoolExecutor(max_workers=min(8, os.cpu_count() or 1)) as ex:
        runs = list(ex.map(lambda s: _c0_run(exe, s), seeds))
    with open(os.path.join(HERE, "edupic_c0_conv_seeds.txt"), "w") as f:
        f.write("# eduPIC 1.0, init cycle + 10 cycles from 1000 + 1000 particles at rest; seed cycle N_e N_i\n")
        for rows in runs:
            for r in rows:
                f.write("%d %d %d %d\n" % r)


if __name__ == "__main__":
    main()
