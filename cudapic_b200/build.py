"""Builds libcudapic.so in-tree with nvcc for sm_100a.

    python -m cudapic_b200.build        (or cudapic_b200.build.build())

Device code is compiled with -fmad=false (no implicit a*b+c contraction: the
kernels' f32 arithmetic is then reproducible by the CPU oracle) and IEEE
division / square root.  Objects go to cudapic_b200/_build/, the library to
cudapic_b200/libcudapic.so.
"""
import concurrent.futures as cf
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
BUILD = os.path.join(HERE, "_build")
LIB = os.path.join(HERE, "libcudapic.so")
GEN = os.path.join(CSRC, "generated", "jump_tables.inc")

NVCC = os.environ.get("NVCC", "nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
COMMON = ["-O3", "-std=c++17", "-lineinfo", "-I", ROOT, "-Xcompiler", "-fPIC,-ffp-contract=off,-Wall",
          "-fmad=false", "-prec-div=true", "-prec-sqrt=true", "-ftz=false", "--expt-relaxed-constexpr"]

SOURCES = ["host.cpp", "state.cpp", "batch.cpp", "checkpoint.cpp", "report.cpp", "kernels_density.cu",
           "kernels_poisson.cu", "kernels_push.cu", "kernels_mcc.cu", "kernels_step.cu", "kernels_inplace.cu", "kernels_batch.cu",
           "kernels_misc.cu", "kernels_xt.cu", "xt.cpp", "noalloc.cu", "sensitivity.cu", "fp64.cu"]


def _newer(target, deps):
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps if os.path.exists(d))


def _headers():
    hs = [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".cuh", ".h"))]
    hs.append(os.path.join(ROOT, "include", "cudapic.h"))
    hs.append(GEN)
    return hs


def _compile(src, verbose_ptxas=False):
    obj = os.path.join(BUILD, os.path.splitext(src)[0] + ".o")
    path = os.path.join(CSRC, src)
    if not _newer(obj, [path] + _headers()):
        return obj, ""
    cmd = [NVCC] + ARCH + COMMON + ["-c", path, "-o", obj]
    if verbose_ptxas and src.endswith(".cu"):
        cmd += ["-Xptxas", "-v"]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError("nvcc failed for %s:\n%s\n%s" % (src, " ".join(cmd), r.stderr))
    return obj, r.stderr


def build(verbose_ptxas=False, force=False):
    """Compile (incrementally) and link libcudapic.so; returns its path."""
    os.makedirs(BUILD, exist_ok=True)
    os.makedirs(os.path.dirname(GEN), exist_ok=True)
    gen_script = os.path.join(CSRC, "gen_jump_tables.py")
    if force or _newer(GEN, [gen_script]):
        subprocess.run([sys.executable, gen_script, GEN], check=True)
    if force:
        for f in os.listdir(BUILD):
            os.remove(os.path.join(BUILD, f))
    with cf.ThreadPoolExecutor(max_workers=min(8, os.cpu_count() or 1)) as ex:
        results = list(ex.map(lambda s: _compile(s, verbose_ptxas), SOURCES))
    objs = [o for o, _ in results]
    if verbose_ptxas:
        for (o, log), s in zip(results, SOURCES):
            if log:
                print("== %s\n%s" % (s, log))
    if force or _newer(LIB, objs):
        cmd = [NVCC] + ARCH + ["-shared", "-o", LIB] + objs + ["-lpthread"]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError("link failed:\n%s\n%s" % (" ".join(cmd), r.stderr))
    return LIB


if __name__ == "__main__":
    build(verbose_ptxas="-v" in sys.argv, force="--force" in sys.argv)
    print(LIB)
