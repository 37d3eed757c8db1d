"""Build libucg.so (the C-ABI library) in-tree with nvcc for sm_100a.

Each translation unit is compiled separately (in parallel) and linked into one
shared library.  rk.cu is compiled without multiply-add contraction: its
elementwise right-hand side and Runge-Kutta combinations round every operation
as written, like the reference's gfortran build on x86-64; the products inside
its matrix-vector kernels use explicit fused multiply-adds.
"""
import concurrent.futures as cf
import glob
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
OBJ = os.path.join(HERE, "_obj")
LIB = os.path.join(HERE, "libucg.so")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
FLAGS = ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC", "--expt-relaxed-constexpr"]
PER_FILE = {"rk.cu": ["-fmad=false"]}


def sources():
    return sorted(glob.glob(os.path.join(CSRC, "*.cu")) + glob.glob(os.path.join(CSRC, "*.cpp")))


def stale():
    if not os.path.exists(LIB):
        return True
    t = os.path.getmtime(LIB)
    deps = sources() + glob.glob(os.path.join(CSRC, "*.cuh")) + glob.glob(os.path.join(CSRC, "*.h")) + [
        os.path.join(HERE, "..", "include", "ucg.h"), __file__]
    return any(os.path.getmtime(p) > t for p in deps)


def build(force=False, verbose=False, extra=None):
    if not force and not stale():
        return LIB
    nvcc = os.environ.get("NVCC", "nvcc")
    os.makedirs(OBJ, exist_ok=True)

    def compile_one(src):
        name = os.path.basename(src)
        obj = os.path.join(OBJ, name + ".o")
        cmd = [nvcc] + ARCH + FLAGS + PER_FILE.get(name, []) + (extra or []) + ["-c", src, "-o", obj]
        if verbose:
            print(" ".join(cmd), file=sys.stderr)
        r = subprocess.run(cmd, capture_output=True, text=True)
        return obj, r

    with cf.ThreadPoolExecutor(max_workers=min(8, os.cpu_count() or 1)) as ex:
        results = list(ex.map(compile_one, sources()))
    for obj, r in results:
        sys.stderr.write(r.stdout + r.stderr)
        if r.returncode != 0:
            raise RuntimeError(f"nvcc failed for {obj}")
    cmd = [nvcc] + ARCH + ["-shared", "-o", LIB + ".tmp"] + [o for o, _ in results] + ["-lcuda"]
    subprocess.run(cmd, check=True)
    os.replace(LIB + ".tmp", LIB)
    return LIB


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose=True,
          extra=["-Xptxas", "-v"] if "--ptxas-v" in sys.argv else None)
    print(LIB)
