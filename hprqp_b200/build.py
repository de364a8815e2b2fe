"""Build libhprqp.so (sm_100a) in-tree with nvcc.

    python -m hprqp_b200.build        # or hprqp_b200.build.build()

Each translation unit compiles to an object under hprqp_b200/_build/ in
parallel; the shared library lands next to this file so it travels with the
source tree.  No Python extension machinery is involved: the library is a
plain C ABI (include/hprqp.h) loaded with ctypes.
"""
import os
import shutil
import subprocess
from concurrent.futures import ThreadPoolExecutor

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
BUILD = os.path.join(HERE, "_build")
LIB = os.path.join(HERE, "libhprqp.so")
SOURCES = ["engine.cu", "solver.cu", "host_setup.cpp", "pool.cpp", "noalloc.cu", "mlp.cu", "batch.cu", "batch_qp.cu", "tc_gemm.cu", "scale.cu"]
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]


def nvcc():
    for cand in (os.environ.get("NVCC"), shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found")


def _flags():
    return ARCH + ["-O3", "-lineinfo", "-std=c++17", "--extended-lambda", "-Xcompiler", "-fPIC,-fopenmp",
                   "-I" + os.path.join(ROOT, "include"), "-ccbin", "/usr/bin/g++"]


def _stale(obj, src):
    if not os.path.exists(obj):
        return True
    deps = [src] + [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".cuh", ".h"))]
    deps += [os.path.join(ROOT, "include", f) for f in os.listdir(os.path.join(ROOT, "include"))]
    t = os.path.getmtime(obj)
    return any(os.path.getmtime(d) > t for d in deps)


def build(verbose=False, force=False):
    os.makedirs(BUILD, exist_ok=True)
    cc = nvcc()
    jobs = []
    for s in SOURCES:
        src = os.path.join(CSRC, s)
        obj = os.path.join(BUILD, s + ".o")
        if force or _stale(obj, src):
            cmd = [cc] + _flags() + ["-c", src, "-o", obj]
            if s.endswith(".cu"):
                cmd += ["-Xptxas", "-v"] if verbose else []
            jobs.append(cmd)

    def run(cmd):
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError("nvcc failed:\n" + " ".join(cmd) + "\n" + r.stdout + r.stderr)
        return r.stdout + r.stderr

    with ThreadPoolExecutor(max_workers=len(SOURCES)) as ex:
        outs = list(ex.map(run, jobs))
    if verbose:
        for o in outs:
            print(o)
    objs = [os.path.join(BUILD, s + ".o") for s in SOURCES]
    if jobs or not os.path.exists(LIB):
        run([cc] + ARCH + ["-shared", "-o", LIB] + objs + ["-lgomp", "-ccbin", "/usr/bin/g++"])
    return LIB


if __name__ == "__main__":
    import sys
    print(build(verbose="-v" in sys.argv, force="-f" in sys.argv))
