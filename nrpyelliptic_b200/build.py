"""Build libnrpyell_gpu.so in-tree with nvcc for sm_100a.

    python -m nrpyelliptic_b200.build      (or call build())

The library holds the CUDA kernels, the extern "C" entry points declared in
include/nrpyell_gpu.h and the host set-up code.  It is linked with
-Bsymbolic so its internal calls (e.g. MoL_step_forward_in_time ->
rhs_eval's kernels) never bind to same-named symbols of another library
loaded into the process, such as a CPU build of the reference.
"""
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
INCLUDE = os.path.join(ROOT, "include")
LIB = os.path.join(HERE, "libnrpyell_gpu.so")

SOURCES = ["capi.cu", "driver.cu", "batch.cu", "tables.cu", "tables_gpu.cu", "kernels_ref.cu", "kernels_fused.cu",
           "kernels_march.cu", "noalloc.cu", "mlp.cu", "setup_gpu.cu", "export.cu",
           "setup.cpp"]
OBJDIR = os.path.join(HERE, "_build")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]


def nvcc():
    for cand in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", "nvcc"):
        if cand and (os.path.sep not in cand or os.path.exists(cand)):
            return cand
    return "nvcc"


def _stale(target, deps):
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


def build(force=False, verbose=False):
    """Compile every source to an object (in parallel) and link the library."""
    srcs = [os.path.join(CSRC, s) for s in SOURCES]
    headers = [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".h", ".cuh"))]
    headers += [os.path.join(INCLUDE, f) for f in os.listdir(INCLUDE) if f.endswith(".h")]
    os.makedirs(OBJDIR, exist_ok=True)
    flags = ARCH + ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC,-fopenmp,-O3", "-I", INCLUDE, "-I", CSRC]
    jobs = []
    for src in srcs:
        obj = os.path.join(OBJDIR, os.path.basename(src) + ".o")
        if force or _stale(obj, [src] + headers):
            jobs.append([nvcc()] + flags + ["-c", src, "-o", obj])
    if verbose:
        for j in jobs:
            print(" ".join(j))
    procs = [subprocess.Popen(j) for j in jobs]
    failed = [j for j, p in zip(jobs, procs) if p.wait() != 0]
    if failed:
        raise subprocess.CalledProcessError(1, failed[0])
    objs = [os.path.join(OBJDIR, os.path.basename(s) + ".o") for s in srcs]
    if not jobs and not _stale(LIB, objs):
        return LIB
    cmd = [nvcc()] + ARCH + ["-shared", "-Xlinker", "-Bsymbolic", "-o", LIB] + objs + ["-lgomp", "-lcudart"]
    if verbose:
        print(" ".join(cmd))
    subprocess.run(cmd, check=True)
    return LIB


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose=True)
