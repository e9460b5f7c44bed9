"""Build recipe for the oracle (test infrastructure only).

  oracle/_build/liboracle.so       the CPU restatement in nrpyell_oracle.c
  oracle/_ref/libnrpyell_ref_v3.so the reference's own NRPyElliptic_Ccodes/*.c
  oracle/_ref/libnrpyell_ref_v4.so (all but main.c) + ref_harness.c, built with
                                   the reference Makefile's flags
                                   (-O2 -fopenmp -std=gnu99 ...) except
                                   -march=native, replaced by x86-64-v3
                                   (AVX2+FMA) and x86-64-v4 (AVX-512) so the
                                   objects run on any host that has the ISA
  oracle/_ref/NRPyElliptic_Playground      the reference main.c, unmodified
  oracle/_ref/NRPyElliptic_Playground_gpu  the same main.c and set-up objects
                                   linked against libnrpyell_gpu.so in place of
                                   the reference hot-path objects (drop-in check)

The _ref products need the reference sources and are only built where they
exist; nothing reads the reference at run time.  Both folders are git-ignored
and travel with the working tree.
"""
import os
import shutil
import subprocess

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
INCLUDE = os.path.join(ROOT, "include")
BUILD = os.path.join(HERE, "_build")
REF_OUT = os.path.join(HERE, "_ref")
# The reference's C sources: NRPYELL_REFERENCE_SRC, else the read-only
# checkout of this container.
REF_SRC = os.environ.get("NRPYELL_REFERENCE_SRC", "/root/reference/NRPyElliptic_Ccodes")
GPU_LIB_DIR = os.path.join(ROOT, "nrpyelliptic_b200")

ORACLE_LIB = os.path.join(BUILD, "liboracle.so")

# Files of the reference hot path: replaced by libnrpyell_gpu.so in the
# drop-in executable.
HOT_PATH = ["rhs_eval.c", "MoL_step_forward_in_time.c", "apply_bcs_outerradiation_and_inner.c",
            "apply_bcs_inner_only.c", "apply_bcs_outerextrap_and_inner.c", "residual_all_points.c",
            "L2_norm_of_gf.c", "MoL_malloc_y_n_gfs.c", "MoL_malloc_non_y_n_gfs.c",
            "MoL_free_memory_y_n_gfs.c", "MoL_free_memory_non_y_n_gfs.c"]
REF_CFLAGS = ["-O2", "-fopenmp", "-Wall", "-Wno-unused-variable", "-std=gnu99", "-fPIC"]


def _run(cmd, cwd=None):
    subprocess.run(cmd, check=True, cwd=cwd, stdout=subprocess.DEVNULL)


def _stale(target, deps):
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


def build_oracle(force=False):
    os.makedirs(BUILD, exist_ok=True)
    src = os.path.join(HERE, "nrpyell_oracle.c")
    if force or _stale(ORACLE_LIB, [src, os.path.join(INCLUDE, "nrpyell_abi.h")]):
        _run(["gcc", "-O2", "-fopenmp", "-ffp-contract=off", "-march=x86-64-v3", "-fPIC", "-shared",
              "-I", INCLUDE, "-o", ORACLE_LIB, src, "-lm"])
    return ORACLE_LIB


def ref_available():
    return os.path.isdir(REF_SRC)


def ref_lib_path(isa):
    return os.path.join(REF_OUT, "libnrpyell_ref_%s.so" % isa)


def _ref_sources():
    return sorted(f for f in os.listdir(REF_SRC) if f.endswith(".c") and f != "main.c")


def build_ref(force=False):
    """Compile the reference sources where they lie; outputs go to oracle/_ref."""
    if not ref_available():
        return None
    os.makedirs(REF_OUT, exist_ok=True)
    srcs = [os.path.join(REF_SRC, f) for f in _ref_sources()]
    harness = os.path.join(HERE, "ref_harness.c")
    built = {}
    for isa in ("v3", "v4"):
        lib = ref_lib_path(isa)
        if force or _stale(lib, srcs + [harness]):
            objdir = os.path.join(REF_OUT, "obj_" + isa)
            os.makedirs(objdir, exist_ok=True)
            objs = []
            for s in srcs:
                o = os.path.join(objdir, os.path.basename(s)[:-2] + ".o")
                _run(["gcc"] + REF_CFLAGS + ["-march=x86-64-" + isa, "-c", s, "-o", o], cwd=REF_SRC)
                objs.append(o)
            ho = os.path.join(objdir, "ref_harness.o")
            _run(["gcc", "-O2", "-fopenmp", "-fPIC", "-march=x86-64-" + isa, "-I", INCLUDE, "-c", harness, "-o", ho])
            _run(["gcc", "-shared", "-fopenmp", "-o", lib] + objs + [ho, "-lm"])
        built[isa] = lib
    # Executables from the unmodified main.c (x86-64-v3 objects).
    objdir = os.path.join(REF_OUT, "obj_v3")
    main_o = os.path.join(objdir, "main.o")
    exe = os.path.join(REF_OUT, "NRPyElliptic_Playground")
    exe_gpu = os.path.join(REF_OUT, "NRPyElliptic_Playground_gpu")
    main_c = os.path.join(REF_SRC, "main.c")
    if force or _stale(main_o, [main_c]):
        _run(["gcc"] + REF_CFLAGS + ["-march=x86-64-v3", "-c", main_c, "-o", main_o], cwd=REF_SRC)
    all_objs = [os.path.join(objdir, f[:-2] + ".o") for f in _ref_sources()]
    setup_objs = [os.path.join(objdir, f[:-2] + ".o") for f in _ref_sources() if f not in HOT_PATH]
    if force or _stale(exe, [main_o] + all_objs):
        _run(["gcc", "-fopenmp", "-o", exe, main_o] + all_objs + ["-lm", "-lgomp"])
    gpu_lib = os.path.join(GPU_LIB_DIR, "libnrpyell_gpu.so")
    if os.path.exists(gpu_lib) and (force or _stale(exe_gpu, [main_o, gpu_lib] + setup_objs)):
        _run(["gcc", "-fopenmp", "-o", exe_gpu, main_o] + setup_objs +
             ["-L" + GPU_LIB_DIR, "-lnrpyell_gpu", "-Wl,-rpath,$ORIGIN/../../nrpyelliptic_b200", "-lm", "-lgomp"])
    built["exe"] = exe
    built["exe_gpu"] = exe_gpu
    return built


def clean_ref_objects():
    for isa in ("v3", "v4"):
        shutil.rmtree(os.path.join(REF_OUT, "obj_" + isa), ignore_errors=True)


if __name__ == "__main__":
    print(build_oracle(force=True))
    print(build_ref(force=True))
