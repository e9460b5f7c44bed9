"""The C-ABI library loads, exports every function its headers declare, and
its struct layout matches the reference layout mirrored in abi.py.  No GPU
work is issued."""
import ctypes as C
import glob
import os
import re

from _util import ROOT

from nrpyelliptic_b200 import _lib, abi

DECL = re.compile(r"^\s*(?:const\s+)?(?:void|int|REAL|double|long long|char)\s*\*?\s*(\w+)\s*\(", re.M)


def declared_functions():
    names = set()
    for h in glob.glob(os.path.join(ROOT, "include", "*.h")):
        txt = open(h).read()
        txt = re.sub(r"/\*.*?\*/", "", txt, flags=re.S)
        for m in DECL.finditer(txt):
            names.add(m.group(1))
    return names


def test_library_loads_and_exports_every_declared_symbol():
    lib = _lib.load()
    names = declared_functions()
    assert "rhs_eval" in names and "MoL_step_forward_in_time" in names and "L2_norm_of_gf" in names
    missing = [n for n in sorted(names) if not hasattr(lib, n)]
    assert not missing, missing


def test_reference_prototypes_are_all_exported():
    lib = _lib.load()
    for n in ["rhs_eval", "MoL_step_forward_in_time", "apply_bcs_outerradiation_and_inner", "apply_bcs_inner_only",
              "apply_bcs_outerextrap_and_inner", "residual_all_points", "L2_norm_of_gf", "MoL_malloc_y_n_gfs",
              "MoL_malloc_non_y_n_gfs", "MoL_free_memory_y_n_gfs", "MoL_free_memory_non_y_n_gfs"]:
        assert hasattr(lib, n), n


def test_struct_layout_matches_reference_layout():
    lib = _lib.load()
    out = (C.c_int * 32)()
    n = lib.nrpyell_abi_layout(out, 32)
    assert list(out[:n]) == abi.layout()
    # 71 REAL + 8 int, in the reference's declaration order
    assert C.sizeof(abi.paramstruct) == 71 * 8 + 8 * 4
    assert abi.layout()[-1] == 5  # NGHOSTS


def test_python_mirror_has_every_paramstruct_field_of_the_header():
    txt = open(os.path.join(ROOT, "include", "nrpyell_abi.h")).read()
    body = txt[txt.index("typedef struct __paramstruct__"):txt.index("} paramstruct;")]
    fields = re.findall(r"(REAL|int)\s+([^;]+);", body)
    names = []
    for _, group in fields:
        names += [x.strip() for x in group.split(",")]
    assert names == abi.PARAM_REALS + abi.PARAM_INTS


def test_status_api_without_gpu_work():
    lib = _lib.load()
    lib.nrpyell_clear_status()
    assert lib.nrpyell_last_status() == 0
    lib.nrpyell_set_step_mode(1)
    assert lib.nrpyell_get_step_mode() == 1
    lib.nrpyell_set_step_mode(0)
    assert lib.nrpyell_get_step_mode() == 0


def test_batched_drivers_reject_empty_batches_without_gpu_work():
    """n <= 0 or missing arrays: -1 and a recorded error before any CUDA call,
    under both status names."""
    lib = _lib.load()
    for name, args in (("nrpyell_relax_batch", (0, None, None, -10.0, 10, 100.0, None, None)),
                       ("nrpyell_relax_batch_mixed", (0, None, None, -10.0, -10.0, 256, 10, 100.0, None, None, None))):
        lib.nrpyell_clear_status()
        assert getattr(lib, name)(*args) == -1, name
        assert lib.nrpyell_last_status() != 0 and lib.nrpyell_gpu_last_status() == lib.nrpyell_last_status()
        assert b"need n > 0" in lib.nrpyell_last_error(), name
    lib.nrpyell_clear_status()
    assert lib.nrpyell_gpu_last_status() == 0


def test_optimum_eta_damping_formula():
    """Eq. (B6) and (36) of arXiv:2111.02424 as the thorn evaluates them."""
    import math

    import pytest

    from nrpyelliptic_b200.problem import CONFIGS, Problem
    lib = _lib.load()
    prob = Problem(CONFIGS["quasicircular_128x128x16"], lib=lib)
    p = prob.params
    A, b, dt = p.AMAX, p.bScale, prob.dt
    c1 = math.cos(p.dxx1 / 2)
    trc = dt / (0.5 * p.dxx1) * math.atanh(A / math.sqrt(A * A + b * b * c1 * c1)) * c1 * math.cos(p.dxx2 / 2)
    assert lib.nrpyell_compute_TRC(A, b, 0.5, dt, p.dxx1, p.dxx2) == pytest.approx(trc, rel=1e-14)
    lib.nrpyell_set_optimum_eta_damping(dt, 0.5, C.byref(p))
    assert p.eta_damping == pytest.approx(6.9 * trc ** -0.79 - 0.7, rel=1e-14)
