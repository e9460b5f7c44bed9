"""L2_norm_of_gf_noalloc: the L2 norm for callers that may not allocate
device memory (fixed-arena frameworks, processes under a device-memory quota,
loops that cannot afford the synchronisation of cudaMalloc).  It is checked
through the C ABI against the allocating L2_norm_of_gf on the same device
data, on two calls in a row, within the L2 tolerance of the other parity tests
(1e-13 in log10), and the library's allocation counter is checked to stay
unchanged across the no-allocation calls -- also in a fresh process whose very
first library call is L2_norm_of_gf_noalloc.  This file is collected last so
that a stop at the first failure has already run every other test; it also
passes on its own in a fresh process."""
import ctypes as C
import os
import subprocess
import sys

import numpy as np
import pytest
from _util import ROOT, golden_grid, load_golden, problem_grid

from nrpyelliptic_b200 import _lib, abi
from nrpyelliptic_b200.problem import CONFIGS, Problem

pytestmark = pytest.mark.gpu
TOL = 1e-13


def _device(lib, a):
    p = lib.nrpyell_device_malloc(a.nbytes)
    lib.nrpyell_memcpy(p, a.ctypes.data, a.nbytes, 0)
    _lib.check(lib)
    return p


def _check_grid(lib, params, xx, residual):
    d = _device(lib, residual)
    as_real = C.cast(C.c_void_p(d), abi.PREAL)
    try:
        for R in (100.0, 1e300):
            ref = lib.L2_norm_of_gf(C.byref(params), abi.UUGF, R, xx, as_real)
            allocs = lib.nrpyell_device_alloc_count()
            first = lib.L2_norm_of_gf_noalloc(C.byref(params), abi.UUGF, R, xx, as_real)
            second = lib.L2_norm_of_gf_noalloc(C.byref(params), abi.UUGF, R, xx, as_real)
            _lib.check(lib)
            assert lib.nrpyell_device_alloc_count() == allocs
            assert np.isfinite(ref)
            assert abs(first - ref) <= TOL, (first, ref)
            assert abs(second - ref) <= TOL, (second, ref)
            assert first == second  # fixed reduction order: same bits every call
    finally:
        lib.nrpyell_device_free(d)


def test_noalloc_l2_matches_l2_norm_of_gf_on_golden_residual():
    lib = _lib.load()
    lib.nrpyell_clear_status()
    gold = load_golden("ops_unequal_24x16x8.npz")
    hg = golden_grid(gold)
    res = np.zeros(2 * hg.Ntot)
    res[:hg.Ntot] = gold["residual"]
    res[np.isnan(res)] = 0.0
    _check_grid(lib, hg.params, hg.xx, res)


def test_noalloc_l2_matches_l2_norm_of_gf_on_production_grid():
    lib = _lib.load()
    lib.nrpyell_clear_status()
    prob = Problem(CONFIGS["quasicircular_128x128x16"])
    hg = problem_grid(prob)
    rng = np.random.default_rng(11)
    res = rng.normal(size=2 * hg.Ntot) * 1e-3
    _check_grid(lib, prob.params, prob.xx, res)
    prob.close()


_FRESH = r"""
import ctypes as C, sys
sys.path.insert(0, sys.argv[1]); sys.path.insert(0, sys.argv[1] + "/tests")
import numpy as np
from _util import golden_grid, load_golden
from nrpyelliptic_b200 import _lib, abi
lib = _lib.load()
rt = C.CDLL("libcudart.so.12")  # the runtime the library is linked against
gold = load_golden("ops_unequal_24x16x8.npz")
hg = golden_grid(gold)
res = np.zeros(2 * hg.Ntot)
res[:hg.Ntot] = np.nan_to_num(gold["residual"])
d = C.c_void_p()
assert rt.cudaMalloc(C.byref(d), C.c_size_t(res.nbytes)) == 0
assert rt.cudaMemcpy(d, res.ctypes.data_as(C.c_void_p), C.c_size_t(res.nbytes), 1) == 0
p = C.cast(d, abi.PREAL)
assert lib.nrpyell_device_alloc_count() == 0
a = lib.L2_norm_of_gf_noalloc(C.byref(hg.params), abi.UUGF, 100.0, hg.xx, p)
b = lib.L2_norm_of_gf_noalloc(C.byref(hg.params), abi.UUGF, 100.0, hg.xx, p)
_lib.check(lib)
assert lib.nrpyell_device_alloc_count() == 0, lib.nrpyell_device_alloc_count()
ref = lib.L2_norm_of_gf(C.byref(hg.params), abi.UUGF, 100.0, hg.xx, p)
_lib.check(lib)
assert a == b and abs(a - ref) <= 1e-13 and abs(a - float(gold["l2_R100"])) <= 1e-13, (a, b, ref)
print("fresh-process noalloc ok", a)
"""


def test_noalloc_l2_first_call_in_a_fresh_process_allocates_nothing():
    """The first library call of a new process is the no-allocation norm: the
    library's allocation counter stays at zero over two calls, and the
    result equals L2_norm_of_gf's and the reference's."""
    r = subprocess.run([sys.executable, "-c", _FRESH, ROOT], capture_output=True, text=True, timeout=600,
                       env=dict(os.environ))
    assert r.returncode == 0, r.stdout + r.stderr
    assert "fresh-process noalloc ok" in r.stdout


def test_noalloc_l2_rejects_grids_beyond_its_fixed_size():
    lib = _lib.load()
    lib.nrpyell_clear_status()
    p = abi.paramstruct()
    lib.nrpyell_set_Cparameters_to_default(C.byref(p))
    p.Nxx0, p.Nxx1, p.Nxx2 = 4096, 64, 8
    p.Nxx_plus_2NGHOSTS0, p.Nxx_plus_2NGHOSTS1, p.Nxx_plus_2NGHOSTS2 = 4106, 74, 18
    xx = (abi.PREAL * 3)()
    out = lib.L2_norm_of_gf_noalloc(C.byref(p), abi.UUGF, 100.0, xx, None)
    assert np.isnan(out)
    assert lib.nrpyell_last_status() != 0
    assert b"exceeds the fixed maximum" in lib.nrpyell_last_error()
    lib.nrpyell_clear_status()
    # padded sizes that disagree with Nxx + 2 NGHOSTS are rejected too
    p.Nxx0, p.Nxx1, p.Nxx2 = 64, 64, 8
    p.Nxx_plus_2NGHOSTS0, p.Nxx_plus_2NGHOSTS1, p.Nxx_plus_2NGHOSTS2 = 74, 80, 18
    out = lib.L2_norm_of_gf_noalloc(C.byref(p), abi.UUGF, 100.0, xx, None)
    assert np.isnan(out)
    assert b"Nxx_plus_2NGHOSTS" in lib.nrpyell_last_error()
    lib.nrpyell_clear_status()
