"""Relaxation drivers beyond main.c's loop: the Einstein Toolkit thorn's
stopping rule (nrpyell_relax_et) against the per-step residual history of
the main.c-semantics driver on the same trajectory."""
import ctypes as C

import numpy as np
import pytest
from _util import ptr

from nrpyelliptic_b200 import _lib
from nrpyelliptic_b200.problem import CONFIGS, DeviceState, Problem

pytestmark = pytest.mark.gpu
TILE = 15  # both drivers on the same tile shape: identical L2 partial sums


@pytest.fixture(scope="module")
def lib():
    lib = _lib.load()
    lib.nrpyell_clear_status()
    lib.nrpyell_set_tile(TILE)
    yield lib
    lib.nrpyell_set_tile(-1)


@pytest.mark.parametrize("every", [1, 7, 50])
def test_et_stopping_rule_matches_history(lib, every):
    prob = Problem(CONFIGS["shipped_64x64x8"], lib=lib)
    ds = DeviceState(prob, lib=lib)
    steps, fin = C.c_int(0), C.c_double(0)
    hist = np.zeros(6001)
    lib.nrpyell_relax(C.byref(ds.g), prob.dt, -11.0, 6000, 100.0, C.byref(steps), C.byref(fin), ptr(hist))
    _lib.check(lib)
    h = hist[:steps.value + 1]
    # the thorn tests after step n (its loop index) -- our history index n + 1
    cand = [n for n in range(1, len(h)) if (n - 1) % every == 0 and h[n] < -10.0]
    assert cand, "history too short"
    n_expect = cand[0]
    ds.set_state(prob.zero_state())
    it, fe = C.c_int(0), C.c_double(0)
    rc = lib.nrpyell_relax_et(C.byref(ds.g), prob.dt, -10.0, 6000, every, 100.0, C.byref(it), C.byref(fe))
    _lib.check(lib)
    assert rc == 0
    assert it.value == n_expect - 1
    assert fe.value == h[n_expect]
    ds.free()


def test_et_reports_a_missed_target(lib):
    prob = Problem(CONFIGS["shipped_64x64x8"], lib=lib)
    ds = DeviceState(prob, lib=lib)
    it, fe = C.c_int(0), C.c_double(0)
    rc = lib.nrpyell_relax_et(C.byref(ds.g), prob.dt, -10.0, 100, 10, 100.0, C.byref(it), C.byref(fe))
    _lib.check(lib)
    assert rc == 1 and it.value == 100 and fe.value > -10.0
    ds.free()
