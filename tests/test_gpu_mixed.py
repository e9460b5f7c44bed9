"""Mixed-precision relaxation (FP32 until the residual stalls near 1e-6 or
reaches it, then FP64 to 1e-10) against the reference's FP64 solution."""
import ctypes as C

import numpy as np
import pytest
from _util import load_golden, ptr

from nrpyelliptic_b200 import _lib
from nrpyelliptic_b200.problem import CONFIGS, DeviceState, Problem

pytestmark = pytest.mark.gpu


def test_mixed_precision_reaches_reference_solution_shipped_64x64x8():
    lib = _lib.load()
    lib.nrpyell_clear_status()
    gold = load_golden("relax_shipped_64x64x8.npz")
    prob = Problem(CONFIGS["shipped_64x64x8"])
    ds = DeviceState(prob)
    n32, n64 = C.c_int(0), C.c_int(0)
    fin = C.c_double(0)
    hist = np.zeros(6001)
    rc = lib.nrpyell_relax_mixed(C.byref(ds.g), prob.dt, -10.0, -6.0, 200, 0.98, 6000, 100.0, C.byref(n32),
                                 C.byref(n64), C.byref(fin), ptr(hist))
    _lib.check(lib)
    assert rc == 0 and fin.value <= -10.0
    assert n32.value > 0
    # the FP32 phase ended at the switch tolerance or at a stall
    assert hist[n32.value] <= -6.0 or n32.value >= 200
    N = prob.N
    uu = ds.download("y_n")[:prob.Ntot].reshape(N[2], N[1], N[0])[5:-5, 5:-5, 5:-5]
    ref = gold["uu_interior"]
    err = np.max(np.abs(uu - ref)) / np.max(np.abs(ref))
    # Both solutions satisfy the discrete equations to log10 L2 <= -10 but
    # reach them along different paths; their difference is of that order.
    assert err < 1e-8, err
    print("mixed 64x64x8: %d FP32 + %d FP64 steps (FP64 alone: %d), max rel err vs reference %.2e"
          % (n32.value, n64.value, int(gold["steps"]), err))
    ds.free()


def test_mixed_precision_history_is_continuous():
    """The FP64 phase starts from the converted FP32 state: its first residual
    is within FP32 rounding of the last FP32 one, and both phases keep the
    history monotone on average."""
    lib = _lib.load()
    prob = Problem(CONFIGS["shipped_64x64x8"])
    ds = DeviceState(prob)
    n32, n64 = C.c_int(0), C.c_int(0)
    fin = C.c_double(0)
    hist = np.zeros(6001)
    lib.nrpyell_relax_mixed(C.byref(ds.g), prob.dt, -10.0, -5.0, 200, 0.98, 6000, 100.0, C.byref(n32), C.byref(n64),
                            C.byref(fin), ptr(hist))
    _lib.check(lib)
    k = n32.value
    assert hist[0] > hist[k] > hist[k + n64.value]
    ds.free()
