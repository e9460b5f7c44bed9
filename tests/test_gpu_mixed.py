"""Mixed-precision relaxation (nrpyell_relax_mixed): an FP32 correction to
an FP64 state, relaxed in stretches of fold_every RK4 steps and folded into
the FP64 state, with the residual and its L2 norm evaluated in FP64 at every
fold; FP64 steps finish from the switch tolerance on.

Checks: the FP32 phase reaches log10 L2 <= -6 before switching (the
tolerance the FP32 phase is specified to reach), the relaxation reaches
-10, and the solution's error against the FP64 solution is stated -- max and
L2 of uu - uu_FP64 relative to max|uu_FP64|, split into r < R_L2 (the
region the stop test's norm covers) and r >= R_L2:
  64x64x8 (shipped punctures), against the reference's own solution:
      max error <= 1e-8 (all steps FP32, fold every 64 steps)
  256x256x32 (the unequal-mass spinning pair), against the FP64 GPU solve:
      max error <= 1e-9 inside and outside R_L2
"""
import ctypes as C

import numpy as np
import pytest
from _util import load_golden, ptr

from nrpyelliptic_b200 import _lib
from nrpyelliptic_b200.problem import CONFIGS, DeviceState, Problem

pytestmark = pytest.mark.gpu


def interior_uu(ds, prob):
    N = prob.N
    return ds.download("y_n")[:prob.Ntot].reshape(N[2], N[1], N[0])[5:-5, 5:-5, 5:-5]


def split_errors(prob, uu, ref):
    """max and L2 of uu - ref relative to max|ref| / |ref|, inside and
    outside the L2 integration radius."""
    inside = np.broadcast_to(prob.radius() < prob.cfg.R_L2, uu.shape)
    d = uu - ref
    sc = np.max(np.abs(ref))
    out = {}
    for name, m in (("in", inside), ("out", ~inside)):
        out["max_" + name] = float(np.max(np.abs(d[m])) / sc) if m.any() else 0.0
        out["l2_" + name] = float(np.sqrt(np.sum(d[m] ** 2) / np.sum(ref[m] ** 2))) if m.any() else 0.0
    return out


def mixed(lib, prob, ds, switch, fold, max_steps):
    n32, n64 = C.c_int(0), C.c_int(0)
    fin = C.c_double(0)
    hist = np.zeros(max_steps + 1)
    lib.nrpyell_memset(ds.ptr["y_n"], 0, 2 * prob.Ntot * 8)
    rc = lib.nrpyell_relax_mixed(C.byref(ds.g), prob.dt, -10.0, switch, fold, max_steps, prob.cfg.R_L2, C.byref(n32),
                                 C.byref(n64), C.byref(fin), ptr(hist))
    _lib.check(lib)
    return rc, n32.value, n64.value, fin.value, hist


def test_mixed_all_fp32_reaches_reference_solution_shipped_64x64x8():
    lib = _lib.load()
    lib.nrpyell_clear_status()
    gold = load_golden("relax_shipped_64x64x8.npz")
    prob = Problem(CONFIGS["shipped_64x64x8"])
    ds = DeviceState(prob)
    rc, n32, n64, fin, hist = mixed(lib, prob, ds, -10.0, 64, 6000)
    assert rc == 0 and fin <= -10.0 and hist[n32 + n64] == fin
    # every step in FP32; the FP64 norm at the folds is the judge
    assert n64 == 0 and abs(n32 - int(gold["steps"])) <= 2
    # the relaxation follows the FP64 trajectory: residual histories agree
    n = min(n32, int(gold["steps"])) + 1
    assert np.max(np.abs(hist[:n] - gold["history"][:n])) < 0.05
    e = split_errors(prob, interior_uu(ds, prob), gold["uu_interior"])
    print("mixed 64x64x8 all-FP32: %d steps (FP64: %d), errors vs reference %s" % (n32, int(gold["steps"]), e))
    assert max(e["max_in"], e["max_out"]) <= 1e-8, e
    ds.free()


def test_mixed_fp32_phase_reaches_1e6_before_switching():
    """Switch tolerance -6: the FP32 phase ends with its FP64-evaluated
    residual at or below 1e-6, the FP64 phase then reaches 1e-10."""
    lib = _lib.load()
    prob = Problem(CONFIGS["quasicircular_128x128x16"])
    ds = DeviceState(prob)
    rc, n32, n64, fin, hist = mixed(lib, prob, ds, -6.0, 256, 8000)
    assert rc == 0 and fin <= -10.0
    assert n32 > 0 and n64 > 0
    assert hist[n32] <= -6.0 + 0.05  # the FP32 evaluation met -6; the FP64 one agrees to rounding
    assert hist[0] > hist[n32] > hist[n32 + n64]
    ds.free()


def test_mixed_256x256x32_error_vs_fp64_solution():
    """The mixed-precision configuration at its own size: FP64 GPU solve and
    the mixed driver (all FP32, and switching at 1e-6) on the same problem;
    the errors of uu are stated split at R_L2."""
    lib = _lib.load()
    prob = Problem(CONFIGS["unequal_spinning_256x256x32"])
    ds = DeviceState(prob)
    st, fin = C.c_int(0), C.c_double(0)
    rc = lib.nrpyell_relax(C.byref(ds.g), prob.dt, -10.0, 60000, prob.cfg.R_L2, C.byref(st), C.byref(fin), None)
    _lib.check(lib)
    assert rc == 0
    ref = interior_uu(ds, prob)
    for switch in (-10.0, -6.0):
        rc, n32, n64, fin, hist = mixed(lib, prob, ds, switch, 256, 60000)
        assert rc == 0 and fin <= -10.0
        e = split_errors(prob, interior_uu(ds, prob), ref)
        print("mixed 256x256x32 switch %g: %d FP32 + %d FP64 steps (FP64 alone %d); errors vs FP64 %s"
              % (switch, n32, n64, st.value, e))
        assert abs(n32 + n64 - st.value) <= 0.01 * st.value
        assert max(e["max_in"], e["max_out"]) <= 1e-9, e
        if switch == -6.0:
            assert hist[n32] <= -6.0 + 0.05
    ds.free()
    prob.close()
