"""Pins the CPU oracle (oracle/nrpyell_oracle.c) to the reference: every
hot-path function applied to the golden inputs reproduces the reference's
recorded outputs.  CPU only."""
import ctypes as C

import numpy as np
import pytest
from _util import golden_grid, interior_mask, load_golden, oracle, problem_grid, ptr, relmax

from nrpyelliptic_b200 import abi
from nrpyelliptic_b200.problem import CONFIGS, Problem

CASES = ["ops_shipped_16x8x6.npz", "ops_unequal_24x16x8.npz"]


@pytest.mark.parametrize("case", CASES)
def test_rhs_eval_bitwise(case):
    gold = load_golden(case)
    hg = golden_grid(gold)
    o = oracle()
    rhs = np.full(2 * hg.Ntot, np.nan)
    y = gold["y_random"].copy()
    o.oracle_rhs_eval(C.byref(hg.params), C.byref(hg.rfm), ptr(hg.aux), ptr(y), ptr(rhs))
    m = np.tile(interior_mask(hg.N), 2)
    np.testing.assert_array_equal(rhs[m], gold["rhs"][m])


@pytest.mark.parametrize("case", CASES)
def test_residual_bitwise_and_l2(case):
    gold = load_golden(case)
    hg = golden_grid(gold)
    o = oracle()
    res = np.full(2 * hg.Ntot, np.nan)
    y = gold["y_consistent"].copy()
    o.oracle_residual_all_points(C.byref(hg.params), C.byref(hg.rfm), ptr(hg.aux), ptr(y), ptr(res))
    m = interior_mask(hg.N)
    np.testing.assert_array_equal(res[:hg.Ntot][m], gold["residual"][m])
    l2 = o.oracle_L2_norm_of_gf(C.byref(hg.params), 0, 100.0, hg.xx, ptr(res))
    assert abs(l2 - float(gold["l2_R100"])) < 1e-13
    l2i = o.oracle_L2_norm_of_gf(C.byref(hg.params), 0, 1e300, hg.xx, ptr(res))
    assert abs(l2i - float(gold["l2_Rinf"])) < 1e-13


@pytest.mark.parametrize("case", CASES)
def test_radiation_and_inner_bc(case):
    gold = load_golden(case)
    hg = golden_grid(gold)
    o = oracle()
    y = gold["y_consistent"].copy()
    rhs = np.full(2 * hg.Ntot, np.nan)
    o.oracle_rhs_eval(C.byref(hg.params), C.byref(hg.rfm), ptr(hg.aux), ptr(y), ptr(rhs))
    cw = (C.c_double * 2)(hg.params.uu_wavespeed_at_OB, hg.params.vv_wavespeed_at_OB)
    fi = (C.c_double * 2)(0.0, 0.0)
    o.oracle_apply_bcs_outerradiation_and_inner(C.byref(hg.params), C.byref(hg.bc), hg.xx, cw, fi, ptr(y), ptr(rhs))
    ref = gold["rhs_bc"]
    assert not np.any(np.isnan(ref))
    for gf in range(2):
        sl = slice(gf * hg.Ntot, (gf + 1) * hg.Ntot)
        assert relmax(rhs[sl], ref[sl]) < 1e-12


@pytest.mark.parametrize("case", CASES)
def test_mol_steps(case):
    gold = load_golden(case)
    hg = golden_grid(gold)
    o = oracle()
    hg.bufs["y_n"][:] = gold["y_consistent"]
    g = hg.griddata()
    dt = float(gold["dt"])
    o.oracle_MoL_step_forward_in_time(C.byref(g), dt)
    assert relmax(hg.bufs["y_n"], gold["y_step1"]) < 1e-13
    for _ in range(9):
        o.oracle_MoL_step_forward_in_time(C.byref(g), dt)
    assert relmax(hg.bufs["y_n"], gold["y_step10"]) < 1e-12


@pytest.mark.parametrize("case", CASES)
def test_extrapolation_branch(case):
    """apply_bcs_outerextrap_and_inner (apply_bcs_outerextrap_and_inner.c:15-75)
    on the random state, and one MoL step with outer_bc_type =
    EXTRAPOLATION_OUTER_BCS (MoL_step_forward_in_time.c, extrapolation calls),
    against the reference build's outputs."""
    gold = load_golden(case)
    hg = golden_grid(gold)
    o = oracle()
    y = gold["y_random"].copy()
    o.oracle_apply_bcs_outerextrap_and_inner(C.byref(hg.params), C.byref(hg.bc), ptr(y))
    assert relmax(y, gold["y_extrap"]) < 1e-15
    hg.params.outer_bc_type = abi.EXTRAPOLATION_OUTER_BCS
    hg.bufs["y_n"][:] = gold["y_consistent"]
    g = hg.griddata()
    o.oracle_MoL_step_forward_in_time(C.byref(g), float(gold["dt"]))
    assert relmax(hg.bufs["y_n"], gold["y_step1_extrap"]) < 1e-13


@pytest.mark.parametrize("case", CASES)
def test_relax_history(case):
    gold = load_golden(case)
    hg = golden_grid(gold)
    o = oracle()
    g = hg.griddata()
    hist = np.zeros(41)
    steps = C.c_int(0)
    o.oracle_relax(C.byref(g), float(gold["dt"]), -30.0, 40, 100.0, ptr(hist), C.byref(steps))
    assert steps.value == 40
    np.testing.assert_allclose(hist, gold["relax_history40"], rtol=0, atol=1e-11)
    assert relmax(hg.bufs["y_n"], gold["y_relax40"]) < 1e-11


def test_relax_to_tolerance_shipped_64x64x8():
    """Full relaxation of the reference's shipped puncture set: the oracle, fed
    by the library's own set-up, converges at the reference's step with the
    reference's solution."""
    gold = load_golden("relax_shipped_64x64x8.npz")
    prob = Problem(CONFIGS["shipped_64x64x8"])
    hg = problem_grid(prob)
    g = hg.griddata()
    o = oracle()
    hist = np.zeros(int(gold["steps"]) + 50)
    steps = C.c_int(0)
    rc = o.oracle_relax(C.byref(g), prob.dt, -10.0, len(hist) - 1, 100.0, ptr(hist), C.byref(steps))
    assert rc == 0
    assert abs(steps.value - int(gold["steps"])) <= 1
    n = min(steps.value, int(gold["steps"])) + 1
    np.testing.assert_allclose(hist[:n], gold["history"][:n], rtol=0, atol=1e-8)
    N = hg.N
    uu = hg.bufs["y_n"][:hg.Ntot].reshape(N[2], N[1], N[0])[5:-5, 5:-5, 5:-5]
    ref = gold["uu_interior"]
    assert np.max(np.abs(uu - ref)) <= 1e-10 * np.max(np.abs(ref))
