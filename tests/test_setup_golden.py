"""The library's host set-up (grid, reference-metric tables, puncture source
terms, wavespeed, time step, boundary maps) against the reference's own
set-up, recorded in the golden fixtures.  CPU only."""
import ctypes as C
import hashlib

import numpy as np
import pytest
from _util import interior_mask, load_golden, outer_records, params_from_bytes

from nrpyelliptic_b200 import _lib, abi
from nrpyelliptic_b200.problem import Config, Problem

CASES = ["ops_shipped_16x8x6.npz", "ops_unequal_24x16x8.npz"]


def problem_for(gold):
    p = params_from_bytes(gold["params"])
    from nrpyelliptic_b200.problem import Punctures
    pu = Punctures(p.bare_mass_0, p.bare_mass_1, (p.puncture_0_x, p.puncture_0_y, p.puncture_0_z),
                   (p.puncture_1_x, p.puncture_1_y, p.puncture_1_z), (p.P0_x, p.P0_y, p.P0_z),
                   (p.P1_x, p.P1_y, p.P1_z), (p.S0_x, p.S0_y, p.S0_z), (p.S1_x, p.S1_y, p.S1_z))
    cfg = Config("golden", tuple(int(x) for x in gold["Nxx"]), pu, bScale=p.bScale, AMAX=p.AMAX, SINHWAA=p.SINHWAA,
                 CFL=float(gold["cfl"]), eta=p.eta_damping)
    return Problem(cfg), p


@pytest.mark.parametrize("case", CASES)
def test_params_grid_dt(case):
    gold = load_golden(case)
    prob, pref = problem_for(gold)
    mine = prob.params
    for f in abi.PARAM_INTS + ["dxx0", "dxx1", "dxx2", "invdx0", "invdx1", "invdx2", "AMAX", "SINHWAA", "bScale",
                               "eta_damping", "bare_mass_0", "bare_mass_1"]:
        assert getattr(mine, f) == getattr(pref, f), f
    xx = prob.xx_arrays()
    for i in range(3):
        np.testing.assert_array_equal(xx[i], gold["xx%d" % i])
    assert abs(prob.dt - float(gold["dt"])) <= 1e-14 * float(gold["dt"])
    assert abs(mine.uu_wavespeed_at_OB - float(gold["c_OB"])) <= 1e-13 * float(gold["c_OB"])


@pytest.mark.parametrize("case", CASES)
def test_rfm_tables(case):
    gold = load_golden(case)
    prob, _ = problem_for(gold)
    rfm = prob.rfm_arrays()
    for name in abi.RFM_FIELDS:
        ref = gold["rfm_" + name]
        scale = np.maximum(np.abs(ref), 1e-300)
        assert np.max(np.abs(rfm[name] - ref) / scale) < 1e-12, name


@pytest.mark.parametrize("case", CASES)
def test_auxevol(case):
    gold = load_golden(case)
    prob, _ = problem_for(gold)
    N = prob.N
    Ntot = prob.Ntot
    aux, ref = prob.aux, gold["aux"]
    psi, psi_r = aux[Ntot:2 * Ntot], ref[Ntot:2 * Ntot]
    assert np.max(np.abs(psi - psi_r) / np.abs(psi_r)) < 1e-13
    aa, aa_r = aux[:Ntot], ref[:Ntot]
    # A_ij A^ij: closed-form derivatives here, expanded SymPy expression there
    assert np.max(np.abs(aa - aa_r)) <= 1e-11 * np.max(np.abs(aa_r))
    m = interior_mask(N)
    ws, ws_r = aux[2 * Ntot:][m], ref[2 * Ntot:][m]
    assert np.max(np.abs(ws - ws_r) / ws_r) < 1e-13


@pytest.mark.parametrize("case", CASES)
def test_bcstruct_identical(case):
    gold = load_golden(case)
    prob, _ = problem_for(gold)
    b = prob.bc
    ni = b.bc_info.num_inner_boundary_points
    inner_ref = gold["inner"]
    assert ni == len(inner_ref)
    raw = np.ctypeslib.as_array(C.cast(b.inner_bc_array, C.POINTER(C.c_int8)),
                                shape=(ni * C.sizeof(abi.innerpt_bc_struct),))
    inner = raw.view(inner_ref.dtype)
    np.testing.assert_array_equal(inner["dst"], inner_ref["dst"])
    np.testing.assert_array_equal(inner["src"], inner_ref["src"])
    np.testing.assert_array_equal(inner["par"][:, 0], inner_ref["par"][:, 0])
    counts, outer = outer_records(b)
    np.testing.assert_array_equal(counts, gold["outer_counts"])
    np.testing.assert_array_equal(outer, gold["outer"])
    lb = np.array([[[b.bc_info.bc_loop_bounds[gz][f][i] for i in range(6)] for f in range(6)] for gz in range(5)])
    np.testing.assert_array_equal(lb, gold["loop_bounds"])


def test_bcmaps_production_grids():
    gold = load_golden("bcmaps.npz")
    lib = _lib.load()
    for name, n_inner, counts, sha, dt in zip(gold["names"], gold["n_inner"], gold["outer_counts"], gold["sha256"],
                                              gold["dt"]):
        grid = tuple(int(x) for x in str(name).split("x"))
        prob = Problem(Config("bc", grid), lib)
        b = prob.bc
        ni = b.bc_info.num_inner_boundary_points
        assert ni == n_inner
        raw = np.ctypeslib.as_array(C.cast(b.inner_bc_array, C.POINTER(C.c_int32)), shape=(ni * 5,)).reshape(ni, 5)
        pairs = raw[:, :2].astype(np.int64)
        pairs = pairs[np.argsort(pairs[:, 0])]
        assert hashlib.sha256(pairs.tobytes()).hexdigest() == str(sha)
        c, _ = outer_records(b)
        np.testing.assert_array_equal(c, counts)
        assert abs(prob.dt - float(dt)) <= 1e-14 * float(dt)
        prob.close()
