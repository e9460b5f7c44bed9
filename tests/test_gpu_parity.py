"""GPU parity: the CUDA library through its C ABI against the reference's
golden outputs and the CPU oracle, on the same inputs.

Tolerances:
  rhs_eval, residual_all_points: bit-for-bit (reference operation order)
  radiation BC, L2: 1e-12 relative to the array maximum / 1e-13 in log10
  MoL steps, reference-order mode: 1e-13 (1 step) .. 1e-12 (10 steps) relative to max
  MoL steps, fused mode (folded metric factors): 1e-12 relative to max
  converged solution: 1e-10 x max|uu| (north-star criterion), same step count +-1
"""
import ctypes as C
import os
import subprocess

import numpy as np
import pytest
from _util import ROOT, Dev, device_grid, golden_grid, interior_mask, load_golden, oracle, problem_grid, ptr, relmax

from nrpyelliptic_b200 import _lib, abi
from nrpyelliptic_b200.problem import CONFIGS, DeviceState, Problem

pytestmark = pytest.mark.gpu
CASES = ["ops_shipped_16x8x6.npz", "ops_unequal_24x16x8.npz"]


@pytest.fixture(scope="module")
def lib():
    lib = _lib.load()
    lib.nrpyell_clear_status()
    return lib


@pytest.mark.parametrize("case", CASES)
def test_rhs_eval_bitwise_vs_reference(lib, case):
    gold = load_golden(case)
    hg = golden_grid(gold)
    aux = Dev(lib, hg.aux)
    y = Dev(lib, gold["y_random"])
    rhs = Dev(lib, np.full(2 * hg.Ntot, np.nan))
    lib.rhs_eval(C.byref(hg.params), C.byref(hg.rfm), aux.ptr, y.ptr, rhs.ptr)
    _lib.check(lib)
    out = rhs.get()
    m = np.tile(interior_mask(hg.N), 2)
    np.testing.assert_array_equal(out[m], gold["rhs"][m])
    assert np.all(np.isnan(out[~m]))  # ghost zones untouched, as in the reference


@pytest.mark.parametrize("case", CASES)
def test_residual_bitwise_and_l2_vs_reference(lib, case):
    gold = load_golden(case)
    hg = golden_grid(gold)
    aux = Dev(lib, hg.aux)
    y = Dev(lib, gold["y_consistent"])
    res = Dev(lib, np.full(2 * hg.Ntot, np.nan))
    lib.residual_all_points(C.byref(hg.params), C.byref(hg.rfm), aux.ptr, y.ptr, res.ptr)
    _lib.check(lib)
    out = res.get()
    m = interior_mask(hg.N)
    np.testing.assert_array_equal(out[:hg.Ntot][m], gold["residual"][m])
    l2 = lib.L2_norm_of_gf(C.byref(hg.params), 0, 100.0, hg.xx, res.ptr)
    assert abs(l2 - float(gold["l2_R100"])) < 1e-13
    l2i = lib.L2_norm_of_gf(C.byref(hg.params), 0, 1e300, hg.xx, res.ptr)
    assert abs(l2i - float(gold["l2_Rinf"])) < 1e-13


@pytest.mark.parametrize("case", CASES)
def test_radiation_bc_vs_reference(lib, case):
    gold = load_golden(case)
    hg = golden_grid(gold)
    aux = Dev(lib, hg.aux)
    y = Dev(lib, gold["y_consistent"])
    rhs = Dev(lib, np.full(2 * hg.Ntot, np.nan))
    lib.rhs_eval(C.byref(hg.params), C.byref(hg.rfm), aux.ptr, y.ptr, rhs.ptr)
    cw = (C.c_double * 2)(hg.params.uu_wavespeed_at_OB, hg.params.vv_wavespeed_at_OB)
    fi = (C.c_double * 2)(0.0, 0.0)
    lib.apply_bcs_outerradiation_and_inner(C.byref(hg.params), C.byref(hg.bc), hg.xx, cw, fi, y.ptr, rhs.ptr)
    _lib.check(lib)
    out = rhs.get()
    ref = gold["rhs_bc"]
    assert not np.any(np.isnan(out))
    for gf in range(2):
        sl = slice(gf * hg.Ntot, (gf + 1) * hg.Ntot)
        assert relmax(out[sl], ref[sl]) < 1e-12


@pytest.mark.parametrize("case", CASES)
def test_inner_only_and_extrapolation_vs_reference(lib, case):
    """apply_bcs_inner_only bit for bit and apply_bcs_outerextrap_and_inner
    (apply_bcs_outerextrap_and_inner.c:15-75) against the reference build's
    outputs on the same random state."""
    gold = load_golden(case)
    hg = golden_grid(gold)
    y0 = gold["y_random"].copy()
    d = Dev(lib, y0)
    lib.apply_bcs_inner_only(C.byref(hg.params), C.byref(hg.bc), d.ptr)
    _lib.check(lib)
    np.testing.assert_array_equal(d.get(), gold["y_consistent"])
    d.set(y0)
    lib.apply_bcs_outerextrap_and_inner(C.byref(hg.params), C.byref(hg.bc), d.ptr)
    _lib.check(lib)
    assert relmax(d.get(), gold["y_extrap"]) < 1e-15


@pytest.mark.parametrize("mode", [0, 1])
@pytest.mark.parametrize("case", CASES)
def test_mol_step_extrapolation_bc_vs_reference(lib, case, mode):
    """One MoL step with outer_bc_type = EXTRAPOLATION_OUTER_BCS: both step
    modes take the reference-order path for this BC type."""
    gold = load_golden(case)
    hg = golden_grid(gold)
    hg.params.outer_bc_type = abi.EXTRAPOLATION_OUTER_BCS
    g, bufs = device_grid(lib, hg, gold["y_consistent"])
    lib.nrpyell_set_step_mode(mode)
    try:
        lib.MoL_step_forward_in_time(C.byref(g), float(gold["dt"]))
        _lib.check(lib)
        assert relmax(bufs["y_n"].get(), gold["y_step1_extrap"]) < 1e-13
    finally:
        lib.nrpyell_set_step_mode(0)


@pytest.mark.parametrize("mode,tol1,tol10", [(1, 1e-13, 1e-12), (0, 1e-12, 1e-12)])
@pytest.mark.parametrize("case", CASES)
def test_mol_steps_vs_reference(lib, case, mode, tol1, tol10):
    gold = load_golden(case)
    hg = golden_grid(gold)
    g, bufs = device_grid(lib, hg, gold["y_consistent"])
    dt = float(gold["dt"])
    lib.nrpyell_set_step_mode(mode)
    try:
        lib.MoL_step_forward_in_time(C.byref(g), dt)
        _lib.check(lib)
        assert relmax(bufs["y_n"].get(), gold["y_step1"]) < tol1
        for _ in range(9):
            lib.MoL_step_forward_in_time(C.byref(g), dt)
        _lib.check(lib)
        assert relmax(bufs["y_n"].get(), gold["y_step10"]) < tol10
    finally:
        lib.nrpyell_set_step_mode(0)


@pytest.mark.parametrize("mode", [0, 1])
def test_mol_steps_production_grid_vs_oracle(lib, mode):
    """128x128x16 quasi-circular set-up, seeded random ghost-consistent state,
    20 RK4 steps on the GPU and in the oracle."""
    prob = Problem(CONFIGS["quasicircular_128x128x16"])
    hg = problem_grid(prob)
    o = oracle()
    rng = np.random.default_rng(7)
    y = np.concatenate([rng.uniform(-0.1, 0.1, hg.Ntot), rng.uniform(-0.5, 0.5, hg.Ntot)])
    o.oracle_apply_bcs_inner_only(C.byref(hg.params), C.byref(hg.bc), ptr(y))
    hg.bufs["y_n"][:] = y
    g_cpu = hg.griddata()
    g, bufs = device_grid(lib, hg, y)
    lib.nrpyell_set_step_mode(mode)
    try:
        for _ in range(20):
            o.oracle_MoL_step_forward_in_time(C.byref(g_cpu), prob.dt)
            lib.MoL_step_forward_in_time(C.byref(g), prob.dt)
        _lib.check(lib)
        got = bufs["y_n"].get()
    finally:
        lib.nrpyell_set_step_mode(0)
    assert relmax(got, hg.bufs["y_n"]) < 1e-12


def test_relax_shipped_64x64x8_matches_reference_solution(lib):
    gold = load_golden("relax_shipped_64x64x8.npz")
    prob = Problem(CONFIGS["shipped_64x64x8"])
    ds = DeviceState(prob)
    steps = C.c_int(0)
    fin = C.c_double(0)
    hist = np.zeros(4001)
    rc = lib.nrpyell_relax(C.byref(ds.g), prob.dt, -10.0, 4000, 100.0, C.byref(steps), C.byref(fin), ptr(hist))
    _lib.check(lib)
    assert rc == 0
    assert abs(steps.value - int(gold["steps"])) <= 1
    n = min(steps.value, int(gold["steps"])) + 1
    np.testing.assert_allclose(hist[:n], gold["history"][:n], rtol=0, atol=1e-8)
    N = prob.N
    uu = ds.download("y_n")[:prob.Ntot].reshape(N[2], N[1], N[0])[5:-5, 5:-5, 5:-5]
    ref = gold["uu_interior"]
    assert np.max(np.abs(uu - ref)) <= 1e-10 * np.max(np.abs(ref))
    ds.free()


def test_relax_quasicircular_128x128x16_matches_reference_solution(lib):
    gold = load_golden("relax_quasicircular_128x128x16.npz")
    prob = Problem(CONFIGS["quasicircular_128x128x16"])
    ds = DeviceState(prob)
    steps = C.c_int(0)
    fin = C.c_double(0)
    hist = np.zeros(8001)
    rc = lib.nrpyell_relax(C.byref(ds.g), prob.dt, -10.0, 8000, 100.0, C.byref(steps), C.byref(fin), ptr(hist))
    _lib.check(lib)
    assert rc == 0 and fin.value <= -10.0
    assert abs(steps.value - int(gold["steps"])) <= 1
    N = prob.N
    uu = ds.download("y_n")[:prob.Ntot].reshape(N[2], N[1], N[0])
    for key, i2 in (("uu_plane_i2_lo", 5), ("uu_plane_i2_mid", N[2] // 2)):
        ref = gold[key]
        assert np.max(np.abs(uu[i2, 5:-5, 5:-5] - ref)) <= 1e-10 * np.max(np.abs(ref))
    # the end-to-end host-buffer entry point gives the same solve
    y = prob.zero_state()
    steps2 = C.c_int(0)
    fin2 = C.c_double(0)
    rc2 = lib.nrpyell_relax_host(C.byref(prob.params), prob.xx, C.byref(prob.bc), C.byref(prob.rfm), ptr(prob.aux),
                                 ptr(y), prob.dt, -10.0, 8000, 100.0, C.byref(steps2), C.byref(fin2))
    _lib.check(lib)
    assert rc2 == 0 and steps2.value == steps.value
    np.testing.assert_array_equal(y, ds.download("y_n"))
    ds.free()


def test_equal_mass_at_rest_converges_immediately(lib):
    """A_ij = 0 and u = 0 is the exact solution: log10 L2 hits the 1e-16 clamp
    at n = 0 and no step is taken."""
    prob = Problem(CONFIGS["equal_mass_rest_64x64x8"])
    ds = DeviceState(prob)
    steps = C.c_int(-1)
    fin = C.c_double(0)
    rc = lib.nrpyell_relax(C.byref(ds.g), prob.dt, -10.0, 100, 100.0, C.byref(steps), C.byref(fin), None)
    _lib.check(lib)
    assert rc == 0 and steps.value == 0 and fin.value == -16.0
    assert not np.any(ds.download("y_n"))
    ds.free()


def test_host_memory_is_rejected_not_dereferenced(lib):
    gold = load_golden(CASES[0])
    hg = golden_grid(gold)
    y = gold["y_random"].copy()
    rhs = np.zeros_like(y)
    lib.nrpyell_clear_status()
    lib.rhs_eval(C.byref(hg.params), C.byref(hg.rfm), ptr(hg.aux), ptr(y), ptr(rhs))
    assert lib.nrpyell_last_status() != 0
    assert b"not device-accessible" in lib.nrpyell_last_error()
    lib.nrpyell_clear_status()
    assert not np.any(rhs)


def test_managed_allocators_and_dropin_step(lib):
    """MoL_malloc_* hand out managed memory that host code can fill in place,
    as the reference main.c does."""
    gold = load_golden(CASES[1])
    hg = golden_grid(gold)
    g = abi.griddata_struct()
    g.params = hg.params
    lib.MoL_malloc_y_n_gfs(C.byref(g.params), C.byref(g.gridfuncs))
    lib.MoL_malloc_non_y_n_gfs(C.byref(g.params), C.byref(g.gridfuncs))
    _lib.check(lib)
    for i in range(3):
        g.xx[i] = hg.xx[i]
    g.bcstruct = hg.bc
    g.rfmstruct = hg.rfm
    n = hg.Ntot
    np.ctypeslib.as_array(g.gridfuncs.y_n_gfs, shape=(2 * n,))[:] = gold["y_consistent"]
    np.ctypeslib.as_array(g.gridfuncs.auxevol_gfs, shape=(3 * n,))[:] = hg.aux
    assert C.addressof(g.gridfuncs.diagnostic_output_gfs.contents) == C.addressof(
        g.gridfuncs.y_nplus1_running_total_gfs.contents)
    lib.MoL_step_forward_in_time(C.byref(g), float(gold["dt"]))
    lib.nrpyell_synchronize()
    _lib.check(lib)
    got = np.ctypeslib.as_array(g.gridfuncs.y_n_gfs, shape=(2 * n,)).copy()
    assert relmax(got, gold["y_step1"]) < 1e-12
    lib.MoL_free_memory_y_n_gfs(C.byref(g.params), C.byref(g.gridfuncs))
    lib.MoL_free_memory_non_y_n_gfs(C.byref(g.params), C.byref(g.gridfuncs))
    _lib.check(lib)


def _run_playground(exe, cwd, args):
    env = dict(os.environ, OMP_NUM_THREADS=os.environ.get("OMP_NUM_THREADS", "8"))
    subprocess.run([exe] + args, cwd=cwd, check=True, env=env, stdout=subprocess.DEVNULL, timeout=600)
    return np.loadtxt(os.path.join(cwd, "output_NRPyElliptic", "residual_l2_norm.txt"))


def test_unmodified_main_c_links_and_matches_reference(tmp_path):
    """The reference main.c and set-up objects linked against this library
    (oracle/_ref/NRPyElliptic_Playground_gpu) print the same residual history
    as the all-CPU reference build of the same sources."""
    ref_exe = os.path.join(ROOT, "oracle", "_ref", "NRPyElliptic_Playground")
    gpu_exe = os.path.join(ROOT, "oracle", "_ref", "NRPyElliptic_Playground_gpu")
    if not (os.path.exists(ref_exe) and os.path.exists(gpu_exe)):
        pytest.skip("drop-in executables are built only where the reference sources exist")
    a = tmp_path / "cpu"
    b = tmp_path / "gpu"
    a.mkdir()
    b.mkdir()
    args = ["64", "64", "8", "300"]
    h_cpu = _run_playground(ref_exe, str(a), args)
    h_gpu = _run_playground(gpu_exe, str(b), args)
    assert h_cpu.shape == h_gpu.shape == (301, 3)
    np.testing.assert_array_equal(h_cpu[:, 0], h_gpu[:, 0])
    np.testing.assert_allclose(h_gpu[:, 2], h_cpu[:, 2], rtol=0, atol=1e-10)
    uu_cpu = np.loadtxt(a / "output_NRPyElliptic" / "uu_final_1D.txt")
    uu_gpu = np.loadtxt(b / "output_NRPyElliptic" / "uu_final_1D.txt")
    assert np.max(np.abs(uu_gpu[:, 1] - uu_cpu[:, 1])) <= 1e-12 * np.max(np.abs(uu_cpu[:, 1]))


def test_python_playground_writes_main_c_files(tmp_path):
    """python -m nrpyelliptic_b200.playground with --snapshots writes the same
    files as the reference executable, with the same coordinates and values
    within the parity tolerances."""
    ref_exe = os.path.join(ROOT, "oracle", "_ref", "NRPyElliptic_Playground")
    if not os.path.exists(ref_exe):
        pytest.skip("the reference executable is built only where the reference sources exist")
    a = tmp_path / "cpu"
    b = tmp_path / "gpu"
    a.mkdir()
    b.mkdir()
    args = ["32", "16", "8", "120"]
    _run_playground(ref_exe, str(a), args)
    from nrpyelliptic_b200 import playground
    assert playground.main(args + ["--snapshots", "--outdir", str(b)]) == 0
    ra, rb = a / "output_NRPyElliptic", b / "output_NRPyElliptic"
    names = sorted(str(p.relative_to(ra)) for p in ra.rglob("*") if p.is_file())
    assert names == sorted(str(p.relative_to(rb)) for p in rb.rglob("*") if p.is_file())
    for name in names:
        x, y = np.loadtxt(ra / name, ndmin=2), np.loadtxt(rb / name, ndmin=2)
        assert x.shape == y.shape, name
        if name == "residual_l2_norm.txt":
            np.testing.assert_array_equal(x[:, :2], y[:, :2])
            np.testing.assert_allclose(y[:, 2], x[:, 2], rtol=0, atol=1e-10)
            continue
        np.testing.assert_allclose(y[:, :-1], x[:, :-1], rtol=1e-14, atol=1e-12, err_msg=name)
        scale = max(np.max(np.abs(x[:, -1])), 1e-300)
        assert np.max(np.abs(y[:, -1] - x[:, -1])) <= 1e-10 * scale, name
