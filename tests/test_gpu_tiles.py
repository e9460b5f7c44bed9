"""Every tile shape of the fused substep kernel (direct, prefetching,
shared-memory planes, marching along i2) against the reference's
golden steps and against each other.

The shapes differ only in how points are assigned to threads and how the
stencil is fetched (through L1, staged in shared memory, or copied ahead by
asynchronous copies); the arithmetic
per point is the same, so RK4 steps are bit-identical across shapes.  The L2
norm of the stop test sums per-tile partials, whose number depends on the
shape, so relaxation histories agree to rounding and step counts to +-1.
The golden grids have partial tiles along every direction (24 x 16 x 8 and
16 x 8 x 6 against 32-point rows and up to 8 planes per tile).
"""
import ctypes as C

import numpy as np
import pytest
from _util import device_grid, golden_grid, load_golden, ptr, relmax

from nrpyelliptic_b200 import _lib
from nrpyelliptic_b200.problem import CONFIGS, DeviceState, Problem

pytestmark = pytest.mark.gpu
CASES = ["ops_shipped_16x8x6.npz", "ops_unequal_24x16x8.npz"]


@pytest.fixture(scope="module")
def lib():
    lib = _lib.load()
    lib.nrpyell_clear_status()
    yield lib
    lib.nrpyell_set_tile(-1)


def tiles(lib):
    out = []
    for t in range(lib.nrpyell_num_tiles()):
        by, p, st = C.c_int(), C.c_int(), C.c_int()
        assert lib.nrpyell_tile_info(t, C.byref(by), C.byref(p), C.byref(st)) == 0
        out.append((t, by.value, p.value, st.value))
    return out


def test_tile_table_has_every_kind(lib):
    tl = tiles(lib)
    assert {k for *_, k in tl} == {0, 2, 4, 5}
    assert lib.nrpyell_tile_info(len(tl), None, None, None) == -1


@pytest.mark.parametrize("case", CASES)
def test_every_tile_gives_identical_steps(lib, case):
    gold = load_golden(case)
    hg = golden_grid(gold)
    dt = float(gold["dt"])
    results = {}
    lib.nrpyell_set_step_mode(0)
    try:
        for t, by, p, kind in tiles(lib):
            lib.nrpyell_set_tile(t)
            g, bufs = device_grid(lib, hg, gold["y_consistent"])
            for _ in range(10):
                lib.MoL_step_forward_in_time(C.byref(g), dt)
            _lib.check(lib)
            y = bufs["y_n"].get()
            assert relmax(y, gold["y_step10"]) < 1e-12, (t, by, p, kind)
            results[t] = y
    finally:
        lib.nrpyell_set_tile(-1)
        lib.nrpyell_set_step_mode(0)
    base = results[0]
    for t, y in results.items():
        np.testing.assert_array_equal(y, base, err_msg="tile %d" % t)


def test_every_tile_relaxes_to_the_same_solution(lib):
    gold = load_golden("relax_shipped_64x64x8.npz")
    prob = Problem(CONFIGS["shipped_64x64x8"])
    N = prob.N
    ref = gold["uu_interior"]
    try:
        for t, by, p, kind in tiles(lib):
            lib.nrpyell_set_tile(t)
            ds = DeviceState(prob)
            steps = C.c_int(0)
            fin = C.c_double(0)
            hist = np.zeros(4001)
            rc = lib.nrpyell_relax(C.byref(ds.g), prob.dt, -10.0, 4000, 100.0, C.byref(steps), C.byref(fin),
                                   ptr(hist))
            _lib.check(lib)
            assert rc == 0 and fin.value <= -10.0, t
            assert abs(steps.value - int(gold["steps"])) <= 1, (t, steps.value)
            n = min(steps.value, int(gold["steps"])) + 1
            np.testing.assert_allclose(hist[:n], gold["history"][:n], rtol=0, atol=1e-8)
            uu = ds.download("y_n")[:prob.Ntot].reshape(N[2], N[1], N[0])[5:-5, 5:-5, 5:-5]
            assert np.max(np.abs(uu - ref)) <= 1e-10 * np.max(np.abs(ref)), t
            ds.free()
    finally:
        lib.nrpyell_set_tile(-1)


def test_correction_form_tiles_in_mixed_precision(lib):
    """The FP32 correction form of the mixed-precision driver on every shape
    that runs it: the marching shapes and the 8-warp direct shapes."""
    gold = load_golden("relax_shipped_64x64x8.npz")
    prob = Problem(CONFIGS["shipped_64x64x8"])
    N = prob.N
    ref = gold["uu_interior"]
    try:
        for t, by, p, kind in tiles(lib):
            if not (kind == 5 or (kind == 0 and by == 8)):
                continue
            lib.nrpyell_set_tile(t)
            ds = DeviceState(prob)
            n32, n64 = C.c_int(0), C.c_int(0)
            fin = C.c_double(0)
            hist = np.zeros(6001)
            rc = lib.nrpyell_relax_mixed(C.byref(ds.g), prob.dt, -10.0, -10.0, 64, 6000, 100.0, C.byref(n32),
                                         C.byref(n64), C.byref(fin), ptr(hist))
            _lib.check(lib)
            assert rc == 0 and fin.value <= -10.0 and n32.value > 0, t
            uu = ds.download("y_n")[:prob.Ntot].reshape(N[2], N[1], N[0])[5:-5, 5:-5, 5:-5]
            assert np.max(np.abs(uu - ref)) / np.max(np.abs(ref)) < 1e-8, t
            ds.free()
    finally:
        lib.nrpyell_set_tile(-1)


def test_programmatic_launch_gives_identical_relaxations(lib):
    """The substep kernels launched with programmatic stream serialization
    (each waits in griddepcontrol.wait for the previous substep) and launched
    plainly give the same relaxation, bit for bit."""
    prob = Problem(CONFIGS["shipped_64x64x8"])
    out = {}
    try:
        for on in (1, 0):
            lib.nrpyell_set_programmatic_launch(on)
            assert lib.nrpyell_get_programmatic_launch() == on
            ds = DeviceState(prob)
            steps, fin = C.c_int(0), C.c_double(0)
            hist = np.zeros(4001)
            rc = lib.nrpyell_relax(C.byref(ds.g), prob.dt, -10.0, 4000, 100.0, C.byref(steps), C.byref(fin),
                                   ptr(hist))
            _lib.check(lib)
            assert rc == 0
            out[on] = (steps.value, fin.value, hist.copy(), ds.download("y_n"))
            ds.free()
    finally:
        lib.nrpyell_set_programmatic_launch(1)
    assert out[1][0] == out[0][0] and out[1][1] == out[0][1]
    np.testing.assert_array_equal(out[1][2], out[0][2])
    np.testing.assert_array_equal(out[1][3], out[0][3])
