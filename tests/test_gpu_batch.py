"""Batched relaxation (nrpyell_relax_batch): several configurations on
grids of different sizes in one launch per substep give, configuration by
configuration, the same solution and step count as relaxing each alone with
the same tile shape."""
import ctypes as C

import numpy as np
import pytest
from _util import ptr

from nrpyelliptic_b200 import _lib
from nrpyelliptic_b200.batch import relax_batch
from nrpyelliptic_b200.problem import CONFIGS, DeviceState, Problem, sample_sweep, with_grid

pytestmark = pytest.mark.gpu
PLANES_8x1 = 15  # a shared-memory planes tile shape (kind 4)
MARCH_8x4 = 20  # a marching tile shape (kind 5)


@pytest.fixture(scope="module")
def lib():
    lib = _lib.load()
    lib.nrpyell_clear_status()
    yield lib
    lib.nrpyell_set_tile(-1)


def _alone(lib, prob, max_steps):
    ds = DeviceState(prob, lib=lib)
    steps, fin = C.c_int(0), C.c_double(0)
    hist = np.zeros(max_steps + 1)
    rc = lib.nrpyell_relax(C.byref(ds.g), prob.dt, -10.0, max_steps, prob.cfg.R_L2, C.byref(steps), C.byref(fin),
                           ptr(hist))
    _lib.check(lib)
    y = ds.download("y_n")
    ds.free()
    return rc, steps.value, fin.value, y


@pytest.mark.parametrize("tile", [PLANES_8x1, MARCH_8x4])
def test_batch_matches_single_runs(lib, tile):
    kind = C.c_int(-1)
    assert lib.nrpyell_tile_info(tile, None, None, C.byref(kind)) == 0 and kind.value in (4, 5)
    cfgs = [CONFIGS["shipped_64x64x8"], with_grid(CONFIGS["quasicircular_128x128x16"], (48, 48, 8)),
            with_grid(sample_sweep(4)[1], (40, 24, 6)), CONFIGS["equal_mass_rest_64x64x8"]]
    probs = [Problem(c, lib=lib) for c in cfgs]
    lib.nrpyell_set_tile(tile)
    try:
        rc, steps, finals, states = relax_batch(probs, tol=-10.0, max_steps=8000, lib=lib)
        assert rc == 0
        assert steps[3] == 0  # the head-on pair at rest is solved by the zero guess
        for i, p in enumerate(probs):
            rc1, s1, f1, y1 = _alone(lib, p, 8000)
            assert rc1 == 0
            assert steps[i] == s1, (cfgs[i].name, steps[i], s1)
            assert finals[i] == f1
            np.testing.assert_array_equal(states[i].download("y_n"), y1, err_msg=cfgs[i].name)
    finally:
        lib.nrpyell_set_tile(-1)
    for s in states:
        s.free()


def _alone_mixed(lib, prob, switch, fold, max_steps):
    ds = DeviceState(prob, lib=lib)
    n32, n64, fin = C.c_int(0), C.c_int(0), C.c_double(0)
    rc = lib.nrpyell_relax_mixed(C.byref(ds.g), prob.dt, -10.0, switch, fold, max_steps, prob.cfg.R_L2, C.byref(n32),
                                 C.byref(n64), C.byref(fin), None)
    _lib.check(lib)
    y = ds.download("y_n")
    ds.free()
    return rc, n32.value, n64.value, fin.value, y


@pytest.mark.parametrize("switch,fold,max_steps", [(-6.0, 64, 8000), (-10.0, 100, 8000), (-10.0, 48, 300)])
def test_batch_mixed_matches_single_mixed_runs(lib, switch, fold, max_steps):
    """nrpyell_relax_batch_mixed against nrpyell_relax_mixed configuration by
    configuration, with the same marching shape for both precisions: equal
    FP32 and FP64 step counts, final norms and y_n bit for bit (switch -6:
    FP32 stretches then an FP64 phase; -10: all steps FP32; max_steps 300:
    stops before convergence)."""
    from nrpyelliptic_b200.batch import relax_batch_mixed
    cfgs = [CONFIGS["shipped_64x64x8"], with_grid(CONFIGS["quasicircular_128x128x16"], (48, 48, 8)),
            with_grid(sample_sweep(4)[1], (40, 24, 6)), CONFIGS["equal_mass_rest_64x64x8"]]
    probs = [Problem(c, lib=lib) for c in cfgs]
    lib.nrpyell_set_tile(MARCH_8x4)
    try:
        rc, s32, s64, finals, states = relax_batch_mixed(probs, tol=-10.0, switch=switch, fold_every=fold,
                                                         max_steps=max_steps, lib=lib)
        not_conv = 0
        for i, p in enumerate(probs):
            rc1, a32, a64, f1, y1 = _alone_mixed(lib, p, switch, fold, max_steps)
            not_conv += rc1
            assert (s32[i], s64[i]) == (a32, a64), (cfgs[i].name, s32[i], s64[i], a32, a64)
            assert finals[i] == f1
            np.testing.assert_array_equal(states[i].download("y_n"), y1, err_msg=cfgs[i].name)
        assert rc == not_conv
        assert s32[3] == 0 and s64[3] == 0  # the head-on pair at rest is solved by the zero guess
        if max_steps == 300:
            assert np.all((s32 + s64 == 300) | (finals <= -10.0))
        else:
            assert rc == 0 and np.all(finals <= -10.0)
            if switch == -10.0:
                assert np.all(s64 == 0)
            else:
                assert np.all(s64[:3] > 0) and np.all(s32[:3] > 0)
    finally:
        lib.nrpyell_set_tile(-1)
    for s in states:
        s.free()


def test_batch_mixed_edge_cases(lib):
    """One configuration equals the single-grid driver; max_steps = 0 takes
    no step and reports the FP64 norm of the start; a fold_every outside
    1..4096 is rejected."""
    from nrpyelliptic_b200.batch import relax_batch_mixed
    prob = Problem(CONFIGS["shipped_64x64x8"], lib=lib)
    lib.nrpyell_set_tile(MARCH_8x4)
    try:
        rc, s32, s64, finals, states = relax_batch_mixed([prob], tol=-10.0, switch=-6.0, fold_every=100,
                                                         max_steps=8000, lib=lib)
        rc1, a32, a64, f1, y1 = _alone_mixed(lib, prob, -6.0, 100, 8000)
        assert rc == rc1 == 0 and (s32[0], s64[0]) == (a32, a64) and finals[0] == f1
        np.testing.assert_array_equal(states[0].download("y_n"), y1)
        states[0].free()
        rc, s32, s64, finals, states = relax_batch_mixed([prob], tol=-10.0, switch=-10.0, fold_every=100,
                                                         max_steps=0, lib=lib)
        assert rc == 1 and s32[0] == 0 and s64[0] == 0 and -8.0 < finals[0] < 0.0
        assert not np.any(states[0].download("y_n")[:prob.Ntot])
        for bad in (0, 4097):
            with pytest.raises(RuntimeError, match="fold_every"):
                relax_batch_mixed([prob], states, fold_every=bad, max_steps=10, lib=lib)
        states[0].free()
    finally:
        lib.nrpyell_set_tile(-1)


def test_batch_autotuned_tile_converges(lib):
    cfgs = [with_grid(c, (32, 32, 8)) for c in sample_sweep(6)]
    probs = [Problem(c, lib=lib) for c in cfgs]
    rc, steps, finals, states = relax_batch(probs, tol=-10.0, max_steps=20000, lib=lib)
    assert rc == 0 and np.all(finals <= -10.0) and np.all(steps > 0)
    for s in states:
        s.free()


def test_auxevol_on_the_gpu_matches_the_host_set_up(lib):
    """nrpyell_auxevol_device against the host restatement, each gridfunction
    within 1e-13 of its largest value (same closed forms, compiled for the
    device and for the host)."""
    from nrpyelliptic_b200 import abi
    for cfg in (CONFIGS["shipped_64x64x8"], with_grid(sample_sweep(3)[2], (48, 40, 8))):
        host = Problem(cfg, lib=lib)
        dev = Problem(cfg, lib=lib, host_aux=False)
        ds = DeviceState(dev, lib=lib)
        aux = ds.download("aux").reshape(abi.NUM_AUXEVOL_GFS, -1)
        ref = host.aux.reshape(abi.NUM_AUXEVOL_GFS, -1)
        for g in range(abi.NUM_AUXEVOL_GFS):
            assert np.max(np.abs(aux[g] - ref[g])) <= 1e-13 * np.max(np.abs(ref[g])), (cfg.name, g)
        assert dev.params.uu_wavespeed_at_OB == pytest.approx(host.params.uu_wavespeed_at_OB, rel=1e-14)
        ds.free()


def test_batch_on_sweep_grids_matches_single_runs(lib):
    """Three draws of the sweep distribution on its own grids (96x96x12 and
    128x128x16, tables and auxevol built on the GPU; the batch's shape
    autotuned) against single-grid relaxations: the same steps and the same
    bits of y_n (every tile shape gives identical steps, test_gpu_tiles); the
    final norms agree to rounding, as the L2 sum's partials follow the tile
    shape, which the two autotuners may choose differently."""
    cfgs = [c for c in sample_sweep(64) if c.Nxx in ((96, 96, 12), (128, 128, 16))][:3]
    assert len(cfgs) == 3
    probs = [Problem(c, lib=lib, host_aux=False, device_tables=True) for c in cfgs]
    rc, steps, finals, states = relax_batch(probs, tol=-10.0, max_steps=20000, lib=lib)
    assert rc == 0 and np.all(finals <= -10.0)
    for i, p in enumerate(probs):
        rc1, s1, f1, y1 = _alone(lib, p, 20000)
        assert rc1 == 0 and steps[i] == s1 and abs(finals[i] - f1) <= 1e-12, (cfgs[i].name, steps[i], s1)
        np.testing.assert_array_equal(states[i].download("y_n"), y1, err_msg=cfgs[i].name)
    for s in states:
        s.free()
