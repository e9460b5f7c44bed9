"""Device tables built on the GPU (nrpyell_setup_tables_device) -- the
reference-metric arrays and folded RHS weights, the inner-boundary map and
the pure outer points with their radiation geometry -- against the
reference's own set-up (golden fixtures generated by the reference build:
rfm_precompute_rfmstruct_define.c, bcstruct_set_up.c) and against the
library's host-built tables.

Tolerances: integer maps entry by entry; rfm arrays 1e-12 relative to the
golden arrays; geometry and folded weights 1e-12 relative to the host build
(device exp/sin/pow against the host's)."""
import ctypes as C
import hashlib

import numpy as np
import pytest
from _util import golden_grid, load_golden, relmax

from nrpyelliptic_b200 import _lib, abi
from nrpyelliptic_b200.problem import CONFIGS, Config, DeviceState, Problem, sample_sweep

pytestmark = pytest.mark.gpu
CASES = ["ops_shipped_16x8x6.npz", "ops_unequal_24x16x8.npz"]
RFM = {5: "f0_of_xx0", 6: "f0_of_xx0__D0", 7: "f0_of_xx0__DD00", 8: "f3_of_xx0", 9: "f3_of_xx0__D0",
       10: "f1_of_xx1", 11: "f1_of_xx1__D1", 12: "f2_of_xx0_xx1", 13: "f2_of_xx0_xx1__D0"}


@pytest.fixture(scope="module")
def lib():
    lib = _lib.load()
    lib.nrpyell_clear_status()
    return lib


def read(lib, params, xx, rfm, bc, what, n, dtype):
    out = np.zeros(n, dtype=dtype)
    got = lib.nrpyell_device_tables_read(C.byref(params), xx, C.byref(rfm), C.byref(bc), what,
                                         out.ctypes.data_as(C.c_void_p), n)
    _lib.check(lib)
    return out[:got]


@pytest.mark.parametrize("case", CASES)
def test_device_tables_match_the_reference_set_up(lib, case):
    gold = load_golden(case)
    hg = golden_grid(gold)
    if hg.params.Nxx0 < 12:
        pytest.skip("the device build needs Nxx0 >= 12 (the radiation column form)")
    rfm0, bc0 = abi.rfm_struct(), abi.bc_struct()  # empty: keys of the device-built tables
    assert lib.nrpyell_setup_tables_device(C.byref(hg.params), hg.xx, C.byref(rfm0), C.byref(bc0)) == 0
    _lib.check(lib)
    inner = gold["inner"]
    n = len(inner)
    pairs = read(lib, hg.params, hg.xx, rfm0, bc0, 0, 2 * n + 2, np.int32).reshape(-1, 2)
    assert len(pairs) == n
    np.testing.assert_array_equal(pairs[:, 0], inner["dst"])
    np.testing.assert_array_equal(pairs[:, 1], inner["src"])
    par = read(lib, hg.params, hg.xx, rfm0, bc0, 1, n, np.int8)
    np.testing.assert_array_equal(par, inner["par"][:, 0])
    outer = read(lib, hg.params, hg.xx, rfm0, bc0, 2, 8 * len(gold["outer"]) + 8, np.int32).reshape(-1, 8)
    np.testing.assert_array_equal(outer, gold["outer"])
    for what, name in RFM.items():
        dev = read(lib, hg.params, hg.xx, rfm0, bc0, what, 1 << 20, np.float64)
        assert relmax(dev, gold["rfm_" + name]) < 1e-12, name
    # geometry and folded weights against the host build from the golden structs
    for what, size in ((3, 6 * len(gold["outer"])), (4, 18 * hg.N[1]), (14, 6 * hg.N[0] * hg.N[1])):
        dev = read(lib, hg.params, hg.xx, rfm0, bc0, what, size, np.float64)
        host = read(lib, hg.params, hg.xx, hg.rfm, hg.bc, what, size, np.float64)
        assert len(dev) == size and relmax(dev, host) < 1e-12, what


def test_device_inner_maps_of_the_production_grids_match_the_reference(lib):
    """bcmaps.npz: the reference's inner-point count and the SHA-256 of its
    sorted (dst, src) pairs for every grid size of the configurations."""
    gold = load_golden("bcmaps.npz")
    for name, n_inner, sha in zip(gold["names"], gold["n_inner"], gold["sha256"]):
        nxx = tuple(int(x) for x in str(name).split("x"))
        prob = Problem(Config("g", nxx), lib=lib, host_aux=False, device_tables=True)
        rfm0, bc0 = abi.rfm_struct(), abi.bc_struct()
        assert lib.nrpyell_setup_tables_device(C.byref(prob.params), prob.xx, C.byref(rfm0), C.byref(bc0)) == 0
        pairs = read(lib, prob.params, prob.xx, rfm0, bc0, 0, 2 * int(n_inner) + 2, np.int32).reshape(-1, 2)
        assert len(pairs) == int(n_inner), name
        p64 = pairs.astype(np.int64)
        p64 = p64[np.argsort(p64[:, 0])]
        assert hashlib.sha256(p64.tobytes()).hexdigest() == str(sha), name
        prob.close()
        lib.nrpyell_release_tables()


def test_relaxation_on_device_tables_matches_host_tables(lib):
    """The shipped puncture set at 64x64x8 relaxed on device-built tables and
    on host-built tables: step counts within one (the folded weights agree to rounding), solutions
    within 1e-10 of max|uu|."""
    out = []
    for dev_tables in (False, True):
        prob = Problem(CONFIGS["shipped_64x64x8"], lib=lib, device_tables=dev_tables)
        ds = DeviceState(prob, lib=lib)
        st, fin = C.c_int(0), C.c_double(0)
        rc = lib.nrpyell_relax(C.byref(ds.g), prob.dt, -10.0, 4000, 100.0, C.byref(st), C.byref(fin), None)
        _lib.check(lib)
        assert rc == 0
        out.append((st.value, ds.download("y_n")))
        ds.free()
    assert abs(out[0][0] - out[1][0]) <= 1
    assert relmax(out[1][1], out[0][1]) < 1e-10


def test_batched_sweep_set_up_on_the_gpu(lib):
    """Set-up of 16 sweep configurations with device tables and auxevol on
    the GPU, against the host tables: the batched relaxation gives the same
    step counts (within one)."""
    import time
    from nrpyelliptic_b200.batch import relax_batch
    cfgs = sample_sweep(16, 20261203, grids=((96, 96, 12), (128, 128, 16)))
    res = {}
    for dev_tables in (False, True):
        lib.nrpyell_release_tables()
        lib.nrpyell_synchronize()
        t0 = time.perf_counter()
        probs = [Problem(c, lib=lib, host_aux=False, device_tables=dev_tables) for c in cfgs]
        states = [DeviceState(p, lib=lib) for p in probs]
        lib.nrpyell_synchronize()
        t_setup = time.perf_counter() - t0
        rc, steps, finals, _ = relax_batch(probs, states, max_steps=20000, lib=lib)
        assert rc == 0
        res[dev_tables] = (t_setup, steps)
        for s in states:
            s.free()
    print("set-up of 16 configurations: host tables %.3f s, device tables %.3f s" % (res[False][0], res[True][0]))
    assert np.max(np.abs(res[True][1] - res[False][1])) <= 1
