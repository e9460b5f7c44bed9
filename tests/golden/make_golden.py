"""Generate the golden fixtures in tests/golden/ from a build of the
reference's own C sources (oracle/_ref/libnrpyell_ref_v4.so, built by
oracle/build.py from NRPyElliptic_Ccodes/*.c).

Run in a checkout that has the reference sources:
    python tests/golden/make_golden.py
    python tests/golden/make_golden.py --add-extrap   (only adds the
        extrapolation-branch arrays to the existing ops_*.npz fixtures)

Fixtures (numpy .npz):
  ops_<case>.npz      set-up outputs (params, xx, rfm tables, auxevol, dt,
                      boundary maps) and one application of each hot-path
                      function to a seeded random state: rhs_eval, the
                      radiation + inner BC, residual_all_points,
                      L2_norm_of_gf, 1 and 10 MoL steps, a 40-step
                      residual history from the zero guess, and the
                      extrapolation branch: apply_bcs_outerextrap_and_inner
                      on the random state and one MoL step with
                      outer_bc_type = EXTRAPOLATION_OUTER_BCS.
  relax_shipped_64x64x8.npz        full relaxation of the reference's shipped
                      puncture set to log10 L2 <= -10 (history + converged uu).
  relax_quasicircular_128x128x16.npz  relaxation of the quasi-circular pair to
                      log10 L2 <= -10 (history + converged uu on two planes).
  bcmaps.npz          boundary-map counts and checksums for the production grids.
"""
import ctypes as C
import hashlib
import os
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

from nrpyelliptic_b200 import abi  # noqa: E402
from nrpyelliptic_b200.problem import CONFIGS, SHIPPED_PUNCTURES, Config, Punctures, set_physical_params  # noqa: E402
from oracle import build as obuild  # noqa: E402

OUT = os.path.dirname(os.path.abspath(__file__))
P = C.POINTER
XX = abi.PREAL * 3


def load_ref(isa="v4"):
    obuild.build_ref()
    lib = C.CDLL(obuild.ref_lib_path(isa))
    abi.declare_reference_api(lib)
    lib.refh_setup.restype = C.c_double
    lib.refh_setup.argtypes = [P(abi.griddata_struct), P(C.c_int), P(abi.paramstruct), C.c_double]
    lib.refh_free.argtypes = [P(abi.griddata_struct)]
    lib.refh_relax.restype = C.c_int
    lib.refh_relax.argtypes = [P(abi.griddata_struct), C.c_double, C.c_double, C.c_int, C.c_double, abi.PREAL,
                               P(C.c_int)]
    lib.set_Cparameters_to_default.argtypes = [P(abi.paramstruct)]
    return lib


def setup(lib, cfg):
    phys = abi.paramstruct()
    lib.set_Cparameters_to_default(C.byref(phys))
    set_physical_params(phys, cfg)
    g = abi.griddata_struct()
    nxx = (C.c_int * 3)(*cfg.Nxx)
    dt = lib.refh_setup(C.byref(g), nxx, C.byref(phys), cfg.CFL)
    return g, dt


def arr(ptr, n):
    return np.ctypeslib.as_array(ptr, shape=(n,)).copy()


def dims(g):
    p = g.params
    N = (p.Nxx_plus_2NGHOSTS0, p.Nxx_plus_2NGHOSTS1, p.Nxx_plus_2NGHOSTS2)
    return N, N[0] * N[1] * N[2]


def bc_tables(g):
    b = g.bcstruct
    ni = b.bc_info.num_inner_boundary_points
    inner = np.ctypeslib.as_array(C.cast(b.inner_bc_array, P(C.c_int8)), shape=(ni * C.sizeof(abi.innerpt_bc_struct),))
    inner = inner.view(np.dtype({"names": ["dst", "src", "par"], "formats": ["<i4", "<i4", ("i1", 10)],
                                 "offsets": [0, 4, 8], "itemsize": C.sizeof(abi.innerpt_bc_struct)})).copy()
    counts = np.array([[b.bc_info.num_pure_outer_boundary_points[gz][d] for d in range(3)] for gz in range(5)])
    outer = []
    for gz in range(5):
        for d in range(3):
            n = counts[gz, d]
            if n:
                raw = np.ctypeslib.as_array(C.cast(b.pure_outer_bc_array[d + 3 * gz], P(C.c_int8)),
                                            shape=(n * C.sizeof(abi.outerpt_bc_struct),))
                rec = raw.view(np.dtype({"names": ["i0", "i1", "i2", "F0", "F1", "F2"],
                                         "formats": ["<i2", "<i2", "<i2", "i1", "i1", "i1"],
                                         "offsets": [0, 2, 4, 6, 7, 8],
                                         "itemsize": C.sizeof(abi.outerpt_bc_struct)})).copy()
                for r in rec:
                    outer.append((gz, d, r["i0"], r["i1"], r["i2"], r["F0"], r["F1"], r["F2"]))
    loop_bounds = np.array(
        [[[b.bc_info.bc_loop_bounds[gz][f][i] for i in range(6)] for f in range(6)] for gz in range(5)], dtype=np.int32)
    return inner, counts, np.array(outer, dtype=np.int32).reshape(-1, 8), loop_bounds


def params_bytes(p):
    return np.frombuffer(bytes(p), dtype=np.uint8).copy()


def make_ops_case(lib, cfg, seed):
    g, dt = setup(lib, cfg)
    N, Ntot = dims(g)
    p = g.params
    out = {"Nxx": np.array(cfg.Nxx), "dt": dt, "params": params_bytes(p), "cfl": cfg.CFL}
    out["xx0"], out["xx1"], out["xx2"] = (arr(g.xx[i], N[i]) for i in range(3))
    for name in abi.RFM_FIELDS:
        n = N[0] if ("xx0" in name and "xx1" not in name) else (N[1] if "xx1" in name and "xx0" not in name else N[0] * N[1])
        out["rfm_" + name] = arr(getattr(g.rfmstruct, name), n)
    aux = arr(g.gridfuncs.auxevol_gfs, 3 * Ntot)
    # ghost-zone wavespeeds are left unset by the reference; record interior only
    ws = aux[2 * Ntot:].reshape(N[2], N[1], N[0])
    mask = np.zeros((N[2], N[1], N[0]), bool)
    mask[5:-5, 5:-5, 5:-5] = True
    ws[~mask] = 0.0
    out["aux"] = aux
    out["c_OB"] = p.uu_wavespeed_at_OB
    inner, counts, outer, lb = bc_tables(g)
    out["inner"], out["outer_counts"], out["outer"], out["loop_bounds"] = inner, counts, outer, lb

    rng = np.random.default_rng(seed)
    y = np.empty(2 * Ntot)
    y[:Ntot] = rng.uniform(-0.2, 0.2, Ntot)
    y[Ntot:] = rng.uniform(-1.0, 1.0, Ntot)
    out["y_random"] = y.copy()
    yc = y.copy()
    lib.apply_bcs_inner_only(C.byref(g.params), C.byref(g.bcstruct), yc.ctypes.data_as(abi.PREAL))
    out["y_consistent"] = yc.copy()

    rhs = np.full(2 * Ntot, np.nan)
    lib.rhs_eval(C.byref(g.params), C.byref(g.rfmstruct), g.gridfuncs.auxevol_gfs, y.ctypes.data_as(abi.PREAL),
                 rhs.ctypes.data_as(abi.PREAL))
    out["rhs"] = rhs.copy()
    rhs_c = np.full(2 * Ntot, np.nan)
    lib.rhs_eval(C.byref(g.params), C.byref(g.rfmstruct), g.gridfuncs.auxevol_gfs, yc.ctypes.data_as(abi.PREAL),
                 rhs_c.ctypes.data_as(abi.PREAL))
    cw = (C.c_double * 2)(p.uu_wavespeed_at_OB, p.vv_wavespeed_at_OB)
    fi = (C.c_double * 2)(0.0, 0.0)
    lib.apply_bcs_outerradiation_and_inner(C.byref(g.params), C.byref(g.bcstruct), g.xx, cw, fi,
                                           yc.ctypes.data_as(abi.PREAL), rhs_c.ctypes.data_as(abi.PREAL))
    out["rhs_bc"] = rhs_c.copy()
    res = np.full(2 * Ntot, np.nan)
    lib.residual_all_points(C.byref(g.params), C.byref(g.rfmstruct), g.gridfuncs.auxevol_gfs,
                            yc.ctypes.data_as(abi.PREAL), res.ctypes.data_as(abi.PREAL))
    out["residual"] = res[:Ntot].copy()
    out["l2_R100"] = lib.L2_norm_of_gf(C.byref(g.params), 0, 100.0, g.xx, res.ctypes.data_as(abi.PREAL))
    out["l2_Rinf"] = lib.L2_norm_of_gf(C.byref(g.params), 0, 1e300, g.xx, res.ctypes.data_as(abi.PREAL))

    # MoL steps from the ghost-consistent random state
    ydev = g.gridfuncs.y_n_gfs
    C.memmove(ydev, yc.ctypes.data, yc.nbytes)
    lib.MoL_step_forward_in_time(C.byref(g), dt)
    out["y_step1"] = arr(ydev, 2 * Ntot)
    for _ in range(9):
        lib.MoL_step_forward_in_time(C.byref(g), dt)
    out["y_step10"] = arr(ydev, 2 * Ntot)

    # relaxation history from the zero guess
    C.memset(ydev, 0, 2 * Ntot * 8)
    hist = np.zeros(41)
    steps = C.c_int(0)
    lib.refh_relax(C.byref(g), dt, -30.0, 40, cfg.R_L2, hist.ctypes.data_as(abi.PREAL), C.byref(steps))
    out["relax_history40"] = hist
    out["y_relax40"] = arr(ydev, 2 * Ntot)
    lib.refh_free(C.byref(g))
    out.update(extrap_case(lib, cfg, out["y_random"], out["y_consistent"]))
    return out


def extrap_case(lib, cfg, y_random, y_consistent):
    """The extrapolation outer-BC branch of the reference
    (apply_bcs_outerextrap_and_inner.c:15-75 and its call sites in
    MoL_step_forward_in_time.c when outer_bc_type == EXTRAPOLATION_OUTER_BCS)."""
    g, dt = setup(lib, cfg)
    N, Ntot = dims(g)
    out = {}
    y = y_random.copy()
    lib.apply_bcs_outerextrap_and_inner(C.byref(g.params), C.byref(g.bcstruct), y.ctypes.data_as(abi.PREAL))
    out["y_extrap"] = y
    g.params.outer_bc_type = abi.EXTRAPOLATION_OUTER_BCS
    ydev = g.gridfuncs.y_n_gfs
    C.memmove(ydev, y_consistent.ctypes.data, y_consistent.nbytes)
    lib.MoL_step_forward_in_time(C.byref(g), dt)
    out["y_step1_extrap"] = arr(ydev, 2 * Ntot)
    lib.refh_free(C.byref(g))
    return out


def make_relax(lib, cfg, planes_only=False, max_steps=40000):
    g, dt = setup(lib, cfg)
    N, Ntot = dims(g)
    hist = np.zeros(max_steps + 1)
    steps = C.c_int(0)
    t0 = time.time()
    rc = lib.refh_relax(C.byref(g), dt, -10.0, max_steps, cfg.R_L2, hist.ctypes.data_as(abi.PREAL), C.byref(steps))
    wall = time.time() - t0
    n = steps.value
    uu = arr(g.gridfuncs.y_n_gfs, Ntot).reshape(N[2], N[1], N[0])
    out = {"Nxx": np.array(cfg.Nxx), "dt": dt, "converged": int(rc == 0), "steps": n, "history": hist[:n + 1],
           "wall_s_8threads": wall, "params": params_bytes(g.params)}
    if planes_only:
        out["uu_plane_i2_lo"] = uu[5, 5:-5, 5:-5].copy()
        out["uu_plane_i2_mid"] = uu[N[2] // 2, 5:-5, 5:-5].copy()
    else:
        out["uu_interior"] = uu[5:-5, 5:-5, 5:-5].copy()
    lib.refh_free(C.byref(g))
    return out


def bcmap_digest(lib, cfg):
    g, dt = setup(lib, cfg)
    inner, counts, outer, lb = bc_tables(g)
    pairs = np.stack([inner["dst"], inner["src"]], axis=1).astype(np.int64)
    pairs = pairs[np.argsort(pairs[:, 0])]
    h = hashlib.sha256(pairs.tobytes()).hexdigest()
    lib.refh_free(C.byref(g))
    return len(inner), counts, h, dt


def ops_cases():
    return {
        "shipped_16x8x6": (Config("g", (16, 8, 6), SHIPPED_PUNCTURES, CFL=0.5), 1),
        "unequal_24x16x8": (Config("g", (24, 16, 8),
                                   Punctures(0.8, 0.2, (0, 0, 1.2), (0, 0, -4.8), (0, 0.06, 0), (0, -0.06, 0),
                                             (0, 0, 0.1), (0.05, 0, -0.03)), bScale=6.0), 2),
    }


def add_extrap(lib):
    """Adds the extrapolation-branch arrays to the existing ops fixtures
    (same configurations, the fixtures' own random states)."""
    for name, (cfg, _) in ops_cases().items():
        path = os.path.join(OUT, "ops_%s.npz" % name)
        d = dict(np.load(path))
        d.update(extrap_case(lib, cfg, d["y_random"], d["y_consistent"]))
        np.savez_compressed(path, **d)
        print("extrap", name)


def main():
    lib = load_ref("v4")
    if "--add-extrap" in sys.argv:
        add_extrap(lib)
        return
    t0 = time.time()
    cases = ops_cases()
    for name, (cfg, seed) in cases.items():
        d = make_ops_case(lib, cfg, seed)
        np.savez_compressed(os.path.join(OUT, "ops_%s.npz" % name), **d)
        print("ops", name, "%.1fs" % (time.time() - t0))
    digests = {}
    for name, grid in [("64x64x8", (64, 64, 8)), ("96x96x12", (96, 96, 12)), ("128x128x16", (128, 128, 16)),
                       ("192x192x24", (192, 192, 24)), ("256x256x32", (256, 256, 32))]:
        cfg = Config("g", grid)
        n, counts, h, dt = bcmap_digest(lib, cfg)
        digests[name] = (n, counts, h, dt)
        print("bcmap", name, n, counts[:, 0].tolist(), h[:12], dt)
    np.savez_compressed(os.path.join(OUT, "bcmaps.npz"),
                        names=np.array(list(digests)), n_inner=np.array([v[0] for v in digests.values()]),
                        outer_counts=np.array([v[1] for v in digests.values()]),
                        sha256=np.array([v[2] for v in digests.values()]),
                        dt=np.array([v[3] for v in digests.values()]))
    d = make_relax(lib, CONFIGS["shipped_64x64x8"])
    np.savez_compressed(os.path.join(OUT, "relax_shipped_64x64x8.npz"), **d)
    print("relax shipped", d["steps"], d["converged"], "%.1fs" % d["wall_s_8threads"])
    if "--skip-c1" not in sys.argv:
        d = make_relax(lib, CONFIGS["quasicircular_128x128x16"], planes_only=True)
        np.savez_compressed(os.path.join(OUT, "relax_quasicircular_128x128x16.npz"), **d)
        print("relax quasicircular", d["steps"], d["converged"], "%.1fs" % d["wall_s_8threads"])


if __name__ == "__main__":
    main()
