"""Shared helpers for the test suite: the oracle loader and reconstruction of
host-side griddata from golden fixtures."""
import ctypes as C
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

from nrpyelliptic_b200 import _lib, abi  # noqa: E402

GOLDEN = os.path.join(ROOT, "tests", "golden")
P = C.POINTER
XX = abi.PREAL * 3

_oracle = None


def oracle():
    """The CPU oracle (oracle/nrpyell_oracle.c), built on demand."""
    global _oracle
    if _oracle is None:
        from oracle import build as obuild
        path = obuild.build_oracle()
        lib = C.CDLL(path)
        sig = {
            "oracle_rhs_eval": (None, [P(abi.paramstruct), P(abi.rfm_struct), abi.PREAL, abi.PREAL, abi.PREAL]),
            "oracle_residual_all_points": (None, [P(abi.paramstruct), P(abi.rfm_struct), abi.PREAL, abi.PREAL,
                                                  abi.PREAL]),
            "oracle_apply_bcs_outerradiation_and_inner": (None, [P(abi.paramstruct), P(abi.bc_struct), XX, abi.PREAL,
                                                                 abi.PREAL, abi.PREAL, abi.PREAL]),
            "oracle_apply_bcs_inner_only": (None, [P(abi.paramstruct), P(abi.bc_struct), abi.PREAL]),
            "oracle_apply_bcs_outerextrap_and_inner": (None, [P(abi.paramstruct), P(abi.bc_struct), abi.PREAL]),
            "oracle_MoL_step_forward_in_time": (None, [P(abi.griddata_struct), C.c_double]),
            "oracle_L2_norm_of_gf": (C.c_double, [P(abi.paramstruct), C.c_int, C.c_double, XX, abi.PREAL]),
            "oracle_relax": (C.c_int, [P(abi.griddata_struct), C.c_double, C.c_double, C.c_int, C.c_double, abi.PREAL,
                                       P(C.c_int)]),
            "oracle_time_iterations": (C.c_double, [P(abi.griddata_struct), C.c_double, C.c_int, C.c_double]),
        }
        for name, (res, args) in sig.items():
            f = getattr(lib, name)
            f.restype = res
            f.argtypes = args
        _oracle = lib
    return _oracle


def ptr(a):
    return a.ctypes.data_as(abi.PREAL)


def load_golden(name):
    return dict(np.load(os.path.join(GOLDEN, name), allow_pickle=False))


class HostGrid:
    """Host-memory griddata rebuilt from arrays (golden fixture or Problem):
    keeps every numpy buffer alive for the lifetime of the object."""

    def __init__(self, params, xx, rfm, aux, inner, outer, outer_counts, loop_bounds=None):
        self.params = params
        self.N = (params.Nxx_plus_2NGHOSTS0, params.Nxx_plus_2NGHOSTS1, params.Nxx_plus_2NGHOSTS2)
        self.Ntot = self.N[0] * self.N[1] * self.N[2]
        self.xx_np = [np.ascontiguousarray(a, dtype=np.float64) for a in xx]
        self.xx = XX(*[ptr(a) for a in self.xx_np])
        self.rfm_np = {k: np.ascontiguousarray(v, dtype=np.float64) for k, v in rfm.items()}
        self.rfm = abi.rfm_struct(**{k: ptr(v) for k, v in self.rfm_np.items()})
        self.aux = np.ascontiguousarray(aux, dtype=np.float64).copy()
        # bc_struct
        ni = len(inner)
        self.inner_arr = (abi.innerpt_bc_struct * max(ni, 1))()
        for i in range(ni):
            e = self.inner_arr[i]
            e.dstpt = int(inner["dst"][i])
            e.srcpt = int(inner["src"][i])
            for t in range(10):
                e.parity[t] = int(inner["par"][i][t])
        self.bc = abi.bc_struct()
        self.bc.inner_bc_array = C.cast(self.inner_arr, P(abi.innerpt_bc_struct))
        self.bc.bc_info.num_inner_boundary_points = ni
        self.outer_arrs = []
        for gz in range(abi.NGHOSTS):
            for d in range(3):
                rows = outer[(outer[:, 0] == gz) & (outer[:, 1] == d)] if len(outer) else outer
                n = len(rows)
                arr = (abi.outerpt_bc_struct * max(n, 1))()
                for k, r in enumerate(rows):
                    arr[k].i0, arr[k].i1, arr[k].i2 = int(r[2]), int(r[3]), int(r[4])
                    arr[k].FACEX0, arr[k].FACEX1, arr[k].FACEX2 = int(r[5]), int(r[6]), int(r[7])
                self.outer_arrs.append(arr)
                self.bc.pure_outer_bc_array[d + 3 * gz] = C.cast(arr, P(abi.outerpt_bc_struct))
                self.bc.bc_info.num_pure_outer_boundary_points[gz][d] = n
                assert n == int(outer_counts[gz][d])
        if loop_bounds is not None:
            for gz in range(5):
                for f in range(6):
                    for i in range(6):
                        self.bc.bc_info.bc_loop_bounds[gz][f][i] = int(loop_bounds[gz][f][i])
        self.bufs = {k: np.zeros(2 * self.Ntot) for k in ("y_n", "acc", "k_odd", "k_even")}

    def griddata(self):
        g = abi.griddata_struct()
        g.params = self.params
        for i in range(3):
            g.xx[i] = self.xx[i]
        g.bcstruct = self.bc
        g.rfmstruct = self.rfm
        f = g.gridfuncs
        f.y_n_gfs = ptr(self.bufs["y_n"])
        f.y_nplus1_running_total_gfs = ptr(self.bufs["acc"])
        f.k_odd_gfs = ptr(self.bufs["k_odd"])
        f.k_even_gfs = ptr(self.bufs["k_even"])
        f.auxevol_gfs = ptr(self.aux)
        f.diagnostic_output_gfs = f.y_nplus1_running_total_gfs
        return g


def params_from_bytes(b):
    p = abi.paramstruct()
    C.memmove(C.byref(p), bytes(np.asarray(b, dtype=np.uint8)), C.sizeof(p))
    return p


def golden_grid(gold):
    p = params_from_bytes(gold["params"])
    rfm = {k[4:]: gold[k] for k in gold if k.startswith("rfm_")}
    return HostGrid(p, [gold["xx0"], gold["xx1"], gold["xx2"]], rfm, gold["aux"], gold["inner"], gold["outer"],
                    gold["outer_counts"], gold["loop_bounds"])


def problem_grid(prob):
    """HostGrid over a nrpyelliptic_b200.problem.Problem's set-up arrays."""
    b = prob.bc
    ni = b.bc_info.num_inner_boundary_points
    raw = np.ctypeslib.as_array(C.cast(b.inner_bc_array, P(C.c_int8)), shape=(ni * C.sizeof(abi.innerpt_bc_struct),))
    inner = raw.view(np.dtype({"names": ["dst", "src", "par"], "formats": ["<i4", "<i4", ("i1", 10)],
                               "offsets": [0, 4, 8], "itemsize": C.sizeof(abi.innerpt_bc_struct)})).copy()
    counts, outer = outer_records(b)
    return HostGrid(prob.params, prob.xx_arrays(), prob.rfm_arrays(), prob.aux, inner, outer, counts)


def outer_records(b):
    counts = np.array([[b.bc_info.num_pure_outer_boundary_points[gz][d] for d in range(3)] for gz in range(5)])
    rows = []
    for gz in range(5):
        for d in range(3):
            n = counts[gz, d]
            if n:
                raw = np.ctypeslib.as_array(C.cast(b.pure_outer_bc_array[d + 3 * gz], P(C.c_int8)),
                                            shape=(n * C.sizeof(abi.outerpt_bc_struct),))
                rec = raw.view(np.dtype({"names": ["i0", "i1", "i2", "F0", "F1", "F2"],
                                         "formats": ["<i2", "<i2", "<i2", "i1", "i1", "i1"],
                                         "offsets": [0, 2, 4, 6, 7, 8],
                                         "itemsize": C.sizeof(abi.outerpt_bc_struct)}))
                for r in rec:
                    rows.append((gz, d, r["i0"], r["i1"], r["i2"], r["F0"], r["F1"], r["F2"]))
    return counts, np.array(rows, dtype=np.int32).reshape(-1, 8)


def interior_mask(N):
    m = np.zeros((N[2], N[1], N[0]), bool)
    m[5:-5, 5:-5, 5:-5] = True
    return m.ravel()


def relmax(a, b):
    """max |a-b| / max |b|"""
    a, b = np.asarray(a), np.asarray(b)
    return float(np.max(np.abs(a - b)) / max(np.max(np.abs(b)), 1e-300))


class Dev:
    """A device buffer holding a numpy array."""

    def __init__(self, lib, a):
        self.lib = lib
        self.n = a.size
        self.p = lib.nrpyell_device_malloc(a.nbytes)
        _lib.check(lib)
        self.set(a)

    def set(self, a):
        a = np.ascontiguousarray(a, dtype=np.float64)
        self.lib.nrpyell_memcpy(self.p, a.ctypes.data, a.nbytes, 0)
        _lib.check(self.lib)

    def get(self):
        out = np.empty(self.n)
        self.lib.nrpyell_memcpy(out.ctypes.data, self.p, out.nbytes, 1)
        _lib.check(self.lib)
        return out

    @property
    def ptr(self):
        return C.cast(C.c_void_p(self.p), abi.PREAL)

    def __del__(self):
        try:
            self.lib.nrpyell_device_free(self.p)
        except Exception:
            pass


def device_grid(lib, hg, y0):
    """griddata_struct over device buffers: y_n = y0, aux from hg, zeroed RK buffers."""
    bufs = {"y_n": Dev(lib, y0), "acc": Dev(lib, np.zeros(2 * hg.Ntot)), "k_odd": Dev(lib, np.zeros(2 * hg.Ntot)),
            "k_even": Dev(lib, np.zeros(2 * hg.Ntot)), "aux": Dev(lib, hg.aux)}
    g = abi.griddata_struct()
    g.params = hg.params
    for i in range(3):
        g.xx[i] = hg.xx[i]
    g.bcstruct = hg.bc
    g.rfmstruct = hg.rfm
    f = g.gridfuncs
    f.y_n_gfs, f.y_nplus1_running_total_gfs = bufs["y_n"].ptr, bufs["acc"].ptr
    f.k_odd_gfs, f.k_even_gfs, f.auxevol_gfs = bufs["k_odd"].ptr, bufs["k_even"].ptr, bufs["aux"].ptr
    f.diagnostic_output_gfs = f.y_nplus1_running_total_gfs
    return g, bufs
