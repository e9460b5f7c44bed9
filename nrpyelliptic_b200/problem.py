"""Host-side set-up of one puncture configuration, mirroring the sequence of
the reference's main.c (NRPyElliptic_Ccodes/main.c:14-105):

  parameters -> SinhSymTP grid -> boundary maps -> time step -> reference-
  metric tables -> zero initial guess -> psi_background, A_ij A^ij ->
  wavespeed -> wavespeed at the outer boundary

All of it runs through libnrpyell_gpu.so's set-up entry points (host C).
The hot path then runs on the GPU through the reference-signature entry
points or the relaxation driver.
"""
import ctypes as C
from dataclasses import dataclass, field, replace

import numpy as np

from . import _lib, abi


@dataclass
class Punctures:
    """Two-puncture Bowen-York / Brill-Lindquist data (bare masses, positions,
    linear momenta, spins), as in NRPyElliptic_Ccodes/free_parameters.h:21-41."""
    m0: float = 0.5
    m1: float = 0.5
    pos0: tuple = (0.0, 0.0, 5.0)
    pos1: tuple = (0.0, 0.0, -5.0)
    P0: tuple = (0.0, 0.0, 0.0)
    P1: tuple = (0.0, 0.0, 0.0)
    S0: tuple = (0.0, 0.0, 0.0)
    S1: tuple = (0.0, 0.0, 0.0)


@dataclass
class Config:
    name: str
    Nxx: tuple
    punctures: Punctures = field(default_factory=Punctures)
    bScale: float = 5.0
    AMAX: float = 1.0e6
    SINHWAA: float = 0.07
    CFL: float = 0.5
    eta: float = 20.0
    R_L2: float = 100.0


# The relaxation configurations (puncture sets and grids) used by the tests
# and the benchmark.
SHIPPED_PUNCTURES = Punctures(
    m0=0.5184199353358704, m1=0.39193567996522616,
    pos0=(0.0, 0.0, 5.0), pos1=(0.0, 0.0, -5.0),
    P0=(0.09530152296974252, 0.0, -0.00084541526517121), P1=(-0.09530152296974252, 0.0, 0.00084541526517121),
    S0=(0.0, 0.09509112426035504, 0.0), S1=(0.0, -0.09156449704142013, 0.0))

CONFIGS = {
    # equal-mass head-on pair at rest: A_ij = 0, u = 0 solves it exactly
    "equal_mass_rest_64x64x8": Config("equal_mass_rest_64x64x8", (64, 64, 8)),
    # the reference's shipped puncture set (free_parameters.h), shipped CFL 0.7
    "shipped_64x64x8": Config("shipped_64x64x8", (64, 64, 8), SHIPPED_PUNCTURES, CFL=0.7),
    # quasi-circular equal-mass pair at production size
    "quasicircular_128x128x16": Config(
        "quasicircular_128x128x16", (128, 128, 16),
        Punctures(0.5, 0.5, (0, 0, 5.0), (0, 0, -5.0), (0, 0.095, 0), (0, -0.095, 0))),
    # unequal masses with spins at 256x256x32
    "unequal_spinning_256x256x32": Config(
        "unequal_spinning_256x256x32", (256, 256, 32),
        Punctures(0.8, 0.2, (0, 0, 1.2), (0, 0, -4.8), (0, 0.06, 0), (0, -0.06, 0), (0, 0, 0.1), (0.05, 0, -0.03)),
        bScale=6.0),
}


def sample_sweep(n=64, seed=20261203, grids=((96, 96, 12), (128, 128, 16), (192, 192, 24))):
    """Seeded puncture sweep: q log-uniform in [1,10] with total bare mass 1,
    separation d uniform in [4,20] with bScale = d/2 and the punctures at
    z = +-d/2, momentum magnitude uniform in [0,0.15] in the xy-plane with
    P1 = -P0, dimensionless spins |chi| uniform in [0,0.8] in uniform random
    directions (S = chi m^2), grid drawn uniformly from `grids`."""
    rng = np.random.default_rng(seed)
    out = []
    for i in range(n):
        q = float(np.exp(rng.uniform(0.0, np.log(10.0))))
        m0, m1 = q / (1 + q), 1 / (1 + q)
        d = float(rng.uniform(4.0, 20.0))
        pm = float(rng.uniform(0.0, 0.15))
        ang = float(rng.uniform(0.0, 2 * np.pi))
        P0 = (pm * np.cos(ang), pm * np.sin(ang), 0.0)
        spins = []
        for m in (m0, m1):
            chi = float(rng.uniform(0.0, 0.8))
            v = rng.normal(size=3)
            v /= np.linalg.norm(v)
            spins.append(tuple(float(x) for x in chi * m * m * v))
        grid = tuple(grids[int(rng.integers(len(grids)))])
        out.append(Config("sweep_%02d" % i, grid,
                          Punctures(m0, m1, (0, 0, d / 2), (0, 0, -d / 2), P0, tuple(-x for x in P0),
                                    spins[0], spins[1]),
                          bScale=d / 2))
    return out


def set_physical_params(p, cfg):
    """Copy the physical parameters of cfg into a paramstruct."""
    pu = cfg.punctures
    p.AMAX, p.SINHWAA, p.bScale, p.eta_damping = cfg.AMAX, cfg.SINHWAA, cfg.bScale, cfg.eta
    p.bare_mass_0, p.bare_mass_1 = pu.m0, pu.m1
    p.puncture_0_x, p.puncture_0_y, p.puncture_0_z = pu.pos0
    p.puncture_1_x, p.puncture_1_y, p.puncture_1_z = pu.pos1
    p.P0_x, p.P0_y, p.P0_z = pu.P0
    p.P1_x, p.P1_y, p.P1_z = pu.P1
    p.S0_x, p.S0_y, p.S0_z = pu.S0
    p.S1_x, p.S1_y, p.S1_z = pu.S1
    p.outer_bc_type = abi.RADIATION_OUTER_BCS
    p.time = 0.0


class Problem:
    """One configuration set up on the host: params, xx, bc_struct, rfm_struct,
    auxevol gridfunctions and dt.  Arrays are numpy views of C memory owned
    by this object (freed in close())."""

    def __init__(self, cfg, lib=None, host_aux=True, device_tables=False):
        self.cfg = cfg
        self.device_tables = device_tables
        self.lib = lib = lib or _lib.load()
        p = abi.paramstruct()
        lib.nrpyell_set_Cparameters_to_default(C.byref(p))
        set_physical_params(p, cfg)
        self.xx = _lib.XX()
        nxx = (C.c_int * 3)(*cfg.Nxx)
        lib.nrpyell_set_Nxx_dxx_invdx_params__and__xx(0, nxx, C.byref(p), self.xx)
        self.params = p
        self.bc = abi.bc_struct()
        self.rfm = abi.rfm_struct()
        self.dt = lib.nrpyell_find_timestep(C.byref(p), self.xx, cfg.CFL)
        if not device_tables:
            lib.nrpyell_bcstruct_set_up(C.byref(p), C.byref(self.bc))
            lib.nrpyell_rfm_precompute_rfmstruct_malloc(C.byref(p), C.byref(self.rfm))
            lib.nrpyell_rfm_precompute_rfmstruct_define(C.byref(p), self.xx, C.byref(self.rfm))
        # else: bc and rfm stay empty; DeviceState builds the device tables
        # on the GPU (nrpyell_setup_tables_device) keyed by these structs
        self.N = (p.Nxx_plus_2NGHOSTS0, p.Nxx_plus_2NGHOSTS1, p.Nxx_plus_2NGHOSTS2)
        self.Ntot = self.N[0] * self.N[1] * self.N[2]
        self._closed = False
        if not host_aux:
            # the auxevol gridfunctions are computed on the GPU by DeviceState
            # (nrpyell_auxevol_device), which also sets the wavespeed at the
            # outer boundary
            self.aux = None
            return
        self.aux = np.zeros(abi.NUM_AUXEVOL_GFS * self.Ntot)
        lib.nrpyell_auxevol_gfs_all_points(C.byref(p), self.xx, _ptr(self.aux))
        lib.nrpyell_wavespeed_gf_all_points(C.byref(p), cfg.CFL, self.dt, self.xx, _ptr(self.aux))
        self.set_wavespeed_at_OB(lib.nrpyell_compute_wavespeed_at_OB(C.byref(p), _ptr(self.aux)))

    def set_wavespeed_at_OB(self, c):
        self.params.uu_wavespeed_at_OB = c
        self.params.vv_wavespeed_at_OB = c

    def wavespeed_OB_index(self):
        """Index in the wavespeed gridfunction read by compute_wavespeed_at_OB.c:10."""
        N0, N1, N2 = self.N
        return (N0 - abi.NGHOSTS - 1) + N0 * (abi.NGHOSTS + N1 * (N2 // 2))

    # numpy views
    def xx_arrays(self):
        return [np.ctypeslib.as_array(self.xx[i], shape=(self.N[i],)).copy() for i in range(3)]

    def rfm_arrays(self):
        n0, n1 = self.N[0], self.N[1]
        out = {}
        for name in abi.RFM_FIELDS:
            n = n0 if "xx0" in name and "xx1" not in name else (n1 if "xx1" in name and "xx0" not in name else n0 * n1)
            out[name] = np.ctypeslib.as_array(getattr(self.rfm, name), shape=(n,)).copy()
        return out

    def radius(self):
        """r(xx0, xx1) of the SinhSymTP grid at the interior (i1, i0) points
        (the radius L2_norm_of_gf.c:19-28 compares with the integration
        radius), shape (Nxx1, Nxx0)."""
        p = self.params
        x0, x1 = self.xx_arrays()[:2]
        x0 = x0[abi.NGHOSTS:-abi.NGHOSTS]
        x1 = x1[abi.NGHOSTS:-abi.NGHOSTS]
        A = p.AMAX * np.sinh(x0 / p.SINHWAA) / np.sinh(1.0 / p.SINHWAA)
        s, c = np.sin(x1)[:, None], np.cos(x1)[:, None]
        return np.sqrt(A[None, :] ** 2 * s ** 2 + (p.bScale ** 2 + A[None, :] ** 2) * c ** 2)

    def zero_state(self):
        return np.zeros(abi.NUM_EVOL_GFS * self.Ntot)

    def griddata(self, gf_ptrs):
        """griddata_struct over this problem's tables and the given gridfunction
        pointers (dict of y_n, acc, k_odd, k_even, aux -> c_void_p / int)."""
        g = abi.griddata_struct()
        g.params = self.params
        for i in range(3):
            g.xx[i] = self.xx[i]
        g.bcstruct = self.bc
        g.rfmstruct = self.rfm
        f = g.gridfuncs
        cast = lambda v: C.cast(C.c_void_p(v) if isinstance(v, int) else v, abi.PREAL)
        f.y_n_gfs = cast(gf_ptrs["y_n"])
        f.y_nplus1_running_total_gfs = cast(gf_ptrs["acc"])
        f.k_odd_gfs = cast(gf_ptrs["k_odd"])
        f.k_even_gfs = cast(gf_ptrs["k_even"])
        f.auxevol_gfs = cast(gf_ptrs["aux"])
        f.diagnostic_output_gfs = f.y_nplus1_running_total_gfs
        return g

    def close(self):
        if self._closed:
            return
        self.lib.nrpyell_rfm_precompute_rfmstruct_freemem(C.byref(self.params), C.byref(self.rfm))
        self.lib.nrpyell_bcstruct_free(C.byref(self.bc))
        self.lib.nrpyell_free_xx(self.xx)
        self._closed = True

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class DeviceState:
    """Device buffers of one problem (y_n, running total, k_odd, k_even,
    auxevol) allocated through the library; the auxevol gridfunctions are
    uploaded once, or computed on the GPU when the problem has no host copy."""

    def __init__(self, prob, lib=None):
        self.lib = lib = lib or prob.lib
        self.prob = prob
        n2 = abi.NUM_EVOL_GFS * prob.Ntot * 8
        self.ptr = {k: lib.nrpyell_device_malloc(n2) for k in ("y_n", "acc", "k_odd", "k_even")}
        self.ptr["aux"] = lib.nrpyell_device_malloc(abi.NUM_AUXEVOL_GFS * prob.Ntot * 8)
        _lib.check(lib)
        if prob.aux is not None:
            self.upload("aux", prob.aux)
        else:
            lib.nrpyell_auxevol_device(C.byref(prob.params), prob.xx, prob.cfg.CFL, prob.dt, self.dptr("aux"))
            _lib.check(lib)
            ws = np.zeros(1)
            off = (abi.WAVESPEEDGF * prob.Ntot + prob.wavespeed_OB_index()) * 8
            lib.nrpyell_memcpy(ws.ctypes.data, self.ptr["aux"] + off, 8, 1)
            prob.set_wavespeed_at_OB(float(ws[0]))
        self.set_state(prob.zero_state())
        for k in ("acc", "k_odd", "k_even"):
            lib.nrpyell_memset(self.ptr[k], 0, n2)
        self.g = prob.griddata(self.ptr)
        if prob.device_tables:
            # the griddata struct holds copies of bc / rfm: key the tables by those
            lib.nrpyell_setup_tables_device(C.byref(prob.params), prob.xx, C.byref(self.g.rfmstruct),
                                            C.byref(self.g.bcstruct))
            _lib.check(lib)

    def upload(self, key, arr):
        arr = np.ascontiguousarray(arr, dtype=np.float64)
        self.lib.nrpyell_memcpy(self.ptr[key], arr.ctypes.data, arr.nbytes, 0)
        _lib.check(self.lib)

    def download(self, key, n=None):
        n = n if n is not None else (abi.NUM_AUXEVOL_GFS if key == "aux" else abi.NUM_EVOL_GFS) * self.prob.Ntot
        out = np.empty(n)
        self.lib.nrpyell_memcpy(out.ctypes.data, self.ptr[key], out.nbytes, 1)
        _lib.check(self.lib)
        return out

    def set_state(self, y):
        self.upload("y_n", y)

    def dptr(self, key):
        return C.cast(C.c_void_p(self.ptr[key]), abi.PREAL)

    def free(self):
        for k, v in list(self.ptr.items()):
            self.lib.nrpyell_device_free(v)
        self.ptr = {}


def _ptr(a):
    return a.ctypes.data_as(abi.PREAL)


def with_grid(cfg, Nxx):
    return replace(cfg, Nxx=tuple(Nxx), name="%s@%dx%dx%d" % (cfg.name, *Nxx))
