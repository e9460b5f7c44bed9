"""Solution export: uu and the ADM quantities of the conformally flat data at
Cartesian points (nrpyell_interpolate_solution), and a binary dump of the
uu gridfunction.

    uu, psi, gamma, K = interpolate(prob, ds, xyz, order=4)
    alpha = initial_lapse(prob, xyz, uu, mode="psi^n", exponent=-2.0)
    dump_uu(prob, ds, "uu.npy")
"""
import ctypes as C

import numpy as np

from . import _lib, abi


def interpolate(prob, ds, xyz, order=4):
    """uu [n], psi [n], gamma_ij [n x 6], K_ij [n x 6] (xx xy xz yy yz zz) at
    the points xyz [n x 3] from the state in ds (a DeviceState whose y_n has
    filled ghost zones, as every relaxation driver leaves it)."""
    lib = prob.lib
    xyz = np.ascontiguousarray(xyz, dtype=np.float64).reshape(-1, 3)
    n = len(xyz)
    uu, psi = np.zeros(n), np.zeros(n)
    gamma, K = np.zeros((n, 6)), np.zeros((n, 6))
    P = lambda a: a.ctypes.data_as(abi.PREAL)
    lib.nrpyell_interpolate_solution(C.byref(prob.params), prob.xx, ds.dptr("y_n"), n, P(xyz), order, P(uu), P(psi),
                                     P(gamma), P(K))
    _lib.check(lib)
    return uu, psi, gamma, K


LAPSE_MODES = {"psi^n": 0, "averaged": 1}


def initial_lapse(prob, xyz, uu=None, mode="psi^n", exponent=-2.0):
    """The thorn's initial lapse at the points xyz [n x 3]: "psi^n" (alpha =
    (psi_BL + uu)^exponent, uu at the points from interpolate()) or
    "averaged" (from the Brill-Lindquist term alone)."""
    lib = prob.lib
    xyz = np.ascontiguousarray(xyz, dtype=np.float64).reshape(-1, 3)
    n = len(xyz)
    alpha = np.zeros(n)
    P = lambda a: a.ctypes.data_as(abi.PREAL)
    u = np.ascontiguousarray(uu, dtype=np.float64) if uu is not None else None
    lib.nrpyell_initial_lapse(C.byref(prob.params), n, P(xyz), P(u) if u is not None else None, LAPSE_MODES[mode],
                              float(exponent), P(alpha))
    _lib.check(lib)
    return alpha


def dump_uu(prob, ds, path):
    """uu with its ghost zones, shape (N2, N1, N0) float64, to a .npy file."""
    uu = ds.download("y_n", prob.Ntot).reshape(prob.N[2], prob.N[1], prob.N[0])
    np.save(path, uu)
    return uu
