"""Command-line relaxation run, the GPU counterpart of the reference's
NRPyElliptic_Playground executable (NRPyElliptic_Ccodes/main.c):

    python -m nrpyelliptic_b200.playground Nx0 Nx1 Nx2 N_final [--config NAME] [--tol T] [--outdir DIR]

Sets up the configuration (default: the reference's shipped puncture set,
free_parameters.h, CFL 0.7), relaxes from the zero guess for at most N_final
RK4 steps on the GPU -- stopping early once log10 L2 <= --tol when given --
and writes, in the reference's formats,
  DIR/output_NRPyElliptic/residual_l2_norm.txt   "%6d %10.4e %.17e" per step (main.c:154)
  DIR/output_NRPyElliptic/uu_final_1D.txt        uu along the z axis (gridfunction_z_axis.c)
"""
import argparse
import ctypes as C
import math
import os
import sys

import numpy as np

from . import _lib, abi
from .problem import CONFIGS, DeviceState, Problem, with_grid


def z_axis_dump(prob, uu):
    """(z, uu) pairs in the order of gridfunction_z_axis.c:10-51."""
    p = prob.params
    N0, N1, N2 = prob.N
    xx = prob.xx_arrays()
    u = uu.reshape(N2, N1, N0)
    i2 = N2 // 2
    iw = 1.0 / p.SINHWAA

    def z(x0, x1):
        e = math.exp(iw * x0) - math.exp(-iw * x0)
        d = math.exp(iw) - math.exp(-iw)
        return math.sqrt(p.AMAX * p.AMAX * (e * e) / (d * d) + p.bScale * p.bScale) * math.cos(x1)

    rows = []
    ng = abi.NGHOSTS
    for i1 in (ng, N1 - ng - 1):
        for i0 in range(ng, N0 - ng):
            rows.append((z(xx[0][i0], xx[1][i1]), u[i2, i1, i0]))
    for i1 in range(ng + 1, N1 - ng - 1):
        rows.append((z(xx[0][ng], xx[1][i1]), u[i2, i1, ng]))
    return rows


def main(argv=None):
    ap = argparse.ArgumentParser(description=__doc__, formatter_class=argparse.RawDescriptionHelpFormatter)
    ap.add_argument("Nxx", type=int, nargs=3)
    ap.add_argument("N_final", type=int)
    ap.add_argument("--config", default="shipped_64x64x8", choices=sorted(CONFIGS))
    ap.add_argument("--tol", type=float, default=None, help="stop once log10 L2 <= tol")
    ap.add_argument("--outdir", default=".")
    ap.add_argument("--no-output", action="store_true")
    a = ap.parse_args(argv)
    if min(a.Nxx) < abi.NGHOSTS or any(n % 2 for n in a.Nxx):
        sys.exit("Nx0 Nx1 Nx2 must be even and at least NGHOSTS (= %d)" % abi.NGHOSTS)
    lib = _lib.load()
    cfg = with_grid(CONFIGS[a.config], a.Nxx)
    prob = Problem(cfg, lib)
    ds = DeviceState(prob)
    hist = np.zeros(a.N_final + 1)
    steps = C.c_int(0)
    fin = C.c_double(0.0)
    tol = a.tol if a.tol is not None else -1e300
    rc = lib.nrpyell_relax(C.byref(ds.g), prob.dt, tol, a.N_final, cfg.R_L2, C.byref(steps), C.byref(fin),
                           hist.ctypes.data_as(abi.PREAL))
    _lib.check(lib)
    n = steps.value
    print("steps %d  log10 L2 %.6f  %s" % (n, fin.value, "converged" if rc == 0 else "not converged"))
    if not a.no_output:
        out = os.path.join(a.outdir, "output_NRPyElliptic")
        os.makedirs(out, exist_ok=True)
        with open(os.path.join(out, "residual_l2_norm.txt"), "w") as f:
            for k in range(n + 1):
                f.write("%6d %10.4e %.17e\n" % (k, k * prob.dt, hist[k]))
        uu = ds.download("y_n")[:prob.Ntot]
        with open(os.path.join(out, "uu_final_1D.txt"), "w") as f:
            for z, v in z_axis_dump(prob, uu):
                f.write("%.17e %.17e\n" % (z, v))
    ds.free()
    prob.close()
    return 0 if rc in (0, 1) else 1


if __name__ == "__main__":
    sys.exit(main())
