"""Command-line relaxation run, the GPU counterpart of the reference's
NRPyElliptic_Playground executable (NRPyElliptic_Ccodes/main.c):

    python -m nrpyelliptic_b200.playground Nx0 Nx1 Nx2 N_final [--config NAME] [--tol T] [--outdir DIR]
                                           [--snapshots] [--no-output]

Sets up the configuration (default: the reference's shipped puncture set,
free_parameters.h, CFL 0.7), relaxes from the zero guess on the GPU -- like
main.c's loop, N_final + 1 residuals and steps, or until log10 L2 <= --tol
when given -- and writes main.c's files in its formats:
  DIR/output_NRPyElliptic/{wavespeed,ADD_times_AUU,psi_background}_gf_1D.txt
                                                 auxevol along the z axis (main.c:120-131)
  DIR/output_NRPyElliptic/residual_l2_norm.txt   "%6d %10.4e %.17e" per step (main.c:154)
  DIR/output_NRPyElliptic/uu_final_1D.txt        uu along the z axis (gridfunction_z_axis.c)
and with --snapshots, every N_final/100 steps (main.c:157-179),
  DIR/output_NRPyElliptic/1D/uu_1D_%08d.dat      uu along the z axis
  DIR/output_NRPyElliptic/2D/uu_2D_%08d.dat      uu on the xz plane (gridfunction_xz_plane.c)
  DIR/output_NRPyElliptic/2D/residual_2D_%08d.dat  the residual on the xz plane
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


def xz_plane_dump(prob, gf):
    """(x, z, value) triples in the order of gridfunction_xz_plane.c:6-52:
    the interior of the i2 = NGHOSTS plane (x < 0), then of i2 = N2/2 (x > 0)."""
    p = prob.params
    N0, N1, N2 = prob.N
    xx = prob.xx_arrays()
    g = gf.reshape(N2, N1, N0)
    iw = 1.0 / p.SINHWAA
    d = math.exp(iw) - math.exp(-iw)
    rows = []
    ng = abi.NGHOSTS
    for i2 in (ng, N2 // 2):
        for i1 in range(ng, N1 - ng):
            for i0 in range(ng, N0 - ng):
                e = math.exp(iw * xx[0][i0]) - math.exp(-iw * xx[0][i0])
                x = p.AMAX * e * math.sin(xx[1][i1]) * math.cos(xx[2][i2]) / d
                z = math.sqrt(p.AMAX * p.AMAX * (e * e) / (d * d) + p.bScale * p.bScale) * math.cos(xx[1][i1])
                rows.append((x, z, g[i2, i1, i0]))
    return rows


def write_rows(path, rows, fmt):
    with open(path, "w") as f:
        for r in rows:
            f.write(fmt % r)


def main(argv=None):
    ap = argparse.ArgumentParser(description=__doc__, formatter_class=argparse.RawDescriptionHelpFormatter)
    ap.add_argument("Nxx", type=int, nargs=3)
    ap.add_argument("N_final", type=int)
    ap.add_argument("--config", default="shipped_64x64x8", choices=sorted(CONFIGS))
    ap.add_argument("--tol", type=float, default=None, help="stop once log10 L2 <= tol")
    ap.add_argument("--outdir", default=".")
    ap.add_argument("--no-output", action="store_true")
    ap.add_argument("--snapshots", action="store_true",
                    help="also write main.c's 1D/2D snapshots every N_final/100 steps (slower: the relaxation "
                         "runs in chunks between them)")
    a = ap.parse_args(argv)
    if min(a.Nxx) < abi.NGHOSTS or any(n % 2 for n in a.Nxx):
        sys.exit("Nx0 Nx1 Nx2 must be even and at least NGHOSTS (= %d)" % abi.NGHOSTS)
    lib = _lib.load()
    cfg = with_grid(CONFIGS[a.config], a.Nxx)
    prob = Problem(cfg, lib)
    ds = DeviceState(prob)
    out = os.path.join(a.outdir, "output_NRPyElliptic")
    if not a.no_output:
        os.makedirs(os.path.join(out, "1D"), exist_ok=True)
        os.makedirs(os.path.join(out, "2D"), exist_ok=True)
        Nt = prob.Ntot
        for name, g in (("wavespeed_gf_1D.txt", abi.WAVESPEEDGF), ("ADD_times_AUU_gf_1D.txt", abi.ADD_TIMES_AUUGF),
                        ("psi_background_gf_1D.txt", abi.PSI_BACKGROUNDGF)):
            write_rows(os.path.join(out, name), z_axis_dump(prob, prob.aux[g * Nt:(g + 1) * Nt]), "%.17e %.17e\n")
    tol = a.tol if a.tol is not None else -1e300
    # main.c:65-68: snapshots every N_final/100 steps
    every = max(1, int(a.N_final / 100.0)) if (a.snapshots and not a.no_output) else a.N_final
    every = max(every, 1)
    hist = []
    n, rc, fin = 0, 1, C.c_double(0.0)
    while True:
        # main.c:145-179: the residual and the snapshots of step n, then the step
        if a.snapshots and not a.no_output and n % every == 0:
            write_rows(os.path.join(out, "1D", "uu_1D_%08d.dat" % n), z_axis_dump(prob, ds.download("y_n")[:prob.Ntot]),
                       "%.17e %.17e\n")
            write_rows(os.path.join(out, "2D", "uu_2D_%08d.dat" % n), xz_plane_dump(prob, ds.download("y_n")[:prob.Ntot]),
                       "%.17e %.17e %.17e\n")
            lib.residual_all_points(C.byref(prob.params), C.byref(prob.rfm), ds.dptr("aux"), ds.dptr("y_n"),
                                    ds.dptr("acc"))
            _lib.check(lib)
            write_rows(os.path.join(out, "2D", "residual_2D_%08d.dat" % n),
                       xz_plane_dump(prob, ds.download("acc")[:prob.Ntot]), "%.17e %.17e %.17e\n")
        if hist and (rc == 0 or n >= a.N_final):
            break
        chunk = min(every, a.N_final - n)
        h = np.zeros(chunk + 1)
        steps = C.c_int(0)
        rc = lib.nrpyell_relax(C.byref(ds.g), prob.dt, tol, chunk, cfg.R_L2, C.byref(steps), C.byref(fin),
                               h.ctypes.data_as(abi.PREAL))
        _lib.check(lib)
        hist.extend(h[(1 if hist else 0):steps.value + 1])
        n += steps.value
        if steps.value < chunk and rc != 0:
            break
    if a.tol is None:
        # main.c's loop also steps after its last residual (n = N_final)
        lib.MoL_step_forward_in_time(C.byref(ds.g), prob.dt)
        _lib.check(lib)
    print("steps %d  log10 L2 %.6f  %s" % (n, fin.value, "converged" if rc == 0 else "not converged"))
    if not a.no_output:
        write_rows(os.path.join(out, "residual_l2_norm.txt"), [(k, k * prob.dt, v) for k, v in enumerate(hist)],
                   "%6d %10.4e %.17e\n")
        write_rows(os.path.join(out, "uu_final_1D.txt"), z_axis_dump(prob, ds.download("y_n")[:prob.Ntot]),
                   "%.17e %.17e\n")
    ds.free()
    prob.close()
    return 0 if rc in (0, 1) else 1


if __name__ == "__main__":
    sys.exit(main())
