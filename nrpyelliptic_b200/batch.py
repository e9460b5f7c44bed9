"""Batched relaxation of many puncture configurations (nrpyell_relax_batch)
and the seeded sweep command line:

    python -m nrpyelliptic_b200.batch [--n 64] [--seed 20261203] [--tol -10] [--max-steps N]

Every RK4 substep of all configurations -- on grids of different sizes -- is
one kernel launch; sixteen RK4 steps are one CUDA graph, replayed until every
configuration has reached the tolerance (each stops on its own).
"""
import argparse
import ctypes as C
import time

import numpy as np

from . import _lib, abi
from .problem import DeviceState, Problem, sample_sweep


def relax_batch(problems, states=None, tol=-10.0, max_steps=100000, lib=None):
    """Relax `problems` together from the zero guess (or from `states`, a
    list of DeviceState).  Returns (n_not_converged, steps, final_log10_l2,
    states)."""
    lib = lib or _lib.load()
    n = len(problems)
    states = states or [DeviceState(p, lib=lib) for p in problems]
    grids = (abi.griddata_struct * n)(*[s.g for s in states])
    dts = np.array([p.dt for p in problems], dtype=np.float64)
    steps = (C.c_int * n)()
    finals = np.zeros(n)
    rc = lib.nrpyell_relax_batch(n, grids, dts.ctypes.data_as(abi.PREAL), tol, max_steps,
                                 float(problems[0].cfg.R_L2), steps, finals.ctypes.data_as(abi.PREAL))
    _lib.check(lib)
    return rc, np.array(steps[:], dtype=np.int64), finals, states


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--n", type=int, default=64)
    ap.add_argument("--seed", type=int, default=20261203)
    ap.add_argument("--tol", type=float, default=-10.0)
    ap.add_argument("--max-steps", type=int, default=100000)
    args = ap.parse_args()
    lib = _lib.load()
    lib.nrpyell_synchronize()  # CUDA context and library stream, outside the set-up timing
    t0 = time.perf_counter()
    cfgs = sample_sweep(args.n, args.seed)
    problems = [Problem(c, lib=lib, host_aux=False, device_tables=True) for c in cfgs]
    states = [DeviceState(p, lib=lib) for p in problems]
    lib.nrpyell_synchronize()
    t1 = time.perf_counter()
    rc, steps, finals, _ = relax_batch(problems, states, args.tol, args.max_steps, lib=lib)
    t2 = time.perf_counter()
    print("| config | grid | q | steps | final log10 L2 |")
    print("|---|---|---|---|---|")
    for c, s, f in zip(cfgs, steps, finals):
        q = c.punctures.m0 / c.punctures.m1
        print("| %s | %dx%dx%d | %.2f | %d | %.2f |" % (c.name, *c.Nxx, q, s, f))
    pts = sum(int(np.prod(c.Nxx)) * int(s) for c, s in zip(cfgs, steps))
    print("\n%d configurations, %d not converged; set-up (host grids, tables and auxevol on the GPU) %.2f s; batched relaxation %.2f s = %.2f solves/s; "
          "%.0f Mpoint-RK4-steps/s" % (len(cfgs), rc, t1 - t0, t2 - t1, len(cfgs) / (t2 - t1), pts / (t2 - t1) / 1e6))
    for s in states:
        s.free()


if __name__ == "__main__":
    main()
