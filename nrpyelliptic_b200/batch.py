"""Batched relaxation of many puncture configurations (nrpyell_relax_batch)
and the seeded sweep command line, on one GPU or sharded by configuration
over several (one process per GPU, torchrun):

    python -m nrpyelliptic_b200.batch [--n 64] [--seed 20261203] [--tol -10] [--max-steps N] [--mixed]
    python -m torch.distributed.run --nproc-per-node 8 --master-addr 127.0.0.1 -m nrpyelliptic_b200.batch

Every RK4 substep of all configurations -- on grids of different sizes -- is
one kernel launch; sixteen RK4 steps are one CUDA graph, replayed until every
configuration has reached the tolerance (each stops on its own).  With
--mixed the sweep runs the FP32 correction form (nrpyell_relax_batch_mixed,
every step FP32, folded into the FP64 state every 256 steps, the FP64 norm as
the stop test).
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


def relax_batch_mixed(problems, states=None, tol=-10.0, switch=-10.0, fold_every=256, max_steps=100000, lib=None):
    """The FP32 correction form (nrpyell_relax_batch_mixed) on `problems`
    together, from the zero guess or from `states`.  Returns
    (n_not_converged, steps_fp32, steps_fp64, final_log10_l2, states)."""
    lib = lib or _lib.load()
    n = len(problems)
    states = states or [DeviceState(p, lib=lib) for p in problems]
    grids = (abi.griddata_struct * n)(*[s.g for s in states])
    dts = np.array([p.dt for p in problems], dtype=np.float64)
    s32, s64 = (C.c_int * n)(), (C.c_int * n)()
    finals = np.zeros(n)
    rc = lib.nrpyell_relax_batch_mixed(n, grids, dts.ctypes.data_as(abi.PREAL), tol, switch, fold_every, max_steps,
                                       float(problems[0].cfg.R_L2), s32, s64, finals.ctypes.data_as(abi.PREAL))
    _lib.check(lib)
    return (rc, np.array(s32[:], dtype=np.int64), np.array(s64[:], dtype=np.int64), finals, states)


def solve_batch(cfgs, lib=None, tol=-10.0, max_steps=100000, device_tables=True, mixed=False):
    """Set up cfgs (tables and auxevol on the GPU) and relax them together in
    one batch (mixed: the FP32 correction form, every step FP32, fold every
    256 steps); per configuration a dict with its RK4 steps, final log10 L2
    and a SHA-256 of its converged y_n (ghost zones included)."""
    import hashlib
    lib = lib or _lib.load()
    problems = [Problem(c, lib=lib, host_aux=False, device_tables=device_tables) for c in cfgs]
    states = [DeviceState(p, lib=lib) for p in problems]
    if mixed:
        rc, s32, s64, finals, _ = relax_batch_mixed(problems, states, tol, tol, 256, max_steps, lib=lib)
        steps = s32 + s64
    else:
        rc, steps, finals, _ = relax_batch(problems, states, tol, max_steps, lib=lib)
    out = []
    for c, p, ds, st, f in zip(cfgs, problems, states, steps, finals):
        y = ds.download("y_n")
        out.append({"name": c.name, "steps": int(st), "final_log10_l2": float(f),
                    "y_sha256": hashlib.sha256(y.tobytes()).hexdigest(), "points": int(np.prod(c.Nxx))})
        ds.free()
    for p in problems:
        p.close()
    lib.nrpyell_release_tables()
    return out


def sweep(cfgs, dist=None, solve=solve_batch, **kw):
    """A sweep sharded by configuration over the ranks of `dist` (a
    replicas.Replicas, one process per GPU): configuration i goes to rank
    i % world, each rank relaxes its share as one batch, and the results are
    gathered on the host (no collective touches the solves).  Returns, on
    every rank, (per-configuration results in cfgs order, seconds of the
    slowest rank)."""
    from .replicas import shard
    rank, world = (dist.rank, dist.world) if dist else (0, 1)
    mine = shard(list(range(len(cfgs))), rank, world)
    if dist:
        dist.barrier()
    t0 = time.perf_counter()
    res = solve([cfgs[i] for i in mine], **kw) if mine else []
    sec = time.perf_counter() - t0
    parts = dist.all_gather((mine, res, sec)) if dist else [(mine, res, sec)]
    out = [None] * len(cfgs)
    for idx, r, _ in parts:
        for i, x in zip(idx, r):
            out[i] = x
    return out, max(p[2] for p in parts)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--n", type=int, default=64)
    ap.add_argument("--seed", type=int, default=20261203)
    ap.add_argument("--tol", type=float, default=-10.0)
    ap.add_argument("--max-steps", type=int, default=100000)
    ap.add_argument("--mixed", action="store_true", help="FP32 correction form (nrpyell_relax_batch_mixed)")
    args = ap.parse_args()
    from .replicas import Replicas
    dist = Replicas()
    try:
        lib = _lib.load()
        lib.nrpyell_set_device(dist.local_rank)
        lib.nrpyell_synchronize()  # CUDA context and library stream, outside the timing
        cfgs = sample_sweep(args.n, args.seed)
        res, sec = sweep(cfgs, dist, lib=lib, tol=args.tol, max_steps=args.max_steps, mixed=args.mixed)
        if dist.rank == 0:
            print("| config | grid | q | steps | final log10 L2 |")
            print("|---|---|---|---|---|")
            for c, r in zip(cfgs, res):
                q = c.punctures.m0 / c.punctures.m1
                print("| %s | %dx%dx%d | %.2f | %d | %.2f |" % (c.name, *c.Nxx, q, r["steps"], r["final_log10_l2"]))
            pts = sum(r["points"] * r["steps"] for r in res)
            bad = sum(r["final_log10_l2"] > args.tol for r in res)
            print("\n%d configurations on %d GPU(s)%s, %d not converged; set-up (grids on the host, tables and "
                  "auxevol on the GPU) and batched relaxation %.2f s (slowest rank) = %.2f solves/s; "
                  "%.0f Mpoint-RK4-steps/s" % (len(cfgs), dist.world, ", FP32 correction form" if args.mixed else "",
                                               bad, sec, len(cfgs) / sec, pts / sec / 1e6))
    finally:
        dist.close()


if __name__ == "__main__":
    main()
