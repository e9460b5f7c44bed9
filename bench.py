#!/usr/bin/env python
"""Benchmark: FP64 hyperbolic relaxation of a binary-puncture Hamiltonian
constraint to log10 L2(residual) <= -10, in solves per second.

Default workload: the quasi-circular equal-mass pair on the 128x128x16
SinhSymTP grid (bare masses 0.5 at z = +-5, P = (0, +-0.095, 0), CFL 0.5,
eta 20), zero initial guess.  One "step" of this benchmark is one complete
solve from the zero guess to the tolerance (about 3070 RK4 steps with a
residual L2 norm before each).

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

ours:      solves on device-resident buffers through nrpyell_relax (value),
           and through nrpyell_relax_host with host buffers, the copies in the
           timed region (e2e).  Multi-GPU: one process per GPU, independent
           solves per rank (replicas; no data-path collective), barrier and
           max-over-ranks timing.
reference: the reference's own C (oracle/_ref, built from its sources with
           OpenMP) on the host cores: every step is one complete solve of the
           same workload from the zero guess (main.c's loop with the stop
           test); rank 0 only.
"""
import argparse
import ctypes as C
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

import numpy as np  # noqa: E402

METRIC = "solves/s to L2 residual <= 1e-10 (FP64 hyperbolic relaxation)"
TOL = -10.0
ALG_BYTES_STAGE2 = 104  # bytes per interior point of one stage-2/3 fused launch (13 doubles)
ALG_BYTES_STEP = 368  # bytes per interior point of one RK4 step (46 doubles)


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--config", default="quasicircular_128x128x16")
    ap.add_argument("--max-steps", type=int, default=40000)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--cpu-seconds", type=float, default=12.0)
    ap.add_argument("--learned-train", type=int, default=384,
                    help="training solves of the learned-guess leg (0: skip the leg)")
    ap.add_argument("--learned-test", type=int, default=24)
    return ap.parse_args()


class Clocks:
    """nvidia-smi samples during the timed region."""
    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index):
        self.idx = str(gpu_index)
        self.proc = None
        self.f = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)

    def start(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "--query-gpu=" + self.Q, "--format=csv,noheader,nounits",
                                          "-lms", "200"], stdout=self.f, stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None

    def stop(self):
        if not self.proc:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        self.f.flush()
        self.f.seek(0)
        rows = [r.split(",") for r in self.f.read().strip().splitlines() if r.strip()]
        rows = [[x.strip() for x in r] for r in rows if len(r) >= 9]
        mine = [r for r in rows if r[0] == self.idx] or rows
        if not mine:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["no samples"]}
        sm = [float(r[1]) for r in mine if r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in mine if r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({n for r in mine for n, v in zip(names, r[5:9]) if v.lower().startswith("active")})
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(mine)}


def measured_hbm_peak():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            return float(json.load(f)["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


# Fused substep kernel of each tile kind (nrpyell_tile_info).
KERNELS = {0: "k_substep", 2: "k_substep", 4: "k_substep_planes", 5: "k_substep_march"}


def profiled_traffic(kernel, tag):
    """DRAM bytes per launch of a fused substep kernel recorded from ncu in
    profiles/ (a line 'dram_bytes_per_launch[<kernel> <tag>]: <n>'), else None."""
    try:
        for name in os.listdir(os.path.join(ROOT, "profiles")):
            if not name.endswith((".md", ".txt")):
                continue
            for line in open(os.path.join(ROOT, "profiles", name)):
                key = "dram_bytes_per_launch[%s %s]:" % (kernel, tag)
                if key in line:
                    return float(line.split(key)[1].split()[0])
    except Exception:
        pass
    return None


def cpu_isa():
    try:
        flags = open("/proc/cpuinfo").read()
        return "v4" if " avx512f " in flags and " avx512vl " in flags else "v3"
    except Exception:
        return "v3"


def reference_steps(cfg_name):
    """Step count at which the reference's own relaxation of this workload
    reached the tolerance (recorded by running the reference build)."""
    path = os.path.join(ROOT, "tests", "golden", "relax_%s.npz" % cfg_name)
    if os.path.exists(path):
        return int(np.load(path)["steps"])
    return None


def cpu_time_per_iteration(cfg, seconds, threads=None):
    """Times main.c loop iterations (residual + L2 + RK4 step) of cfg on the
    host cores: the reference's own build when present, else the oracle port.
    Returns (seconds per iteration, kind, cores, iterations)."""
    from nrpyelliptic_b200 import abi
    from nrpyelliptic_b200.problem import set_physical_params
    from oracle import build as obuild
    ref = obuild.ref_lib_path(cpu_isa())
    P = C.POINTER
    if os.path.exists(ref):
        lib = C.CDLL(ref)
        lib.refh_setup.restype = C.c_double
        lib.refh_setup.argtypes = [P(abi.griddata_struct), P(C.c_int), P(abi.paramstruct), C.c_double]
        lib.refh_time_iterations.restype = C.c_double
        lib.refh_time_iterations.argtypes = [P(abi.griddata_struct), C.c_double, C.c_int, C.c_double]
        lib.refh_free.argtypes = [P(abi.griddata_struct)]
        lib.refh_max_threads.restype = C.c_int
        lib.set_Cparameters_to_default.argtypes = [P(abi.paramstruct)]
        if threads:
            lib.refh_set_threads(threads)
        phys = abi.paramstruct()
        lib.set_Cparameters_to_default(C.byref(phys))
        set_physical_params(phys, cfg)
        g = abi.griddata_struct()
        dt = lib.refh_setup(C.byref(g), (C.c_int * 3)(*cfg.Nxx), C.byref(phys), cfg.CFL)
        timer = lambda n: lib.refh_time_iterations(C.byref(g), dt, n, cfg.R_L2)
        kind, cores = "reference", lib.refh_max_threads()
        cleanup = lambda: lib.refh_free(C.byref(g))
    else:
        sys.path.insert(0, os.path.join(ROOT, "tests"))
        from _util import oracle, problem_grid

        from nrpyelliptic_b200.problem import Problem
        o = oracle()
        prob = Problem(cfg)
        hg = problem_grid(prob)
        g = hg.griddata()
        timer = lambda n: o.oracle_time_iterations(C.byref(g), prob.dt, n, cfg.R_L2)
        kind, cores = "port", os.cpu_count()
        cleanup = lambda: None
    timer(2)  # warm-up
    n_done, t_done, batch = 0, 0.0, 5
    while t_done < seconds and n_done < 5000:
        t_done += timer(batch)
        n_done += batch
        batch = min(batch * 2, 100)
    cleanup()
    return t_done / n_done, kind, cores, n_done


def cpu_solver(cfg):
    """One complete solve of cfg from the zero guess on the host cores per
    call: the reference's own build (main.c's loop with the stop test,
    refh_relax) when present, else the oracle port.  Returns (solve,
    cleanup, kind, cores); solve() returns (seconds, steps, converged)."""
    from nrpyelliptic_b200 import abi
    from nrpyelliptic_b200.problem import set_physical_params
    from oracle import build as obuild
    ref = obuild.ref_lib_path(cpu_isa())
    P = C.POINTER
    if os.path.exists(ref):
        lib = C.CDLL(ref)
        lib.refh_setup.restype = C.c_double
        lib.refh_setup.argtypes = [P(abi.griddata_struct), P(C.c_int), P(abi.paramstruct), C.c_double]
        lib.refh_relax.restype = C.c_int
        lib.refh_relax.argtypes = [P(abi.griddata_struct), C.c_double, C.c_double, C.c_int, C.c_double, abi.PREAL,
                                   P(C.c_int)]
        lib.refh_free.argtypes = [P(abi.griddata_struct)]
        lib.refh_max_threads.restype = C.c_int
        lib.set_Cparameters_to_default.argtypes = [P(abi.paramstruct)]
        phys = abi.paramstruct()
        lib.set_Cparameters_to_default(C.byref(phys))
        set_physical_params(phys, cfg)
        g = abi.griddata_struct()
        dt = lib.refh_setup(C.byref(g), (C.c_int * 3)(*cfg.Nxx), C.byref(phys), cfg.CFL)
        relax = lib.refh_relax
        kind, cores = "reference", lib.refh_max_threads()
        cleanup = lambda: lib.refh_free(C.byref(g))
    else:
        sys.path.insert(0, os.path.join(ROOT, "tests"))
        from _util import oracle, problem_grid

        from nrpyelliptic_b200.problem import Problem
        o = oracle()
        prob = Problem(cfg)
        hg = problem_grid(prob)
        g = hg.griddata()
        dt = prob.dt
        relax = o.oracle_relax
        kind, cores = "port", os.cpu_count()
        cleanup = lambda: None
    p = g.params
    n2 = 2 * p.Nxx_plus_2NGHOSTS0 * p.Nxx_plus_2NGHOSTS1 * p.Nxx_plus_2NGHOSTS2 * 8

    def solve(max_steps=40000):
        C.memset(g.gridfuncs.y_n_gfs, 0, n2)  # initial_guess_all_points: uu = vv = 0
        steps = C.c_int(0)
        t0 = time.perf_counter()
        rc = relax(C.byref(g), dt, TOL, max_steps, cfg.R_L2, None, C.byref(steps))
        return time.perf_counter() - t0, steps.value, rc == 0

    return solve, cleanup, kind, cores


def run_reference(args, dist):
    """The reference's own CPU implementation of the path: every bench step is
    one complete solve of the workload from the zero guess to the tolerance
    (main.c's loop: residual, L2, RK4 step, with the stop test)."""
    from nrpyelliptic_b200.problem import CONFIGS
    if dist.rank != 0:
        return
    cfg = CONFIGS[args.config]
    solve, cleanup, kind, cores = cpu_solver(cfg)
    times, steps_seen = [], set()
    for i in range(args.warmup + args.steps):
        t, n, ok = solve(args.max_steps)
        if not ok:
            raise RuntimeError("reference solve did not converge in %d steps" % args.max_steps)
        steps_seen.add(n)
        if i >= args.warmup:
            times.append(t)
    cleanup()
    t_solve = sum(times) / len(times)
    value = 1.0 / t_solve
    # per-iteration sample of the same loop, for comparison with the GPU arm's cpu_baseline
    t_it, _, _, n_it = cpu_time_per_iteration(cfg, max(2.0, args.cpu_seconds / 4))
    sample = ("%d complete solves of %s from the zero guess to log10 L2 <= %g (main.c loop: residual, L2, "
              "RK4 step), %s steps each" % (args.steps, args.config, TOL, "/".join(str(s) for s in sorted(steps_seen))))
    line = {"metric": METRIC, "value": value, "unit": "solves/s", "n_gpus": args.gpus, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": t_solve * 1e3, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded puncture parameters, zero guess)",
            "impl": "reference",
            "config": {"workload": args.config, "grid": list(cfg.Nxx), "tolerance_log10": TOL,
                       "steps_to_tolerance": max(steps_seen), "parallelism": "host OpenMP"},
            "cpu_baseline": {"value": value, "unit": "solves/s", "cores": cores, "kind": kind, "sample": sample},
            "e2e": {"value": value, "unit": "solves/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
            "per_iteration_sample": {"s_per_iteration": t_it, "iterations": n_it,
                                     "solves_per_s_extrapolated": 1.0 / (t_it * (max(steps_seen) + 1))}}
    print(json.dumps(line))


def split_errors(prob, uu, ref):
    """max and L2 of uu - ref relative to max|ref| / |ref|, at r < R_L2 and
    r >= R_L2 (uu, ref: interior arrays)."""
    inside = np.broadcast_to(prob.radius() < prob.cfg.R_L2, uu.shape)
    d = uu - ref
    sc = float(np.max(np.abs(ref)))
    out = {}
    for name, m in (("r_lt_RL2", inside), ("r_ge_RL2", ~inside)):
        out["max_" + name] = float(np.max(np.abs(d[m])) / sc) if m.any() else 0.0
        out["l2_" + name] = float(np.sqrt(np.sum(d[m] ** 2) / np.sum(ref[m] ** 2))) if m.any() else 0.0
    return out


def mixed_leg(lib, dist, prob, ds, args, ms_fp64=None, steps_fp64=None, fold=256):
    """The mixed-precision driver on one problem (prob/ds, or the 256x256x32
    configuration when None): one timed solve per variant after a short
    warm-up (tile tuning, graph capture), against one timed FP64 solve
    (ms_fp64 given: the bench's own)."""
    from nrpyelliptic_b200.problem import CONFIGS, DeviceState, Problem
    own = prob is None
    if own:
        prob = Problem(CONFIGS["unequal_spinning_256x256x32"], lib)
        ds = DeviceState(prob)
    n2 = 2 * prob.Ntot * 8
    cfg = prob.cfg
    st, fin = C.c_int(0), C.c_double(0)
    n32, n64 = C.c_int(0), C.c_int(0)

    def interior():
        N = prob.N
        return ds.download("y_n")[:prob.Ntot].reshape(N[2], N[1], N[0])[5:-5, 5:-5, 5:-5]

    def timed(fn):
        lib.nrpyell_memset(ds.ptr["y_n"], 0, n2)
        lib.nrpyell_flush_l2()
        dist.barrier()
        lib.nrpyell_event_record(6)
        rc = fn()
        lib.nrpyell_event_record(7)
        _lib_check(lib)
        if rc != 0:
            raise RuntimeError("mixed-precision leg: a solve did not converge")
        return dist.max(lib.nrpyell_event_elapsed_ms(6, 7))

    fp64 = lambda m: lib.nrpyell_relax(C.byref(ds.g), prob.dt, TOL, m, cfg.R_L2, C.byref(st), C.byref(fin), None)
    if ms_fp64 is None:
        lib.nrpyell_memset(ds.ptr["y_n"], 0, n2)
        fp64(64)
        ms_fp64 = timed(lambda: fp64(args.max_steps * 2))
        steps_fp64 = st.value
    else:
        timed(lambda: fp64(args.max_steps * 2))
    ref = interior()
    out = {"grid": "%dx%dx%d" % cfg.Nxx, "fold_every": fold, "fp64_solves_per_s": 1e3 / ms_fp64,
           "fp64_steps": steps_fp64, "variants": []}
    for switch in (TOL, -6.0):
        mx = lambda m: lib.nrpyell_relax_mixed(C.byref(ds.g), prob.dt, TOL, switch, fold, m, cfg.R_L2, C.byref(n32),
                                               C.byref(n64), C.byref(fin), None)
        lib.nrpyell_memset(ds.ptr["y_n"], 0, n2)
        mx(2 * fold)  # warm-up: tile tuning and graph capture
        ms = timed(lambda: mx(args.max_steps * 2))
        v = {"switch_log10_l2": switch, "solves_per_s": dist.world * 1e3 / ms, "speedup_vs_fp64": ms_fp64 / ms,
             "fp32_steps": n32.value, "fp64_steps": n64.value, "final_log10_l2": fin.value,
             "error_vs_fp64": split_errors(prob, interior(), ref)}
        out["variants"].append(v)
    if own:
        ds.free()
        prob.close()
    return out


def learned_leg(lib, args):
    """The learned initial guess on the 128x128x16 sweep distribution with a
    reduced training set (args.learned_train batched training solves, 64 POD
    modes, 300 epochs): the plain FP64 form against the learned guess alone,
    with the mixed-precision driver, with the batched driver and with both, on
    args.learned_test held-out draws (nrpyelliptic_b200.learned.compare_solvers)."""
    from nrpyelliptic_b200 import learned
    t0 = time.perf_counter()
    train = learned.configs(args.learned_train, 20261203)
    snaps, steps = learned.solve_snapshots(train, lib, log=lambda *a: None)
    t_solves = time.perf_counter() - t0
    mean, basis, coeffs, energy = learned.pod(snaps, 64)
    del snaps
    feats = np.array([learned.features(c) for c in train])
    guess = learned.Guess(lib, mean, basis, coeffs, feats)
    t1 = time.perf_counter()
    last, hist = guess.train(feats, coeffs, 300)
    t_train = time.perf_counter() - t1
    out = learned.compare_solvers(lib, guess, learned.configs(args.learned_test, 20261204))
    guess.free()
    out.update({"grid": "128x128x16", "training_solves": len(train), "training_solves_s": t_solves,
                "pod_modes": int(basis.shape[0]), "pod_energy": energy, "mlp_epochs": 300, "mlp_train_s": t_train,
                "mlp_loss_first_last": [float(hist[0]), float(last)]})
    return out


def _lib_check(lib):
    from nrpyelliptic_b200 import _lib
    _lib.check(lib)


def run_ours(args, dist):
    from nrpyelliptic_b200 import _lib, abi
    from nrpyelliptic_b200.problem import CONFIGS, DeviceState, Problem, with_grid
    lib = _lib.load()
    lib.nrpyell_set_device(dist.local_rank)
    cfg = CONFIGS[args.config]
    prob = Problem(cfg, lib)
    ds = DeviceState(prob)
    n2 = abi.NUM_EVOL_GFS * prob.Ntot * 8
    steps = C.c_int(0)
    fin = C.c_double(0.0)

    def solve():
        lib.nrpyell_memset(ds.ptr["y_n"], 0, n2)
        lib.nrpyell_flush_l2()
        rc = lib.nrpyell_relax(C.byref(ds.g), prob.dt, TOL, args.max_steps, cfg.R_L2, C.byref(steps), C.byref(fin),
                               None)
        _lib.check(lib)
        if rc != 0:
            raise RuntimeError("solve did not converge (rc=%d, steps=%d, log10 L2=%g)" % (rc, steps.value, fin.value))

    for _ in range(args.warmup):
        solve()
    steps_to_tol = steps.value

    clocks = Clocks(os.environ.get("CUDA_VISIBLE_DEVICES", str(dist.local_rank)).split(",")[0]
                    if dist.world == 1 else dist.local_rank)
    clocks.start()
    time.sleep(0.3)
    dist.barrier()
    lib.nrpyell_synchronize()
    launches0 = lib.nrpyell_launch_count()
    lib.nrpyell_event_record(0)
    for _ in range(args.steps):
        solve()
    lib.nrpyell_event_record(1)
    ms = lib.nrpyell_event_elapsed_ms(0, 1)
    launches = lib.nrpyell_launch_count() - launches0
    dist.barrier()
    clk = clocks.stop()
    ms_max = dist.max(ms)
    value = dist.world * args.steps / (ms_max * 1e-3)

    # Mixed precision (nrpyell_relax_mixed, the FP32 correction form): on the
    # bench workload and on the 256x256x32 mixed-precision configuration,
    # all steps in FP32 (switch = tolerance) and switching to FP64 at 1e-6;
    # solves/s, steps per phase, speed-up over the FP64 driver on the same
    # problem, and the solution's error against the FP64 solve.
    mixed = {args.config: mixed_leg(lib, dist, prob, ds, args, ms_max / args.steps, steps_to_tol)}
    mixed["unequal_spinning_256x256x32"] = mixed_leg(lib, dist, None, None, args)

    # End to end through the host-buffer entry point: H2D of the auxevol
    # gridfunctions and the initial guess, the solve, D2H of the solution.
    aux_h = lib.nrpyell_host_pinned_malloc(abi.NUM_AUXEVOL_GFS * prob.Ntot * 8)
    y_h = lib.nrpyell_host_pinned_malloc(n2)
    C.memmove(aux_h, prob.aux.ctypes.data, prob.aux.nbytes)
    as_real = lambda p: C.cast(C.c_void_p(p), abi.PREAL)

    def solve_host():
        C.memset(y_h, 0, n2)
        lib.nrpyell_flush_l2()
        rc = lib.nrpyell_relax_host(C.byref(prob.params), prob.xx, C.byref(prob.bc), C.byref(prob.rfm), as_real(aux_h),
                                    as_real(y_h), prob.dt, TOL, args.max_steps, cfg.R_L2, C.byref(steps), C.byref(fin))
        _lib.check(lib)
        if rc != 0:
            raise RuntimeError("host-buffer solve did not converge")

    solve_host()
    dist.barrier()
    lib.nrpyell_event_record(2)
    for _ in range(args.steps):
        solve_host()
    lib.nrpyell_event_record(3)
    ms_e2e = dist.max(lib.nrpyell_event_elapsed_ms(2, 3))
    e2e = dist.world * args.steps / (ms_e2e * 1e-3)
    lib.nrpyell_host_pinned_free(aux_h)
    lib.nrpyell_host_pinned_free(y_h)

    # Roofline of the dominant kernel: the fused RK4 substep (RHS + radiation
    # BC + RK combination), stage 2, timed over 200 graph-replayed launches.
    peak, peak_kind = measured_hbm_peak()
    n_int = cfg.Nxx[0] * cfg.Nxx[1] * cfg.Nxx[2]
    ms_k, ms_s = C.c_double(0), C.c_double(0)
    lib.nrpyell_time_fused(C.byref(ds.g), prob.dt, 2, 200, C.byref(ms_k), C.byref(ms_s))
    _lib.check(lib)
    bx, by, planes = C.c_int(0), C.c_int(0), C.c_int(0)

    def kernel_of(tile):
        kind = C.c_int(-1)
        lib.nrpyell_tile_info(tile, None, None, C.byref(kind))
        return KERNELS.get(kind.value, "k_substep")

    t_small = lib.nrpyell_get_tile(C.byref(prob.params), 0, C.byref(bx), C.byref(by), C.byref(planes))
    tile = [bx.value, by.value, planes.value]
    kern = kernel_of(t_small)
    achieved = ALG_BYTES_STAGE2 * n_int / (ms_k.value * 1e-3) / 1e9
    tag = "%dx%dx%d" % cfg.Nxx
    traffic = profiled_traffic(kern, tag)
    # The bench grid's 43.6 MB working set stays in the 126 MB L2, so HBM does
    # not bound its kernel: the L2 copy bandwidth, measured here with the
    # library's copy kernel on footprints below the L2 size, is the roofline
    # that does (best over footprints of 24-96 MB).
    l2_peaks = {mb: lib.nrpyell_copy_bandwidth(mb << 20, 10) for mb in (24, 48, 96)}
    _lib.check(lib)
    l2_peak = max(l2_peaks.values())
    roofline_l2 = {"bound": "l2", "achieved": 0.0, "peak": l2_peak, "unit": "GB/s", "frac": 0.0,
                   "peak_kind": "measured in this run (library copy kernel, best of footprints %s MB)"
                                % sorted(l2_peaks),
                   "peak_by_footprint_MB": {str(k): v for k, v in l2_peaks.items()},
                   "hbm_copy_GBps_2GB": lib.nrpyell_copy_bandwidth(2 << 30, 5)}
    roofline = {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                "traffic": traffic, "kernel": "%s<double,2>" % kern, "tile_index": t_small, "tile": tile, "peak_kind": peak_kind,
                "alg_bytes_per_launch": ALG_BYTES_STAGE2 * n_int, "us_per_launch": ms_k.value * 1e3,
                "rk4_step_us": ms_s.value * 1e3,
                "rk4_step_GBps": ALG_BYTES_STEP * n_int / (ms_s.value * 1e-3) / 1e9,
                "working_set_bytes": 11 * prob.Ntot * 8, "l2_resident": 11 * prob.Ntot * 8 < 126e6}
    roofline_l2["achieved"] = achieved
    roofline_l2["frac"] = achieved / l2_peak
    roofline_l2["rk4_step_frac"] = roofline["rk4_step_GBps"] / l2_peak
    # The same kernel on a working set larger than L2 (256x256x32, 262 MB).
    big = Problem(CONFIGS["unequal_spinning_256x256x32"], lib)
    dsb = DeviceState(big)
    lib.nrpyell_time_fused(C.byref(dsb.g), big.dt, 2, 50, C.byref(ms_k), C.byref(ms_s))
    _lib.check(lib)
    t_big = lib.nrpyell_get_tile(C.byref(big.params), 0, C.byref(bx), C.byref(by), C.byref(planes))
    kern_b = kernel_of(t_big)
    nb = 256 * 256 * 32
    ach_b = ALG_BYTES_STAGE2 * nb / (ms_k.value * 1e-3) / 1e9
    roofline_big = {"bound": "hbm", "achieved": ach_b, "peak": peak, "unit": "GB/s", "frac": ach_b / peak,
                    "traffic": profiled_traffic(kern_b, "256x256x32"), "kernel": "%s<double,2>" % kern_b,
                    "tile_index": t_big, "tile": [bx.value, by.value, planes.value],
                    "grid": "256x256x32", "us_per_launch": ms_k.value * 1e3, "rk4_step_us": ms_s.value * 1e3,
                    "rk4_step_GBps": ALG_BYTES_STEP * nb / (ms_s.value * 1e-3) / 1e9}
    dsb.free()
    big.close()

    line = {"metric": METRIC, "value": value, "unit": "solves/s", "n_gpus": dist.world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms_max / args.steps, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded puncture parameters, zero guess)",
            "config": {"workload": args.config, "grid": list(cfg.Nxx), "tolerance_log10": TOL,
                       "steps_to_tolerance": steps_to_tol, "rk4_steps_per_s": steps_to_tol * value,
                       "mpoints_rk4_steps_per_s": n_int * steps_to_tol * value / 1e6,
                       "parallelism": "replicas" if dist.world > 1 else "single",
                       "l2_flush": "256 MiB write before every solve (inside the timed region)"},
            "e2e": {"value": e2e, "unit": "solves/s", "h2d_bytes_per_step": (abi.NUM_AUXEVOL_GFS + 2) * prob.Ntot * 8,
                    "d2h_bytes_per_step": n2},
            "gpu_launches": int(launches), "clocks": clk, "roofline": roofline,
            "roofline_l2": roofline_l2, "roofline_out_of_l2": roofline_big, "mixed_precision": mixed}
    ds.free()
    if dist.world == 1 and args.learned_train > 0:
        line["learned_guess"] = learned_leg(lib, args)
    if dist.rank == 0 and dist.world == 1 and not args.no_cpu_baseline:
        t_it, kind, cores, n = cpu_time_per_iteration(cfg, args.cpu_seconds)
        line["cpu_baseline"] = {
            "value": 1.0 / (t_it * (steps_to_tol + 1)), "unit": "solves/s", "cores": cores, "kind": kind,
            "sample": "%d main.c-loop iterations (residual, L2, RK4 step) of %s timed, x %d iterations per solve"
                      % (n, args.config, steps_to_tol + 1)}
    if dist.rank == 0:
        print(json.dumps(line))


def main():
    from nrpyelliptic_b200.replicas import Replicas
    args = parse()
    dist = Replicas()
    try:
        if args.impl == "reference":
            run_reference(args, dist)
        else:
            run_ours(args, dist)
    finally:
        dist.close()


if __name__ == "__main__":
    main()
