"""Device time of every tile shape of the fused RK4 substep kernel on a
configuration's grid -- the table the autotuner chooses from.

    python -m nrpyelliptic_b200.tiles [CONFIG ...] [--launches N] [--tile T]
    python -m nrpyelliptic_b200.tiles [CONFIG ...] --mixed STEPS

--mixed runs STEPS RK4 steps of the mixed-precision driver's FP32 correction
form from the zero guess instead (after a warm-up of the same length) and
prints the time per step: the launch to capture when profiling the FP32
correction kernels.

For each shape: the stage-1, stage-2 and stage-4 kernels (CUDA-event time
averaged over N launches replayed from a CUDA graph) and one whole RK4 step,
with the stage-2 algorithmic bandwidth (104 bytes per interior point: read
uu, vv of the stage input, three auxevol fields, y_n and the running total;
write the running total and the stage output).
"""
import argparse
import ctypes as C

from . import _lib
from .problem import CONFIGS, DeviceState, Problem

STAGE2_BYTES = 104
KINDS = {0: "direct", 2: "direct+prefetch", 4: "smem planes", 5: "smem march"}


def shapes(lib):
    out = []
    for t in range(lib.nrpyell_num_tiles()):
        by, p, st = C.c_int(), C.c_int(), C.c_int()
        lib.nrpyell_tile_info(t, C.byref(by), C.byref(p), C.byref(st))
        out.append((t, by.value, p.value, st.value))
    return out


def sweep(name, launches=50, lib=None, only=None):
    """Rows (tile, by, planes, kind, us stage 1, us stage 2, GB/s stage 2, us stage 4, us per RK4 step);
    `only`: a single tile index."""
    lib = lib or _lib.load()
    prob = Problem(CONFIGS[name], lib=lib)
    ds = DeviceState(prob)
    npts = prob.cfg.Nxx[0] * prob.cfg.Nxx[1] * prob.cfg.Nxx[2]
    rows = []
    try:
        for t, by, p, st in shapes(lib):
            if only is not None and t != only:
                continue
            lib.nrpyell_set_tile(t)
            us = []
            step = C.c_double()
            for stage in (1, 2, 4):
                mk = C.c_double()
                lib.nrpyell_time_fused(C.byref(ds.g), prob.dt, stage, launches, C.byref(mk), C.byref(step))
                us.append(mk.value * 1e3)
            _lib.check(lib)
            rows.append((t, by, p, st, us[0], us[1], STAGE2_BYTES * npts / (us[1] * 1e-6) / 1e9, us[2],
                         step.value * 1e3))
    finally:
        lib.nrpyell_set_tile(-1)
        ds.free()
    return rows


def mixed_steps(name, steps, lib=None, tile=None):
    """Microseconds per RK4 step of the FP32 correction form (nrpyell_relax_mixed
    with every step in FP32, folds every 256 steps) over `steps` steps."""
    import time
    lib = lib or _lib.load()
    prob = Problem(CONFIGS[name], lib=lib)
    ds = DeviceState(prob)
    n32, n64, fin = C.c_int(), C.c_int(), C.c_double()
    if tile is not None:
        lib.nrpyell_set_tile(tile)
    out = []
    for _ in range(2):  # warm-up (autotuning, graph capture), then timed
        lib.nrpyell_memset(ds.ptr["y_n"], 0, 2 * prob.Ntot * 8)
        lib.nrpyell_synchronize()
        t0 = time.perf_counter()
        lib.nrpyell_relax_mixed(C.byref(ds.g), prob.dt, -30.0, -30.0, 256, steps, prob.cfg.R_L2, C.byref(n32),
                                C.byref(n64), C.byref(fin), None)
        lib.nrpyell_synchronize()
        out.append((time.perf_counter() - t0) * 1e6 / max(1, n32.value))
        _lib.check(lib)
    tile = lib.nrpyell_get_tile(C.byref(prob.params), 2, None, None, None)
    lib.nrpyell_set_tile(-1)
    ds.free()
    return out[-1], n32.value, tile


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("configs", nargs="*", default=["quasicircular_128x128x16", "unequal_spinning_256x256x32"])
    ap.add_argument("--launches", type=int, default=50)
    ap.add_argument("--tile", type=int, default=None, help="time this tile shape only")
    ap.add_argument("--mixed", type=int, default=0, help="time STEPS steps of the FP32 correction form instead")
    args = ap.parse_args()
    if args.mixed:
        for name in args.configs:
            us, n, tile = mixed_steps(name, args.mixed, tile=args.tile)
            print("%s: FP32 correction form, %d steps, %.2f us per RK4 step (wall clock, folds included), tile %d"
                  % (name, n, us, tile))
        return
    for name in args.configs:
        print("| %s | tile | 32 x by x planes | kind | stage 1 us | stage 2 us | stage 2 GB/s | stage 4 us | RK4 step us |"
              % name)
        print("|---|---|---|---|---|---|---|---|---|")
        for t, by, p, st, u1, u2, gbs, u4, step in sweep(name, args.launches, only=args.tile):
            print("| | %d | 32 x %d x %d | %s | %.2f | %.2f | %.0f | %.2f | %.2f |"
                  % (t, by, p, KINDS.get(st, str(st)), u1, u2, gbs, u4, step), flush=True)


if __name__ == "__main__":
    main()
