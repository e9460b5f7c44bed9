"""Device time of every tile shape of the fused RK4 substep kernel on a
configuration's grid -- the table the autotuner chooses from.

    python -m nrpyelliptic_b200.tiles [CONFIG ...] [--launches N] [--tile T]

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
KINDS = {0: "direct", 2: "direct+prefetch", 3: "tma pipeline", 4: "smem planes", 5: "smem march"}


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


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("configs", nargs="*", default=["quasicircular_128x128x16", "unequal_spinning_256x256x32"])
    ap.add_argument("--launches", type=int, default=50)
    ap.add_argument("--tile", type=int, default=None, help="time this tile shape only")
    args = ap.parse_args()
    for name in args.configs:
        print("| %s | tile | 32 x by x planes | kind | stage 1 us | stage 2 us | stage 2 GB/s | stage 4 us | RK4 step us |"
              % name)
        print("|---|---|---|---|---|---|---|---|---|")
        for t, by, p, st, u1, u2, gbs, u4, step in sweep(name, args.launches, only=args.tile):
            print("| | %d | 32 x %d x %d | %s | %.2f | %.2f | %.0f | %.2f | %.2f |"
                  % (t, by, p, KINDS.get(st, str(st)), u1, u2, gbs, u4, step), flush=True)


if __name__ == "__main__":
    main()
