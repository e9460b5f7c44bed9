"""Host-side pieces of bench.py that need no GPU: the DRAM traffic it reports
beside the roofline comes from the ncu summaries under profiles/, keyed by
kernel and grid, and every tile kind maps to the kernel that runs it."""
import importlib.util
import os
import re

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _bench():
    spec = importlib.util.spec_from_file_location("bench_under_test", os.path.join(ROOT, "bench.py"))
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)  # module level defines only; main() runs under __main__
    return mod


def test_profiled_traffic_reads_each_kernel_and_grid():
    bench = _bench()
    found = {}
    for name in os.listdir(os.path.join(ROOT, "profiles")):
        for line in open(os.path.join(ROOT, "profiles", name)):
            m = re.match(r"dram_bytes_per_launch\[(\S+) (\S+)\]: (\d+)", line.strip())
            if m:
                found[(m.group(1), m.group(2))] = float(m.group(3))
    # the kernels bench.py reports: the bench grid and the out-of-L2 grid
    assert ("k_substep", "128x128x16") in found
    assert ("k_substep_march", "256x256x32") in found
    for (kernel, tag), value in found.items():
        assert bench.profiled_traffic(kernel, tag) == value
        assert value > 0
    assert bench.profiled_traffic("no_such_kernel", "128x128x16") is None
    assert bench.profiled_traffic("k_substep_march", "1x1x1") is None


def test_every_tile_kind_names_a_kernel():
    bench = _bench()
    # kinds of nrpyell_tile_info: 0 direct, 2 direct with prefetch, 4
    # shared-memory planes, 5 marching
    assert set(bench.KERNELS) == {0, 2, 4, 5}
    assert bench.KERNELS[5] == "k_substep_march" and bench.KERNELS[4] == "k_substep_planes"
