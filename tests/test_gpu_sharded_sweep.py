"""A sweep sharded over two ranks (batch.sweep over a gloo Replicas) with
the real GPU solver: both ranks run on cuda:0 here (one GPU per call), each
relaxing its own configurations as one batch -- independent work, no kernel
of one rank waits for the other's.  The gathered per-configuration results
(RK4 steps, final log10 L2, SHA-256 of the converged y_n) equal a
single-process sweep of the same configurations bit for bit: every tile
shape and batch composition gives identical steps.  Multi-GPU scaling of
the sweep is not measured here."""
import os
import socket

import pytest
import torch.multiprocessing as mp

from nrpyelliptic_b200 import _lib
from nrpyelliptic_b200.batch import sweep
from nrpyelliptic_b200.problem import sample_sweep

pytestmark = pytest.mark.gpu
GRIDS = ((32, 32, 8), (48, 48, 8))


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _worker(rank, world, port, q):
    os.environ.update(RANK=str(rank), WORLD_SIZE=str(world), LOCAL_RANK="0", MASTER_ADDR="127.0.0.1",
                      MASTER_PORT=str(port))
    from nrpyelliptic_b200.replicas import Replicas
    r = Replicas(backend="gloo", timeout_s=300)
    try:
        lib = _lib.load()
        lib.nrpyell_set_device(0)
        res, sec = sweep(sample_sweep(8, 31, grids=GRIDS), r, lib=lib)
        q.put((rank, res))
    except Exception as e:  # reported to the parent, which fails the test
        q.put((rank, repr(e)))
    finally:
        r.close()


def test_two_rank_sweep_equals_single_process_sweep():
    world = 2
    port = _free_port()
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_worker, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    out = sorted((q.get(timeout=600) for _ in range(world)), key=lambda x: x[0])
    for p in procs:
        p.join(timeout=120)
        assert p.exitcode == 0
    for rank, res in out:
        assert not isinstance(res, str), res
    lib = _lib.load()
    single, _ = sweep(sample_sweep(8, 31, grids=GRIDS), None, lib=lib)
    assert all(x["final_log10_l2"] <= -10.0 for x in single)
    for rank, res in out:
        assert res == single
