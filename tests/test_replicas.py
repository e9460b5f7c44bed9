"""Multi-process plumbing of the replica runs (bench.py --gpus N): two gloo
ranks on the CPU exercise the barrier, the max-over-ranks timing and the
round-robin sharding of configurations.  No GPU work."""
import os
import socket

import pytest
import torch.multiprocessing as mp

from nrpyelliptic_b200.replicas import Replicas, shard, throughput


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _worker(rank, world, port, q):
    os.environ.update(RANK=str(rank), WORLD_SIZE=str(world), LOCAL_RANK=str(rank), MASTER_ADDR="127.0.0.1",
                      MASTER_PORT=str(port))
    r = Replicas(backend="gloo", timeout_s=60)
    try:
        r.barrier()
        t_max = r.max(1.0 + rank)          # per-rank "time"
        units = r.sum(len(shard(list(range(64)), rank, world)))
        mine = shard(list(range(64)), rank, world)
        q.put((rank, t_max, units, mine))
        r.barrier()
    finally:
        r.close()


def test_two_rank_gloo_barrier_max_and_shard():
    world = 2
    port = _free_port()
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_worker, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    out = [q.get(timeout=120) for _ in range(world)]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    out.sort()
    assert [o[1] for o in out] == [2.0, 2.0]          # both ranks see the slowest rank's time
    assert [o[2] for o in out] == [64.0, 64.0]        # every configuration counted once
    mine0, mine1 = out[0][3], out[1][3]
    assert not set(mine0) & set(mine1) and sorted(mine0 + mine1) == list(range(64))
    # whole-job throughput: all ranks' units over the slowest rank's time
    assert throughput(32 * world, 2.0, 3) == pytest.approx(96.0)


def test_single_process_is_a_no_op():
    r = Replicas()
    assert r.world == 1 and r.max(3.5) == 3.5 and r.sum(2.0) == 2.0
    r.barrier()
    r.close()
