"""Sweeps sharded by configuration over ranks (batch.sweep,
learned.solve_snapshots with a Replicas): two gloo ranks on the CPU with a
stand-in solver check that every configuration is solved exactly once, on
rank i % world, and that the gathered results come back in the sweep's
order on every rank.  No GPU work (the solver is a host function)."""
import os
import socket

import torch.multiprocessing as mp

from nrpyelliptic_b200.batch import sweep
from nrpyelliptic_b200.problem import sample_sweep
from nrpyelliptic_b200.replicas import Replicas


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def fake_solve(cfgs, tag):
    rank = int(os.environ["RANK"])
    return [{"name": c.name, "rank": rank, "steps": len(c.name) + int(c.name[-2:]), "tag": tag} for c in cfgs]


def _worker(rank, world, port, q):
    os.environ.update(RANK=str(rank), WORLD_SIZE=str(world), LOCAL_RANK=str(rank), MASTER_ADDR="127.0.0.1",
                      MASTER_PORT=str(port))
    r = Replicas(backend="gloo", timeout_s=60)
    try:
        cfgs = sample_sweep(11, 5)
        res, sec = sweep(cfgs, r, solve=fake_solve, tag="x")
        q.put((rank, res, sec))
    finally:
        r.close()


def test_two_rank_sweep_solves_each_configuration_once_and_gathers_in_order():
    world = 2
    port = _free_port()
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_worker, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    out = sorted(q.get(timeout=120) for _ in range(world))
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    cfgs = sample_sweep(11, 5)
    single, _ = sweep(cfgs, None, solve=lambda c, tag: [dict(x, rank=i % world) for i, x in
                                                        enumerate(fake_solve_local(c, tag))], tag="x")
    for rank, res, sec in out:
        assert [x["name"] for x in res] == [c.name for c in cfgs]
        assert [x["rank"] for x in res] == [i % world for i in range(len(cfgs))]
        assert res == single
        assert sec >= 0.0


def fake_solve_local(cfgs, tag):
    return [{"name": c.name, "rank": 0, "steps": len(c.name) + int(c.name[-2:]), "tag": tag} for c in cfgs]
