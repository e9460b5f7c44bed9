"""One process per GPU for independent relaxations (replicas).

A single relaxation does not shard across GPUs (the inner boundary gathers
across the axis and the RK4 stages are sequential), so multi-GPU runs solve
independent puncture configurations per rank: no collective touches the data
path.  torch.distributed supplies only the plumbing around it -- a barrier
before and after a timed region, the max of the per-rank times and the
gathering of per-configuration results on the host after a sharded sweep --
over NCCL on GPUs (gloo on CPU-only hosts and in the tests).
"""
import datetime
import os


class Replicas:
    def __init__(self, backend=None, timeout_s=300):
        self.rank = int(os.environ.get("RANK", "0"))
        self.world = int(os.environ.get("WORLD_SIZE", "1"))
        self.local_rank = int(os.environ.get("LOCAL_RANK", "0"))
        self.torch = None
        self.dist = None
        if self.world > 1:
            import torch
            import torch.distributed as dist
            self.torch = torch
            self.dist = dist
            if backend is None:
                backend = "nccl" if torch.cuda.is_available() else "gloo"
            self.backend = backend
            if backend == "nccl":
                torch.cuda.set_device(self.local_rank)
            dist.init_process_group(backend, timeout=datetime.timedelta(seconds=timeout_s))

    def _device(self):
        return "cuda" if self.backend == "nccl" else "cpu"

    def barrier(self):
        if self.dist:
            self.dist.barrier()

    def max(self, x):
        """Maximum of a float over ranks."""
        if not self.dist:
            return float(x)
        t = self.torch.tensor([float(x)], dtype=self.torch.float64, device=self._device())
        self.dist.all_reduce(t, op=self.dist.ReduceOp.MAX)
        return float(t.item())

    def sum(self, x):
        if not self.dist:
            return float(x)
        t = self.torch.tensor([float(x)], dtype=self.torch.float64, device=self._device())
        self.dist.all_reduce(t, op=self.dist.ReduceOp.SUM)
        return float(t.item())

    def all_gather(self, obj):
        """Every rank's `obj` (picklable host data), in rank order, on every
        rank -- for gathering per-configuration results after the solves."""
        if not self.dist:
            return [obj]
        out = [None] * self.world
        self.dist.all_gather_object(out, obj)
        return out

    def close(self):
        if self.dist:
            self.dist.destroy_process_group()
            self.dist = None


def shard(items, rank, world):
    """The items of `rank` when len(items) work units are dealt round-robin
    over `world` ranks (every unit on exactly one rank)."""
    return [it for i, it in enumerate(items) if i % world == rank]


def throughput(units_per_rank, seconds_per_rank, reps):
    """Whole-job throughput: all units processed / slowest rank's time."""
    return reps * units_per_rank / seconds_per_rank
