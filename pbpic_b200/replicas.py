"""Independent replicas, one process per GPU.

The single-domain step does not shard in this library (the y-slab
decomposition of the reference's MPI version is not built), so N GPUs run N
independent replicas of a workload, each with its own seed. There is no
data-path collective: ranks meet only at barriers and in the reduction of the
timings (the slowest rank's time), and the whole-job throughput is
N x particles x steps / that time (weak scaling).
"""
import datetime
import os


class Ranks:
    def __init__(self, backend="nccl", timeout_s=120):
        self.world = int(os.environ.get("WORLD_SIZE", "1"))
        self.rank = int(os.environ.get("RANK", "0"))
        self.local_rank = int(os.environ.get("LOCAL_RANK", "0"))
        self.backend = backend
        self.dist = None
        if self.world > 1:
            import torch.distributed as dist
            dist.init_process_group(backend, timeout=datetime.timedelta(seconds=timeout_s))
            self.dist = dist

    def replica_seed(self, seed):
        """Seed of this rank's replica: independent plasmas on every rank."""
        return seed + self.rank

    def barrier(self):
        if self.dist is not None:
            self.dist.barrier()

    def max(self, x):
        """Maximum of x over ranks (the job's time is the slowest rank's)."""
        if self.dist is None:
            return float(x)
        import torch
        dev = "cuda" if self.backend == "nccl" else "cpu"
        t = torch.tensor([float(x)], dtype=torch.float64, device=dev)
        self.dist.all_reduce(t, op=self.dist.ReduceOp.MAX)
        return float(t.item())

    def throughput(self, units_per_rank, steps, max_ms):
        """Whole-job units per second: every rank processed units_per_rank x steps."""
        return self.world * units_per_rank * steps / (max_ms * 1e-3)

    def close(self):
        if self.dist is not None:
            self.dist.destroy_process_group()
            self.dist = None
