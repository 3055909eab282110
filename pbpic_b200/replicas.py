"""Ranks of a multi-GPU run (one process per GPU) and independent replicas.

`Ranks` holds the process group, the barriers and the max-over-ranks
reduction of the timings that every multi-GPU run uses. With replicas, N GPUs
run N independent copies of a workload, each with its own seed, with no
data-path collective: the whole-job throughput is N x particles x steps / the
slowest rank's time (weak scaling). The batched ensemble is replicas only;
the single-domain step shards as y slabs (slab.py, bench.py's default for
N > 1).
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
