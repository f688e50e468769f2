"""Replica plumbing for one process per GPU.

The assemble + solve path does not shard: N GPUs run N independent copies of
the workload (weak scaling).  The only collectives are the barriers around a
timed region and the maximum of the per-rank times; none is on the data path.
Rank, world size and local rank come from the launcher's environment (RANK,
WORLD_SIZE, LOCAL_RANK, MASTER_ADDR, MASTER_PORT)."""
import datetime
import os


def env():
    return (int(os.environ.get("WORLD_SIZE", "1")), int(os.environ.get("RANK", "0")),
            int(os.environ.get("LOCAL_RANK", "0")))


class Replicas:
    def __init__(self, backend="nccl", timeout_s=600):
        self.ws, self.rank, self.local = env()
        self.dist = None
        self.device = "cpu"
        if self.ws > 1:
            import torch
            import torch.distributed as dist
            if backend == "nccl":
                torch.cuda.set_device(self.local)
                self.device = "cuda"
            dist.init_process_group(backend, init_method="env://", timeout=datetime.timedelta(seconds=timeout_s))
            self.dist = dist

    def barrier(self):
        if self.dist:
            self.dist.barrier()

    def max(self, value):
        """Maximum of a per-rank value (a time) over all ranks."""
        if not self.dist:
            return float(value)
        import torch
        t = torch.tensor([float(value)], dtype=torch.float64, device=self.device)
        self.dist.all_reduce(t, op=self.dist.ReduceOp.MAX)
        return float(t.item())

    def job_rate(self, units_per_rank, seconds_max):
        """Whole-job throughput: every rank processed units_per_rank in at most seconds_max."""
        return self.ws * units_per_rank / seconds_max

    def close(self):
        if self.dist:
            self.dist.barrier()
            self.dist.destroy_process_group()
            self.dist = None
