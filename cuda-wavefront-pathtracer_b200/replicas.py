"""Replica runs on several GPUs of one node.

The diffuse path does not shard across GPUs: every (pixel, sample) path is independent, so each rank renders its own
frames (or traces its own ray batches, or serves its own request stream) on its own GPU, and only timings and counts
cross ranks. One process per GPU under torchrun; the barrier and the reductions go through torch.distributed (NCCL
between GPUs, gloo for the same calls on the CPU). Whole-job throughput = the units all ranks processed / the slowest
rank's time.
"""
import datetime
import os


class Replicas:
    def __init__(self, backend=None, timeout_s=120.0):
        self.ws = int(os.environ.get("WORLD_SIZE", "1"))
        self.rank = int(os.environ.get("RANK", "0"))
        self.local = int(os.environ.get("LOCAL_RANK", str(self.rank)))
        self.dist = None
        self.device = "cpu"
        if self.ws > 1:
            import torch
            import torch.distributed as dist
            backend = backend or ("nccl" if torch.cuda.is_available() else "gloo")
            kw = {}
            if backend == "nccl":
                self.device = f"cuda:{self.local}"
                kw["device_id"] = torch.device("cuda", self.local)
            dist.init_process_group(backend, timeout=datetime.timedelta(seconds=timeout_s), **kw)
            self.dist = dist

    def barrier(self):
        if self.dist is not None:
            self.dist.barrier()

    def _all_reduce(self, x, op):
        import torch
        t = torch.tensor([float(x)], dtype=torch.float64, device=self.device)
        self.dist.all_reduce(t, op=op)
        return float(t.item())

    def max(self, x):
        """the largest value over ranks (times: the job ends with its slowest rank)"""
        return float(x) if self.dist is None else self._all_reduce(x, self.dist.ReduceOp.MAX)

    def sum(self, x):
        """the total over ranks (units processed)"""
        return float(x) if self.dist is None else self._all_reduce(x, self.dist.ReduceOp.SUM)

    def throughput(self, units, seconds):
        """whole-job throughput: all ranks' units over the slowest rank's time (every rank takes part)"""
        total, slowest = self.sum(units), self.max(seconds)
        return total / slowest if slowest > 0 else 0.0, total, slowest

    def close(self):
        if self.dist is not None:
            self.dist.barrier()
            self.dist.destroy_process_group()
            self.dist = None
