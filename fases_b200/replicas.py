"""Independent replicas across the GPUs of one node: one process per GPU, each stepping its own
room; no collective on the data path. The only collectives are the host-side ones that bracket a
timed region (barrier) and take the slowest rank's time (max), over NCCL when the ranks have GPUs
and over gloo otherwise (the CPU tests). Ranks, world size and the local GPU come from the
torchrun environment (RANK, WORLD_SIZE, LOCAL_RANK, MASTER_ADDR, MASTER_PORT)."""
import datetime
import os


class Replicas:
    def __init__(self, backend=None, timeout_s=600):
        self.rank = int(os.environ.get("RANK", "0"))
        self.world = int(os.environ.get("WORLD_SIZE", "1"))
        self.local = int(os.environ.get("LOCAL_RANK", "0"))
        self.pg = None
        self.cuda = False
        if self.world > 1:
            import torch
            import torch.distributed as dist
            if backend is None:
                backend = "nccl" if torch.cuda.is_available() else "gloo"
            self.cuda = backend == "nccl"
            if self.cuda:
                torch.cuda.set_device(self.local)
            dist.init_process_group(backend, timeout=datetime.timedelta(seconds=timeout_s))
            self.pg = dist

    def barrier(self):
        """All ranks reach this point (and, on GPUs, their device work is done)."""
        if self.pg is None:
            return
        self.pg.barrier()
        if self.cuda:
            import torch
            torch.cuda.synchronize()

    def max(self, x):
        """The largest value of x over the ranks (the job's time is its slowest rank's)."""
        if self.pg is None:
            return float(x)
        import torch
        t = torch.tensor([float(x)], dtype=torch.float64, device="cuda" if self.cuda else "cpu")
        self.pg.all_reduce(t, op=self.pg.ReduceOp.MAX)
        return float(t.item())

    def aggregate_rate(self, units_per_rank, seconds):
        """Whole-job throughput of weak-scaled replicas: every rank's units over the slowest time."""
        return self.world * float(units_per_rank) / self.max(seconds)

    def close(self):
        if self.pg is not None:
            self.pg.destroy_process_group()
            self.pg = None
