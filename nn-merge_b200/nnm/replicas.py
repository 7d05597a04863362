"""Host side of a multi-GPU run in which every rank builds its own graph
(independent replicas, weak scaling): one process per GPU, launched by
torchrun; ranks meet only at barriers around the timed region and for the
max of their timings.  There is no data-path collective: builds do not
exchange anything.
"""
import datetime
import os


class Replicas:
    """Rank, world size and the few collectives a replicated run needs.

    backend "nccl" on GPUs (tensors on the rank's device), "gloo" on CPU.
    With WORLD_SIZE 1 (or unset) nothing is initialised and every call is
    local.
    """

    def __init__(self, backend="nccl", timeout_s=600):
        self.rank = int(os.environ.get("RANK", "0"))
        self.world = int(os.environ.get("WORLD_SIZE", "1"))
        self.local = int(os.environ.get("LOCAL_RANK", "0"))
        self.backend = backend
        self._dist = None
        if self.world > 1:
            import torch.distributed as dist
            dist.init_process_group(backend, timeout=datetime.timedelta(seconds=timeout_s))
            self._dist = dist

    @property
    def leader(self):
        """Only rank 0 prints the result line."""
        return self.rank == 0

    def data_seed(self, base):
        """Every rank builds from its own seeded data."""
        return base + self.rank

    def barrier(self):
        if self._dist:
            self._dist.barrier()

    def max(self, v):
        """The max of a float over ranks (a timing: the slowest rank)."""
        if not self._dist:
            return float(v)
        import torch
        dev = "cuda" if self.backend == "nccl" else "cpu"
        t = torch.tensor([float(v)], dtype=torch.float64, device=dev)
        self._dist.all_reduce(t, op=self._dist.ReduceOp.MAX)
        return float(t.item())

    def close(self):
        if self._dist:
            self._dist.destroy_process_group()
            self._dist = None
