"""Execution backends for the ensemble drivers.

Restates the reference's execution interface (``src/driver/execution.jl``:
``_rank``, ``_nprocs``, ``_phase``, ``_gather``, ``_broadcast``,
``_check_arguments``) and its MPI extension (``ext/StoPEPSMPIExt.jl:8-51``)
over ``torch.distributed`` (NCCL between GPUs, gloo on CPU).  Samples are
independent after the shared sampling cache, so the only exchanges are the
gathers of per-sample scalar records; there is no data-path collective.
"""
from __future__ import annotations


class SerialExecution:
    """``SerialExecution`` (``src/driver/execution.jl:1-34``)."""

    def rank(self):
        return 0

    def nprocs(self):
        return 1

    def phase(self, f):
        return f()

    def gather(self, x):
        return [x]

    def broadcast(self, f):
        return f()

    def check_arguments(self, signature):
        return None


class TorchExecution:
    """One process per rank over an initialised ``torch.distributed`` group.

    ``phase`` runs a local piece of work and then exchanges error strings, so
    a failure on any rank raises the same error on every rank
    (``ext/StoPEPSMPIExt.jl:17-29``).
    """

    def __init__(self, group=None):
        import torch.distributed as dist
        if not dist.is_initialized():
            raise RuntimeError("torch.distributed is not initialised")
        self.dist = dist
        self.group = group

    def rank(self):
        return self.dist.get_rank(self.group)

    def nprocs(self):
        return self.dist.get_world_size(self.group)

    def gather(self, x):
        out = [None] * self.nprocs()
        self.dist.all_gather_object(out, x, group=self.group)
        return out

    def broadcast(self, f):
        box = [f() if self.rank() == 0 else None]
        self.dist.broadcast_object_list(box, src=0, group=self.group)
        return box[0]

    def phase(self, f):
        result, err = None, None
        try:
            result = f()
        except Exception as ex:   # collected, then raised on every rank
            err = f"rank {self.rank()}: {type(ex).__name__}: {ex}"
        errors = [m for m in self.gather(err) if m is not None]
        if errors:
            raise RuntimeError("; ".join(errors))
        return result

    def check_arguments(self, signature):
        """``_check_arguments`` (``src/driver/execution.jl:17-23``)."""
        sigs = self.gather(signature)
        if any(s != sigs[0] for s in sigs):
            raise RuntimeError("MPI ranks supplied different parameters")
