"""Sample-parallel distribution over one process per GPU (torch.distributed).

The reference distributes complete statistics blocks round robin over MPI
ranks, keeps H and S replicated, and gathers the raw float64 block sums to the
root, which normalises once (src/kubo_msd/parallel.py:11-102,
src/kubo_msd/solvers/stochastic.py:122-218).  Here the ranks are the
processes of a torch.distributed group (NCCL between GPUs, gloo on CPU); the
only data exchange is the gather of the float64 block sums, a few KB to MB,
so it goes through the process group's object collectives.  Every stage
agrees on success before the next collective, so a failing rank makes every
rank raise instead of leaving the others waiting.
"""
from __future__ import annotations

import numpy as np

from .errors import KuboMSDError, NumericalError


def owned_blocks(nsamples, block_size, rank, size):
    """Round-robin ownership of statistics blocks (parallel.py:11-14)."""
    if nsamples < 1 or block_size < 1 or size < 1 or not 0 <= rank < size:
        raise KuboMSDError("invalid sample/block/rank partition")
    return list(range(rank, (nsamples + block_size - 1) // block_size, size))


class ParallelContext:
    """Serial when `group` is None; otherwise over an initialised process group."""

    def __init__(self, distributed=False):
        self.dist = None
        self.rank, self.size = 0, 1
        if distributed:
            import torch.distributed as dist
            if not dist.is_initialized():
                raise KuboMSDError("distributed transport requires an initialised torch.distributed group")
            self.dist = dist
            self.rank, self.size = dist.get_rank(), dist.get_world_size()

    @property
    def root(self):
        return self.rank == 0

    def allgather(self, value):
        if self.dist is None:
            return [value]
        out = [None] * self.size
        self.dist.all_gather_object(out, value)
        return out

    def broadcast(self, value):
        if self.dist is None:
            return value
        box = [value]
        self.dist.broadcast_object_list(box, src=0)
        return box[0]

    def stage(self, label, action, root_only=False):
        """Run local work, then agree on success before the next collective
        (parallel.py:46-62)."""
        result, error = None, None
        try:
            if not root_only or self.root:
                result = action()
        except Exception as exc:  # noqa: BLE001
            if self.dist is None:
                raise
            error = {"rank": self.rank, "type": type(exc).__name__, "message": str(exc)}
        errors = [e for e in self.allgather(error) if e is not None]
        if errors:
            failure = NumericalError(f"distributed stage {label!r} failed: " +
                                     "; ".join(f"rank {e['rank']}: {e['message']}" for e in errors))
            failure.diagnostics = {"stage": label, "failures": errors}
            raise failure
        return result

    def root_call(self, label, action):
        return self.broadcast(self.stage(label, action, root_only=True))

    def gather_blocks(self, local, block_ids, nblocks):
        """Disjoint float64 block slabs gathered to root in global order
        (parallel.py:68-102)."""
        if self.dist is None:
            if list(block_ids) != list(range(nblocks)):
                raise NumericalError("serial block coverage mismatch")
            return np.asarray(local)
        local = np.ascontiguousarray(local, dtype=np.float64)
        parts = self.allgather((list(block_ids), local))
        ids = [j for part, _ in parts for j in part]
        if sorted(ids) != list(range(nblocks)):
            raise NumericalError("distributed statistical blocks must cover the global set exactly once")
        tails = {arr.shape[1:] for _, arr in parts}
        if len(tails) != 1 or any(arr.shape[0] != len(part) for part, arr in parts):
            raise NumericalError("distributed statistical block shapes disagree")
        if not self.root:
            return None
        packed = np.concatenate([arr for _, arr in parts], axis=0)
        result = np.empty_like(packed)
        result[np.asarray(ids, dtype=int)] = packed
        return result

    def metadata(self):
        return {"distribution": "torch.distributed" if self.dist is not None else "serial",
                "world_size": self.size, "partition": "complete global statistics blocks, round robin",
                "operator_storage": "replicated per rank",
                "reduction": "raw numerator and DOS block sums, normalized once on root",
                "backend": self.dist.get_backend() if self.dist is not None else None}
