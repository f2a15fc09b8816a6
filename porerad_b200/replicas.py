"""Independent replicas of the path on N GPUs of one node: one process per GPU.

Cases are independent, so N GPUs run N replicas with no collective on the data path.
The process group only brackets timed regions (barrier) and takes the maximum of the
per-rank device times.  NCCL on GPUs; gloo for the CPU tests of this logic.
"""

from __future__ import annotations

import os
from datetime import timedelta

_dist = None


def world_size() -> int:
    return int(os.environ.get("WORLD_SIZE", "1"))


def rank() -> int:
    return int(os.environ.get("RANK", "0"))


def local_rank() -> int:
    return int(os.environ.get("LOCAL_RANK", "0"))


def init(backend: str | None = None, timeout_s: float = 300.0) -> None:
    """Join the process group when launched with WORLD_SIZE > 1 (torchrun sets the env)."""

    global _dist
    if world_size() <= 1 or _dist is not None:
        return
    import torch.distributed as dist

    if backend is None:
        import torch

        backend = "nccl" if torch.cuda.is_available() else "gloo"
    os.environ.setdefault("MASTER_ADDR", "127.0.0.1")
    dist.init_process_group(backend, timeout=timedelta(seconds=timeout_s))
    _dist = dist


def barrier() -> None:
    if _dist is not None:
        _dist.barrier()


def max_over_ranks(values):
    """Element-wise maximum of a list of floats over all ranks (identity with one rank)."""

    values = [float(v) for v in values]
    if _dist is None:
        return values
    import torch

    dev = "cuda" if _dist.get_backend() == "nccl" else "cpu"
    t = torch.tensor(values, dtype=torch.float64, device=dev)
    _dist.all_reduce(t, op=_dist.ReduceOp.MAX)
    return [float(v) for v in t.cpu()]


def all_equal(values) -> bool:
    """True when every rank passed the same list of integers (True with one rank).

    Replicas of a seeded case must agree to the last integer (DDA steps, pairs per ray set);
    the check takes the element-wise minimum and maximum over the ranks and compares them.
    """

    values = [int(v) for v in values]
    if _dist is None:
        return True
    import torch

    dev = "cuda" if _dist.get_backend() == "nccl" else "cpu"
    lo = torch.tensor(values, dtype=torch.int64, device=dev)
    hi = lo.clone()
    _dist.all_reduce(lo, op=_dist.ReduceOp.MIN)
    _dist.all_reduce(hi, op=_dist.ReduceOp.MAX)
    return bool(torch.equal(lo.cpu(), hi.cpu()))


def finalize() -> None:
    global _dist
    if _dist is not None:
        _dist.barrier()
        _dist.destroy_process_group()
        _dist = None
