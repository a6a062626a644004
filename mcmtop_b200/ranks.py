"""Host side of a multi-GPU run: one process per GPU, each advancing its own
independent bodies (the weak-scaling partition of independent bodies; one
body is never split across GPUs, so no collective sits on the data path).
The collectives are the barrier around the timed region, the maximum of the
ranks' device times, which makes the job's time that of its slowest rank, and
after the run the gathering of per-body results (losses, gradients) and of
the ranks' work counts."""
from __future__ import annotations

import os


def dist_env() -> tuple:
    """(world size, rank, local rank) from the launcher's environment."""
    return (int(os.environ.get("WORLD_SIZE", "1")), int(os.environ.get("RANK", "0")),
            int(os.environ.get("LOCAL_RANK", "0")))


def max_over_ranks(ms: float, device: str = "cpu") -> float:
    """The largest ms of all ranks (all_reduce MAX of one float64; `device`
    is where the backend wants the tensor: a CUDA device for NCCL, the CPU for
    gloo).  Returns ms unchanged without a process group."""
    import torch
    import torch.distributed as dist

    if not (dist.is_available() and dist.is_initialized()) or dist.get_world_size() == 1:
        return ms
    t = torch.tensor([ms], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def job_rate(units_per_rank: float, world_size: int, ms_max: float) -> float:
    """Whole-job throughput: the units all ranks processed over the slowest
    rank's time."""
    return world_size * units_per_rank / (ms_max / 1e3)


def share(n_items: int, world_size: int, rank: int) -> range:
    """The contiguous block of n_items (bodies of an ensemble) that a rank
    owns; the blocks of all ranks cover every item once."""
    base, extra = divmod(n_items, world_size)
    start = rank * base + min(rank, extra)
    return range(start, start + base + (1 if rank < extra else 0))


def gather_items(values: dict, n_items: int, device: str = "cpu", width: int = 1):
    """Per-item results of an ensemble, gathered on every rank: each rank
    passes {item index: value (a float or `width` floats)} for the items it
    owns (its share), and gets back an (n_items, width) float64 array holding
    every rank's values (all_reduce SUM of zero-filled blocks, so each entry
    is exactly the owner's value).  Without a process group the array holds
    the local values only."""
    import numpy as np
    import torch
    import torch.distributed as dist

    buf = np.zeros((n_items, width), dtype=np.float64)
    for k, v in values.items():
        buf[k] = v
    if not (dist.is_available() and dist.is_initialized()) or dist.get_world_size() == 1:
        return buf
    t = torch.from_numpy(buf).to(device)
    dist.all_reduce(t, op=dist.ReduceOp.SUM)
    return t.cpu().numpy()


def sum_over_ranks(x: float, device: str = "cpu") -> float:
    """The sum of x over all ranks (x alone without a process group)."""
    import torch
    import torch.distributed as dist

    if not (dist.is_available() and dist.is_initialized()) or dist.get_world_size() == 1:
        return x
    t = torch.tensor([x], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.SUM)
    return float(t.item())
