"""Multi-GPU plumbing: one process per GPU.

The solver's configurations are single domains and the batched and
warm-start workloads are sets of independent problems, so several GPUs run
either replicas of one problem or disjoint shares of a problem set.  The
lattice steps exchange nothing; the collectives are the final timing and
count reductions (max of device times, sum of updates) and, for the
surrogate's data-parallel training, one flat all-reduce of the gradients
per step and of the output statistics once.  They run on the process group
`torch.distributed` opened from the launcher's environment (RANK,
WORLD_SIZE, MASTER_ADDR, MASTER_PORT), over NCCL on GPUs or gloo on CPUs.
The reference has no multi-GPU path.
"""

from __future__ import annotations

import os
from datetime import timedelta


def world_from_env() -> tuple[int, int, int]:
    """(world size, rank, local rank) of this process."""
    return (int(os.environ.get("WORLD_SIZE", "1")), int(os.environ.get("RANK", "0")),
            int(os.environ.get("LOCAL_RANK", "0")))


def init(backend: str | None = None, timeout_s: float = 600.0) -> tuple[int, int, int]:
    """Open the default process group when WORLD_SIZE > 1."""
    world, rank, local = world_from_env()
    if world > 1:
        import torch
        import torch.distributed as dist

        if not dist.is_initialized():
            if backend is None:
                backend = "nccl" if torch.cuda.is_available() else "gloo"
            dist.init_process_group(backend, timeout=timedelta(seconds=timeout_s))
    return world, rank, local


def deal(items, rank: int, world: int):
    """Round-robin share of `items` for `rank` (instances of uneven size
    spread evenly on average)."""
    return list(items)[rank::world]


def reduce_times_and_counts(times, counts, device=None):
    """(max over ranks of each time, sum over ranks of each count)."""
    import torch
    import torch.distributed as dist

    t = torch.tensor([float(v) for v in times], dtype=torch.float64, device=device)
    c = torch.tensor([float(v) for v in counts], dtype=torch.float64, device=device)
    if dist.is_available() and dist.is_initialized() and dist.get_world_size() > 1:
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        dist.all_reduce(c, op=dist.ReduceOp.SUM)
    return [float(v) for v in t.tolist()], [float(v) for v in c.tolist()]


def world_and_rank() -> tuple[int, int]:
    """(world size, rank) of the open process group, (1, 0) without one."""
    import torch.distributed as dist

    if dist.is_available() and dist.is_initialized():
        return dist.get_world_size(), dist.get_rank()
    return 1, 0


def allreduce_(tensors, op: str = "sum") -> None:
    """Reduce `tensors` (one dtype, one device) elementwise over the ranks in
    place, through one flat buffer: op "sum" or "max".  No-op on one rank."""
    world, _ = world_and_rank()
    tensors = list(tensors)
    if world == 1 or not tensors:
        return
    import torch
    import torch.distributed as dist

    flat = torch.cat([t.reshape(-1) for t in tensors])
    dist.all_reduce(flat, op=dist.ReduceOp.SUM if op == "sum" else dist.ReduceOp.MAX)
    off = 0
    for t in tensors:
        n = t.numel()
        t.copy_(flat[off:off + n].view_as(t))
        off += n


def finalize() -> None:
    import torch.distributed as dist

    if dist.is_available() and dist.is_initialized():
        dist.destroy_process_group()
