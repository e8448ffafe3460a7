"""Host-side plumbing for running the ray-shooting path on several GPUs.

Rays are independent and lenses are read-only, so the path needs no
collective: every process (one per GPU) holds a replica of the lens and shoots
its own grid (weak scaling, ``bench.py --gpus N``).  The only communication is
timing: ``max_over_ranks`` (the slowest rank sets the time) over whatever
torch.distributed backend the process group uses (NCCL on GPUs, gloo in the
CPU tests).
"""
from __future__ import annotations


def max_over_ranks(value: float, device=None) -> float:
    """The largest `value` over all ranks (1 process: the value itself)."""
    import torch
    import torch.distributed as dist
    if not (dist.is_available() and dist.is_initialized()) or dist.get_world_size() == 1:
        return float(value)
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())
