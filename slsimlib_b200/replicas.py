"""Host-side plumbing for running the ray-shooting path on several GPUs.

Rays are independent and lenses are read-only, so the path needs no
collective: every process (one per GPU) holds a replica of the lens and shoots
its own rays.  Two layouts:

* weak scaling (``bench.py``): every rank shoots a full grid;
* strong scaling: one grid split into contiguous, Morton-ordered ray ranges,
  ``shard(n, rank, world)``.

The only communication is timing: ``max_over_ranks`` (the slowest rank sets
the wall time) and barriers, over whatever torch.distributed backend the
process group uses (NCCL on GPUs, gloo in the CPU tests).
"""
from __future__ import annotations


def shard(n: int, rank: int, world: int) -> tuple[int, int]:
    """Contiguous range [lo, hi) of n rays for `rank`; sizes differ by <= 1."""
    if world <= 0 or not 0 <= rank < world:
        raise ValueError("rank outside [0, world)")
    q, r = divmod(n, world)
    lo = rank * q + min(rank, r)
    return lo, lo + q + (1 if rank < r else 0)


def max_over_ranks(value: float, device=None) -> float:
    """The largest `value` over all ranks (1 process: the value itself)."""
    import torch
    import torch.distributed as dist
    if not (dist.is_available() and dist.is_initialized()) or dist.get_world_size() == 1:
        return float(value)
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())
