"""Frame-range sharding across GPUs (one process per GPU).

Output frames are independent given their 2r+1 source frames, so a clip is
split into contiguous output ranges; each rank also needs r frames of halo
on each side (clamped at the clip ends, cpu_source/getframe_impl.cpp:296-298).
No data-path collective is involved; only timings are reduced.
"""
from __future__ import annotations


def frame_shard(total: int, rank: int, world: int, radius: int) -> tuple[int, int, int, int]:
    """(out_lo, out_hi, in_lo, in_hi) for ``rank`` of ``world``."""
    if not 0 <= rank < world:
        raise ValueError("rank out of range")
    lo = total * rank // world
    hi = total * (rank + 1) // world
    in_lo = max(lo - radius, 0)
    in_hi = min(hi + radius, total)
    return lo, hi, in_lo, in_hi


def max_over_ranks(value: float, distributed: bool) -> float:
    """Max of a host scalar over all ranks (timings are taken as the slowest rank)."""
    if not distributed:
        return value
    import torch
    import torch.distributed as dist

    dev = torch.device("cuda", torch.cuda.current_device()) if dist.get_backend() == "nccl" else torch.device("cpu")
    t = torch.tensor([float(value)], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())
