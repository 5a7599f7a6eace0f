"""Multi-GPU form: frame pairs are independent, so GPUs act as replicas (one process per GPU, no
collective on the data path). Each rank computes a contiguous shard of the sequence's frame pairs;
per-frame values are gathered to rank 0 on the host, where the sequence mean is taken in frame
order with compensated summation, as the reference does (apps/QMIV/src/xMetricQMIV.cpp:98-102,
libs/pmbb-core/src/xKBNS.h:36-43)."""
from __future__ import annotations

import math


def shard(n_items: int, rank: int, world: int) -> range:
    """Contiguous block of item indices owned by `rank` (sizes differ by at most one)."""
    if world <= 0 or not 0 <= rank < world:
        raise ValueError("bad rank/world")
    base, extra = divmod(n_items, world)
    start = rank * base + min(rank, extra)
    return range(start, start + base + (1 if rank < extra else 0))


def kbns_sum(values) -> float:
    s = c = 0.0
    for v in values:
        t = s + v
        if abs(s) >= abs(v):
            c += (s - t) + v
        else:
            c += (v - t) + s
        s = t
    return s + c


def sequence_mean(per_frame) -> float:
    """xMetricStat::calcAvgMetric: compensated sum over frames in order, divided by the frame count."""
    per_frame = list(per_frame)
    if not per_frame:
        return math.nan
    return kbns_sum(per_frame) / float(len(per_frame))


def gather_ordered(local: list, indices: range, n_items: int, group=None) -> list | None:
    """Gather (index, value) pairs of every rank to rank 0 in sequence order (None on other ranks)."""
    import torch.distributed as dist
    world = dist.get_world_size(group)
    rank = dist.get_rank(group)
    mine = list(zip(indices, local))
    parts = [None] * world if rank == 0 else None
    dist.gather_object(mine, parts, dst=0, group=group)
    if rank != 0:
        return None
    out = [None] * n_items
    for part in parts:
        for i, v in part:
            out[i] = v
    return out
