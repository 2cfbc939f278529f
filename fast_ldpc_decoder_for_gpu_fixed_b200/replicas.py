"""Multi-GPU use: independent replicas, one process per GPU.

Frames are independent, so the decoder shards by frame with no data-path
collective: every rank decodes its own batch (weak scaling).  The only
exchanges are host-level bookkeeping over torch.distributed: the max over
ranks of a timed region, and the sum of the Monte-Carlo counters (frames, bit
errors, frame errors) of a BER/FER simulation.  Each rank draws channel noise
from its own Philox stream (offset = rank), so no two ranks decode the same
frames.  The reference is single-GPU (src/main.cpp:113 hard-codes device 0).
"""
import torch
import torch.distributed as dist


def shard(total, rank, world, align=4):
    """Contiguous share [start, start+count) of `total` items for `rank`, in
    multiples of `align` (4 frames = one 32-bit word of the reference packing)."""
    units = total // align
    base, extra = divmod(units, world)
    start = rank * base + min(rank, extra)
    count = base + (1 if rank < extra else 0)
    return start * align, count * align


def channel_offset(rank, batch):
    """Philox offset of (rank, batch): disjoint noise streams for every rank and batch."""
    return (int(batch) << 16) | int(rank)


def max_over_ranks(value, device="cpu"):
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    if dist.is_available() and dist.is_initialized() and dist.get_world_size() > 1:
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def sum_counters(counts):
    """counts: int64 tensor [frames, bit_errors, frame_errors] -> summed over ranks (in place)."""
    if dist.is_available() and dist.is_initialized() and dist.get_world_size() > 1:
        dist.all_reduce(counts, op=dist.ReduceOp.SUM)
    return counts
