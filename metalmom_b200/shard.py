"""Clip sharding across GPUs (one process per GPU).

Clips are independent -- the only intra-clip coupling, the top_db floor's
clip-global maximum, never leaves the GPU that owns the clip -- so multi-GPU
work is a partition of clips with no collective on the data path.
"""

import heapq


def frames_of(length, n_fft=2048, hop=512, center=True):
    padded = length + (2 * (n_fft // 2) if center else 0)
    return 0 if padded < n_fft else 1 + (padded - n_fft) // hop


def balanced_shards(lengths, world, n_fft=2048, hop=512, center=True):
    """Assign clip indices to `world` ranks, balancing frame counts
    (longest-processing-time greedy; deterministic tie-break on rank)."""
    if world < 1:
        raise ValueError("world must be >= 1")
    order = sorted(range(len(lengths)), key=lambda i: (-frames_of(lengths[i], n_fft, hop, center), i))
    heap = [(0, r) for r in range(world)]
    shards = [[] for _ in range(world)]
    for i in order:
        load, r = heapq.heappop(heap)
        shards[r].append(i)
        heapq.heappush(heap, (load + frames_of(lengths[i], n_fft, hop, center), r))
    return [sorted(s) for s in shards]


def max_over_ranks(value, dist=None, device=None):
    """Max of a float over all ranks (elapsed-time reduction); identity without a group."""
    if dist is None or not dist.is_initialized():
        return float(value)
    import torch
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())
