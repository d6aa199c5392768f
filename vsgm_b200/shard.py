"""Multi-GPU sharding of one view's roots (one process per GPU).

Every match is rooted at exactly one source, so a view's sources split into
disjoint shards with no data exchange; the only collective is one sum of the
per-query uint64 counts (the reference sums per-consumer counts on the host,
src/app/pattern_matching_pipeline.cu:191-195).
"""
import numpy as np


def roots_of_rank(n_sources, rank, world, sources=None):
    """Strided shard: rank r takes sources r, r + world, ... (balances hubs, which
    cluster at one end of a degree-ordered id range)."""
    idx = np.arange(rank, n_sources, world, dtype=np.uint64)
    if sources is None:
        return idx.astype(np.uint32)
    return np.ascontiguousarray(np.asarray(sources, dtype=np.uint32)[idx])


def allreduce_counts(counts, device=None):
    """Sum per-rank exact counts across the process group (int64 tensors; counts < 2^63)."""
    import torch
    import torch.distributed as dist

    t = torch.tensor([int(c) for c in counts], dtype=torch.int64, device=device)
    if dist.is_initialized() and dist.get_world_size() > 1:
        dist.all_reduce(t)
    return [int(x) for x in t.tolist()]
