"""Host logic of multi-GPU runs: replicas only.

A stereo pair does not shard (vertical and diagonal paths cross any split of
the image), so N GPUs run N independent replicas, one process per GPU: each
rank takes its own frames or its own pairs of a batch, no collective touches
the data path, and a run's time is the maximum over the ranks' device times.
"""
import heapq


def shard_indices(weights, rank, world):
    """Indices of the items rank `rank` processes when `world` ranks share
    items of the given weights (e.g. W*H*D of each pair): longest first, each
    to the least-loaded rank (ties to the lowest rank), so every item goes to
    exactly one rank and the loads are balanced; deterministic."""
    if world < 1 or not 0 <= rank < world:
        raise ValueError("need 0 <= rank < world")
    order = sorted(range(len(weights)), key=lambda i: (-weights[i], i))
    heap = [(0, r) for r in range(world)]
    mine = []
    for i in order:
        load, r = heapq.heappop(heap)
        if r == rank:
            mine.append(i)
        heapq.heappush(heap, (load + weights[i], r))
    return sorted(mine)


def shard_pairs(pairs, rank, world):
    """This rank's share of a batch of stereo pairs, each (left, right,
    max_disp, ...) with (H, W) images: shard_indices over the pairs' cell
    counts W*H*D.  Returns (indices into `pairs`, those pairs); every rank
    then runs its own persistent batch (api.Batch) over its share."""
    weights = [int(p[0].shape[0]) * int(p[0].shape[1]) * int(p[2]) for p in pairs]
    idx = shard_indices(weights, rank, world)
    return idx, [pairs[i] for i in idx]


def max_over_ranks(values, device="cpu"):
    """Element-wise maximum of per-rank values (e.g. device milliseconds)
    over all ranks of the default process group; the values themselves when
    no group is initialised."""
    import torch
    import torch.distributed as dist
    t = torch.tensor([float(v) for v in values], dtype=torch.float64, device=device)
    if dist.is_available() and dist.is_initialized() and dist.get_world_size() > 1:
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return [float(v) for v in t.cpu()]
