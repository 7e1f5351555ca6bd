"""Multi-GPU plumbing: one process per GPU, profiles sharded across ranks.

Profiles are independent, so there is no collective on the data path: each
rank integrates its own disjoint share on its own engine and the results are
gathered to rank 0 on the host.  Timing uses the maximum over ranks.
torch.distributed (NCCL between GPUs, gloo on CPU) is used only for this
plumbing.
"""
from __future__ import annotations


def shard_indices(n, rank, world, costs=None):
    """Indices of the profiles rank `rank` integrates.  With `costs`, profiles are
    dealt largest-first to the least-loaded rank (greedy balancing); otherwise
    contiguous blocks."""
    if costs is None:
        base, extra = divmod(n, world)
        lo = rank * base + min(rank, extra)
        hi = lo + base + (1 if rank < extra else 0)
        return list(range(lo, hi))
    order = sorted(range(n), key=lambda i: -costs[i])
    load = [0.0] * world
    owner = [0] * n
    for i in order:
        r = min(range(world), key=lambda k: load[k])
        owner[i] = r
        load[r] += costs[i]
    return [i for i in range(n) if owner[i] == rank]


def gather_to_rank0(local, indices, n, group=None):
    """Gathers per-profile results (a list aligned with `indices`) to rank 0 in
    global order; returns the full list on rank 0 and None elsewhere."""
    import torch.distributed as dist

    world = dist.get_world_size(group)
    payload = list(zip(indices, local))
    parts = [None] * world if dist.get_rank(group) == 0 else None
    dist.gather_object(payload, parts, dst=0, group=group)
    if dist.get_rank(group) != 0:
        return None
    out = [None] * n
    for part in parts:
        for i, v in part:
            out[i] = v
    return out


def max_over_ranks(value, group=None, device=None):
    """Maximum of a float over all ranks (the slowest rank bounds the step)."""
    import torch
    import torch.distributed as dist

    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX, group=group)
    return float(t.item())
