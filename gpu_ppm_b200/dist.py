"""Multi-GPU plumbing: one process per GPU.

Batches of independent profiles shard by profile: each rank integrates its own
disjoint share on its own engine and the results are gathered to rank 0 on the
host, with no collective on the data path.  One large profile (N_side >= 512)
shards by HEALPix ring instead: the rings are split into contiguous windows of
about equal work, every rank integrates its window (ppm_batch_create_rings) and
one sum-reduce of the flux and counts pools to rank 0 finishes the profile —
the only collective, since flux and counts are linear in the rings.  Timing
uses the maximum over ranks.  torch.distributed (NCCL between GPUs, gloo on
CPU) carries the plumbing.
"""
from __future__ import annotations

import math

import numpy as np


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


# ---------------------------------------------------------------------------- ring sharding
def _ring_z_phi(N, i):
    """Centre cos(theta) of HEALPix ring i and the azimuths of its elements
    (cpu/grid.hpp:194-250, gpu/healpix.cuh:12-91)."""
    ii = i if i <= 2 * N else 4 * N - i
    if ii < N:
        z = 1.0 - ii * ii / (3.0 * N * N)
        jmax = 4 * ii
        phi = math.pi / (2.0 * ii) * (np.arange(1, jmax + 1) - 0.5)
    else:
        z = (4.0 / 3.0) - 2.0 * ii / (3.0 * N)
        jmax = 4 * N
        s = (ii - N + 1) % 2
        phi = math.pi / (2.0 * N) * (np.arange(1, jmax + 1) - s / 2.0)
    return (z if i <= 2 * N else -z), phi


def ring_costs(p):
    """Work per ring index 0 .. 4 N_side - 1 of a profile: active elements of each
    HEALPix ring (index 0 holds point-source spots).  Used only for balancing."""
    N = p.n_side
    costs = np.zeros(4 * N)
    for k in range(p.n_spots):
        sp = p.spots[k]
        if sp.kind == 1:
            costs[0] += 1.0
            continue
        c1, s1 = math.cos(sp.theta1), math.sin(sp.theta1)
        c2, s2 = math.cos(sp.theta2), math.sin(sp.theta2)
        ca1, ca2 = math.cos(sp.angrad1), math.cos(sp.angrad2)
        for i in range(1, 4 * N):
            z, phi = _ring_z_phi(N, i)
            st = math.sqrt(max(0.0, 1.0 - z * z))
            # the disk's latitude band first: most rings hold nothing
            if abs(math.acos(max(-1.0, min(1.0, z))) - sp.theta1) > abs(sp.angrad1) + 1e-9 and abs(sp.angrad1) < math.pi:
                continue
            in1 = s1 * st * np.cos(phi - sp.phi1) + c1 * z > ca1
            in2 = s2 * st * np.cos(phi - sp.phi2) + c2 * z > ca2
            costs[i] += float(np.count_nonzero(in1 & ~in2))
    return costs


def ring_partition(costs, world):
    """Contiguous ring windows [begin, end), one per rank, covering all ring
    indices, each holding about 1/world of the total cost."""
    costs = np.asarray(costs, dtype=np.float64)
    n = len(costs)
    total = costs.sum()
    cum = np.cumsum(costs)
    bounds = [0]
    for r in range(1, world):
        target = total * r / world
        b = int(np.searchsorted(cum, target, side="left")) + 1 if total > 0 else (n * r) // world
        bounds.append(min(n, max(bounds[-1], b)))
    bounds.append(n)
    return [(bounds[r], bounds[r + 1]) for r in range(world)]


def reduce_sum_to_rank0(arrays, group=None, device=None):
    """Sums equal-shaped arrays over all ranks into rank 0 (numpy arrays on CPU,
    torch tensors as given).  Returns the sums on rank 0 and None elsewhere."""
    import torch
    import torch.distributed as dist

    out = []
    for a in arrays:
        t = a if isinstance(a, torch.Tensor) else torch.from_numpy(np.ascontiguousarray(a, dtype=np.float64))
        if device is not None:
            t = t.to(device)
        dist.reduce(t, dst=0, op=dist.ReduceOp.SUM, group=group)
        out.append(t)
    if dist.get_rank(group) != 0:
        return None
    return [t.cpu().numpy() if isinstance(t, torch.Tensor) else t for t in out]


class _DevicePool:
    """A device array of doubles exposed to torch without a copy."""

    def __init__(self, ptr, n):
        self.__cuda_array_interface__ = {"shape": (int(n),), "typestr": "<f8", "data": (int(ptr), False),
                                         "version": 3}


def profile_sharded(engine, p, group=None, stream=0):
    """One profile split over the ranks of `group` by HEALPix ring: every rank
    integrates its ring window on its own GPU and the flux and counts pools are
    sum-reduced (NCCL) into rank 0.  Returns (flux, counts) as host arrays on
    rank 0 and (None, None) elsewhere."""
    import torch
    import torch.distributed as dist

    world, rank = dist.get_world_size(group), dist.get_rank(group)
    windows = ring_partition(ring_costs(p), world)
    batch = engine.batch([p], rings=windows[rank])
    try:
        batch.launch(stream)
        torch.cuda.synchronize()
        flux = torch.as_tensor(_DevicePool(batch.flux_ptr, batch.n_flux), device="cuda")
        counts = torch.as_tensor(_DevicePool(batch.counts_ptr, batch.n_counts), device="cuda")
        tensors = [flux] + ([counts] if batch.n_counts > 0 else [])
        for t in tensors:
            dist.reduce(t, dst=0, op=dist.ReduceOp.SUM, group=group)
        torch.cuda.synchronize()
        if rank != 0:
            return None, None
        f = flux.cpu().numpy().reshape(p.n_bins, -1)
        c = counts.cpu().numpy().reshape(-1, p.n_bins) if batch.n_counts > 0 else None
        return f, c
    finally:
        batch.close()
