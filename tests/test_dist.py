"""Multi-rank path on CPU: two gloo ranks each integrate their shard of a
profile set (the FP64 oracle stands in for the per-GPU engine, which needs a
GPU) and gather to rank 0; the gathered result equals one process doing all
profiles, and the max-over-ranks timing helper agrees across ranks."""
import os
import socket

import numpy as np
import torch.multiprocessing as mp

from gpu_ppm_b200 import dist as pdist
from gpu_ppm_b200 import synth


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _worker(rank, world, port, out_q):
    import torch.distributed as dist

    import oracle

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    lens = synth.small_lensing()
    E = synth.energy_grid(12, 0.5, 6.0)
    plist, _ = synth.draw_prior(6, seed=4, lens_u=(0.3, 0.5), n_side=8, n_bins=8)
    for p in plist:
        p.atmosphere = 1
        p.precision = 1
        for s in range(p.n_spots):
            p.spots[s].kT_keV = 0.3
    costs = [p.spots[0].angrad1 for p in plist]
    idx = pdist.shard_indices(len(plist), rank, world, costs)
    ora = oracle.Oracle(lens)
    local = [ora.profile(plist[i], E)[0] for i in idx]
    full = pdist.gather_to_rank0(local, idx, len(plist))
    t = pdist.max_over_ranks(1.0 + rank)
    if rank == 0:
        ref = [ora.profile(p, E)[0] for p in plist]
        ok = all(np.array_equal(a, b) for a, b in zip(full, ref))
        out_q.put((ok, t, sorted(idx)))
    else:
        out_q.put((True, t, sorted(idx)))
    dist.barrier()
    dist.destroy_process_group()


def test_two_rank_shard_and_gather():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = [q.get(timeout=300) for _ in procs]
    for p in procs:
        p.join(timeout=120)
        assert p.exitcode == 0
    assert all(ok for ok, _, _ in res)
    assert all(t == 2.0 for _, t, _ in res)
    shards = sorted(i for _, _, idx in res for i in idx)
    assert shards == list(range(6))


def test_shard_indices_cover_and_balance():
    for n, w in ((10, 3), (1, 4), (7, 7)):
        got = sorted(i for r in range(w) for i in pdist.shard_indices(n, r, w))
        assert got == list(range(n))
    costs = [10, 1, 1, 1, 1, 1, 1, 1, 1, 1]
    loads = [sum(costs[i] for i in pdist.shard_indices(10, r, 2, costs)) for r in range(2)]
    assert max(loads) == 10


def _ring_worker(rank, world, port, out_q):
    import torch.distributed as dist

    import oracle

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    lens = synth.small_lensing()
    E = synth.energy_grid(10, 0.5, 6.0)
    p = synth.config1_params(0)
    p.n_side = 16
    p.n_bins = 8
    windows = pdist.ring_partition(pdist.ring_costs(p), world)
    ora = oracle.Oracle(lens)
    part, _ = ora.profile_rings(p, E, *windows[rank])
    total = pdist.reduce_sum_to_rank0([part])
    if rank == 0:
        full, _ = ora.profile(p, E)
        err = float(np.max(np.abs(total[0] - full)) / np.max(np.abs(full)))
        out_q.put((err, windows))
    else:
        out_q.put((0.0, windows))
    dist.barrier()
    dist.destroy_process_group()


def test_two_rank_ring_split_reduces_to_full_profile():
    """One profile split by HEALPix ring windows over two gloo ranks (the FP64
    oracle stands in for each rank's engine): the sum-reduce to rank 0 equals
    the whole profile."""
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_ring_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = [q.get(timeout=300) for _ in procs]
    for p in procs:
        p.join(timeout=120)
        assert p.exitcode == 0
    assert max(e for e, _ in res) < 1e-12
    w = res[0][1]
    assert w[0][0] == 0 and w[0][1] == w[1][0] and w[1][1] == 4 * 16


def test_ring_partition_balances_costs():
    costs = np.array([0, 5, 5, 5, 5, 0, 0, 10, 10, 0], dtype=float)
    for world in (1, 2, 3, 4):
        win = pdist.ring_partition(costs, world)
        assert win[0][0] == 0 and win[-1][1] == len(costs)
        assert all(a[1] == b[0] for a, b in zip(win, win[1:]))
        loads = [costs[b:e].sum() for b, e in win]
        assert sum(loads) == costs.sum()
        assert max(loads) <= costs.sum() / world + costs.max()
    p = synth.config2_params(0, -1, n_side=32, n_bins=8)
    import oracle

    assert pdist.ring_costs(p).sum() == sum(oracle.count_active(p.spots[k], 32) for k in range(p.n_spots))
