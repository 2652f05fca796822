"""The multi-GPU exchange join's host logic on CPU: two gloo ranks.

Each rank holds a strided shard of R and of S; the exchange moves every
tuple to the rank named by its key bits above the local join's bits, each
rank joins what it received, and an all-reduce adds the results.  Here the
grouping by destination and the local join are CPU stand-ins (a stable
sort, the CPU radix join of the oracle); on GPUs the same code path calls
the library's partitioner and engine.  The all-reduced result must equal
the single-process join of the whole relations, and every tuple must land
on the rank its key names.
"""
import datetime
import os
import socket

import numpy as np
import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp


def free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def cpu_group_by(keys, pays, shift, g):
    import distributed as D
    d = D.destinations(keys, shift, g)
    order = torch.argsort(d, stable=True)
    tuples = torch.stack([keys, pays], 1)[order].contiguous()
    return tuples, torch.bincount(d, minlength=1 << g)


def cpu_join(rk, rp, sk, sp, bits, scheme):
    import oracle as O
    if rk.numel() == 0 or sk.numel() == 0:
        return 0, 0
    s, c, _, _ = O.cpu_radix_join(rk.numpy().astype(np.int64), rp.numpy().astype(np.int64),
                                  sk.numpy().astype(np.int64), sp.numpy().astype(np.int64),
                                  bits[0], bits[1], 2, use_reference=False)
    return (s + (1 << 63)) % (1 << 64) - (1 << 63), c  # as int64


def relations(n, dt):
    import oracle as O
    r = O.primary_keys(n, 21, dt)
    rp = O.uniform_foreign_keys(n, 1 << 30, 22, dt)
    s = O.uniform_foreign_keys(3 * n, 2 * n, 23, dt)  # about half the probes miss
    sp = O.uniform_foreign_keys(3 * n, 1 << 30, 24, dt)
    return r, rp, s, sp


def worker(rank, world, port, dt, out):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=60))
    try:
        import distributed as D
        r, rp, s, sp = (torch.from_numpy(a[rank::world].copy())
                        for a in relations(1 << 14, dt))
        bits = (4, 4)
        # every tuple lands on the rank its exchange bits name
        g = D.exchange_bits(world)
        rk2, _ = D.shuffle(r, rp, sum(bits), group_by=cpu_group_by)
        assert bool((D.destinations(rk2, sum(bits), g) == rank).all())
        res = D.exchange_join(r, rp, s, sp, bits=bits, scheme=2,
                              group_by=cpu_group_by, local_join=cpu_join)
        out.put((rank, res, rk2.numel()))
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("dt", [np.int32, np.int64])
def test_exchange_join_two_ranks(oracle, dt):
    ctx = mp.get_context("spawn")
    out = ctx.Queue()
    world = 2
    mp.spawn(worker, args=(world, free_port(), dt, out), nprocs=world, join=True)
    got = sorted(out.get(timeout=60) for _ in range(world))
    r, rp, s, sp = relations(1 << 14, dt)
    exp_s, exp_c, _, _ = oracle.cpu_radix_join(r.astype(np.int64), rp.astype(np.int64),
                                               s.astype(np.int64), sp.astype(np.int64),
                                               4, 4, 2, use_reference=False)
    exp = ((exp_s + (1 << 63)) % (1 << 64) - (1 << 63), exp_c)
    assert got[0][1] == got[1][1] == exp
    assert got[0][2] + got[1][2] == len(r)  # the R tuples, each on one rank


def test_exchange_needs_power_of_two():
    import distributed as D
    with pytest.raises(ValueError):
        D.exchange_bits(3)
    assert D.exchange_bits(8) == 3


def plan_worker(rank, world, port, out):
    """The peer exchange's plan on gloo ranks: all-gathered counts and each
    sender's region in every receiver's columns."""
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=60))
    try:
        import distributed as D
        g = D.exchange_bits(world)
        keys = torch.from_numpy(np.random.default_rng(rank).integers(
            0, 1 << 20, 1000 + 337 * rank))
        counts = torch.bincount(D.destinations(keys, 12, g), minlength=world)
        mat = D.all_gather_counts(counts)
        base, recv = D.region_bases(mat, rank)
        out.put((rank, mat.tolist(), base, recv, counts.tolist()))
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("world", [2, 4])
def test_peer_exchange_plan(world):
    ctx = mp.get_context("spawn")
    out = ctx.Queue()
    mp.spawn(plan_worker, args=(world, free_port(), out), nprocs=world, join=True)
    got = sorted(out.get(timeout=60) for _ in range(world))
    mats = [g[1] for g in got]
    assert all(m == mats[0] for m in mats)  # every rank sees one matrix
    for rank, mat, base, recv, counts in got:
        assert mat[rank] == counts  # row s = sender s's counts
        assert recv == [sum(mat[s][d] for s in range(world)) for d in range(world)]
    for d in range(world):  # the senders' regions tile each receiver's columns
        spans = sorted((got[s][2][d], got[s][2][d] + mats[0][s][d]) for s in range(world))
        assert spans[0][0] == 0 and spans[-1][1] == got[0][3][d]
        assert all(a[1] == b[0] for a, b in zip(spans, spans[1:]))


def test_region_bases_small():
    import distributed as D
    mat = [[3, 1], [2, 5]]
    assert D.region_bases(mat, 0) == ([0, 0], [5, 6])
    assert D.region_bases(mat, 1) == ([3, 1], [5, 6])
