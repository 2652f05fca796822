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
                              group_by=cpu_group_by, local_join=cpu_join,
                              exchange="nccl")
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


def peer_protocol_worker(rank, world, port, out):
    """PeerExchange's host protocol on gloo ranks, with the two kernels and
    CUDA IPC replaced by host fakes: the fake scatter records what it was
    given and writes this rank's own share into its own columns."""
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=60))
    try:
        import distributed as D
        import fi_sqlops as fi
        g = D.exchange_bits(world)
        state = {"calls": [], "fail_rank": None, "ex": None}

        def hist(keys, shift, gg, counts=None, stream=None):
            return torch.bincount(D.destinations(keys, shift, gg), minlength=1 << gg)

        def scatter(keys, pays, shift, gg, dests, cursors=None, status=None, stream=None):
            state["calls"].append([(int(k), int(p), int(b), int(c)) for k, p, b, c in dests])
            d = D.destinations(keys, shift, gg)
            ex, sel = state["ex"], d == rank
            b = int(dests[rank][2])
            ex.keys[b:b + int(sel.sum())] = keys[sel]
            ex.pays[b:b + int(sel.sum())] = pays[sel]
            if state["fail_rank"] == rank:
                status.fill_(-7)
            return cursors

        fi.exchange_histogram, fi.exchange_scatter = hist, scatter
        fi.ipc_handle = lambda t: (b"h%d" % rank, 16 * rank)
        fi.ipc_open = lambda h: 1 << (20 + int(h[1:]))
        fi.ipc_close = lambda ptr: None
        rng = np.random.default_rng(rank)
        keys = torch.from_numpy(rng.integers(0, 1 << 16, 5000 + 1000 * rank))
        cap = 8000
        ex = D.PeerExchange(cap, torch.int64, device="cpu")
        state["ex"] = ex
        got_k, got_p = ex.shuffle(keys, keys * 3, 10)
        b_self = state["calls"][0][rank][2]
        n_self = int((D.destinations(keys, 10, g) == rank).sum())
        own_k, own_p = got_k[b_self:b_self + n_self], got_p[b_self:b_self + n_self]
        res = {"calls": state["calls"][0], "n": len(got_k),
               "mine_ok": bool((D.destinations(own_k, 10, g) == rank).all())
               and bool(torch.equal(own_p, own_k * 3))}
        # a sender's recorded error fails both ranks alike
        state["fail_rank"] = 1
        try:
            ex.shuffle(keys, keys, 10)
            res["status_raised"] = False
        except fi.SqlOpsError as e:
            res["status_raised"] = e.code == -7
        # too little room anywhere: every rank raises before sending
        small = D.PeerExchange(100, torch.int64, device="cpu")
        try:
            small.shuffle(keys, keys, 10)
            res["cap_raised"] = False
        except fi.SqlOpsError as e:
            res["cap_raised"] = e.code == -7
        dist.barrier()  # the group still works after both errors
        small.close()
        ex.close()
        out.put((rank, res))
    finally:
        dist.destroy_process_group()


def test_peer_exchange_protocol_two_ranks():
    import distributed as D
    ctx = mp.get_context("spawn")
    out = ctx.Queue()
    mp.spawn(peer_protocol_worker, args=(2, free_port(), out), nprocs=2, join=True)
    got = dict(out.get(timeout=60) for _ in range(2))
    # rebuild the count matrix the ranks shared
    mats = []
    for r in range(2):
        keys = torch.from_numpy(np.random.default_rng(r).integers(0, 1 << 16, 5000 + 1000 * r))
        mats.append(torch.bincount(D.destinations(keys, 10, 1), minlength=2).tolist())
    for r in range(2):
        res = got[r]
        base, recv = D.region_bases(mats, r)
        assert res["n"] == recv[r] and res["mine_ok"]
        assert res["status_raised"] and res["cap_raised"]
        for d, (kp, pp, b, c) in enumerate(res["calls"]):
            assert (b, c) == (base[d], 8000)
            if d != r:  # the peer's columns: mapped base + its offset, payloads after keys
                assert kp == (1 << (20 + d)) + 16 * d and pp == kp + 8000 * 8


def sharded_worker(rank, world, port, n, out):
    """The sharded bench workload's host logic on gloo ranks: shards made by
    the bench's rule (distributed.shard_primary_keys for R, a seed per rank
    for S's uniform foreign keys over all ranks' keys, payload = key), the
    exchange join, and its closed form."""
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=60))
    try:
        import distributed as D
        import oracle as O
        rk = torch.from_numpy(O.primary_keys(n, 7, np.int64))
        D.shard_primary_keys(rk, world, rank)
        sk = torch.from_numpy(O.uniform_foreign_keys(n, world * n, 8 + rank, np.int64))
        part = torch.tensor([int(sk.sum())], dtype=torch.int64)
        dist.all_reduce(part)
        res = D.exchange_join(rk, rk.clone(), sk, sk.clone(), bits=(3, 3), scheme=2,
                              group_by=cpu_group_by, local_join=cpu_join,
                              exchange="nccl")
        out.put((rank, res, int(part.item()), sorted(rk.tolist())))
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("world", [2, 4])
def test_sharded_bench_rule(world):
    """Every S key is a foreign key of the ranks' R shards, which together
    are a permutation of 1..world*n: count = world * n, sum = all S keys."""
    n = 1 << 12
    ctx = mp.get_context("spawn")
    out = ctx.Queue()
    mp.spawn(sharded_worker, args=(world, free_port(), n, out), nprocs=world, join=True)
    got = sorted(out.get(timeout=60) for _ in range(world))
    keys = sorted(k for g in got for k in g[3])
    assert keys == list(range(1, world * n + 1))
    for rank, (s, c), total, _ in got:
        assert c == world * n
        assert s == (total + (1 << 63)) % (1 << 64) - (1 << 63)
