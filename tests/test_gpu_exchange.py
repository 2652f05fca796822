"""The fused radix exchange (partition + send in one kernel) on one GPU.

Ranks are emulated as shards of one relation: every emulated sender runs
the histogram and the fused scatter into the receive columns of all
emulated receivers (local buffers standing in for peer pointers), one after
the other, with no kernel waiting on another.  The receive regions must
hold exactly the sender's tuples for that receiver (key and payload still
paired), the per-receiver joins must add up to the join of the whole
relations, and a capacity violation must be recorded, not written.  One
test runs two real processes on the one GPU, mapping each other's receive
columns through CUDA IPC, with gloo ordering the host steps.
"""
import datetime
import os
import socket

import numpy as np
import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

from _helpers import to_dev

pytestmark = pytest.mark.gpu


def dests_of(keys, shift, g):
    return ((keys.astype(np.int64).view(np.uint64) >> np.uint64(shift))
            & np.uint64((1 << g) - 1)).astype(np.int64)


def emulate_exchange(fi, shards, shift, g, dtype):
    """Runs the exchange of `shards` [(keys, pays) device tensors] and
    returns (receive columns per receiver, count matrix, bases per sender)."""
    import distributed as D
    W = 1 << g
    counts = [fi.exchange_histogram(k, shift, g) for k, _ in shards]
    mat = torch.stack(counts).cpu()
    recv = mat.sum(0).tolist()
    cols = [(torch.full((max(n, 1),), -7, dtype=dtype, device="cuda"),
             torch.full((max(n, 1),), -7, dtype=dtype, device="cuda")) for n in recv]
    status = torch.zeros(1, dtype=torch.int32, device="cuda")
    bases = []
    for s, (k, p) in enumerate(shards):
        base, r2 = D.region_bases(mat, s)
        assert r2 == recv
        bases.append(base)
        dests = [(cols[d][0].data_ptr(), cols[d][1].data_ptr(), base[d], recv[d])
                 for d in range(W)]
        cur = fi.exchange_scatter(k, p, shift, g, dests, status=status)
        assert cur.cpu().tolist() == mat[s].tolist()  # tuples sent per receiver
    torch.cuda.synchronize()
    assert int(status.item()) == 0
    return cols, mat, bases


@pytest.mark.parametrize("dtype,ndt", [(torch.int32, np.int32), (torch.int64, np.int64)])
@pytest.mark.parametrize("g", [0, 1, 2, 3])
def test_regions_hold_each_senders_tuples(fi, oracle, dtype, ndt, g):
    W, shift = 1 << g, 10
    sizes = [1_000_003, 0, 4096, 77_777, 12_288, 1, 300_001, 5][:max(W, 2)]
    shards = []
    for s, n in enumerate(sizes):
        k = oracle.uniform_u64_keys(n, 40 + s).astype(ndt)
        p = np.arange(n, dtype=ndt) * 7 + s
        shards.append((k, p))
    dev = [(to_dev(k), to_dev(p)) for k, p in shards]
    if W == 1:
        dev, shards = dev[:1], shards[:1]
    cols, mat, bases = emulate_exchange(fi, dev, shift, g, dtype)
    for s, (k, p) in enumerate(shards):
        d_of = dests_of(k, shift, g)
        assert mat[s].tolist() == np.bincount(d_of, minlength=W).tolist()
        for d in range(W):
            n = int(mat[s][d])
            got_k = cols[d][0][bases[s][d]:bases[s][d] + n].cpu().numpy()
            got_p = cols[d][1][bases[s][d]:bases[s][d] + n].cpu().numpy()
            sel = d_of == d
            exp = np.sort(np.stack([k[sel], p[sel]], 1).view(
                [("k", ndt), ("p", ndt)]).ravel(), order=["k", "p"])
            got = np.sort(np.stack([got_k, got_p], 1).view(
                [("k", ndt), ("p", ndt)]).ravel(), order=["k", "p"])
            assert np.array_equal(got, exp)


@pytest.mark.parametrize("dtype,ndt", [(torch.int32, np.int32), (torch.int64, np.int64)])
def test_exchange_then_local_joins_equal_whole_join(fi, oracle, dtype, ndt):
    """Four emulated ranks, 4+4 local bits, exchange bits [8, 10): the sum
    of the four local joins equals the single join of R and S."""
    g, bits = 2, (4, 4)
    n = 1 << 20
    r = oracle.primary_keys(n, 61, ndt)
    rp = oracle.uniform_foreign_keys(n, 1 << 30, 62, ndt)
    s = oracle.uniform_foreign_keys(3 * n, 2 * n, 63, ndt)
    sp = oracle.uniform_foreign_keys(3 * n, 1 << 30, 64, ndt)
    W = 1 << g
    shardR = [(to_dev(r[i::W]), to_dev(rp[i::W])) for i in range(W)]
    shardS = [(to_dev(s[i::W]), to_dev(sp[i::W])) for i in range(W)]
    colsR, matR, _ = emulate_exchange(fi, shardR, sum(bits), g, dtype)
    colsS, matS, _ = emulate_exchange(fi, shardS, sum(bits), g, dtype)
    tot_s, tot_c = 0, 0
    for d in range(W):
        nr, ns = int(matR[:, d].sum()), int(matS[:, d].sum())
        if nr == 0 or ns == 0:
            continue
        e = fi.RadixJoinEngine(nr, ns, dtype, fi.RadixBits(*bits),
                               fi.HashingScheme.BucketChaining)
        sm, c = e.run(colsR[d][0][:nr], colsR[d][1][:nr], colsS[d][0][:ns],
                      colsS[d][1][:ns])
        e.status()
        tot_s += sm
        tot_c += c
    whole = fi.RadixJoinEngine(n, 3 * n, dtype, fi.RadixBits(*bits),
                               fi.HashingScheme.BucketChaining)
    exp = whole.run(to_dev(r), to_dev(rp), to_dev(s), to_dev(sp))
    mask = (1 << 64) - 1
    assert ((tot_s & mask), tot_c) == ((exp[0] & mask), exp[1])


def test_capacity_is_checked_per_store(fi, oracle):
    """A receiver whose cap is one slot short: the kernel records
    FI_ERR_CAPACITY and writes nothing past cap (the guard stays intact)."""
    n, g, shift = 100_000, 1, 3
    k = to_dev(oracle.uniform_u64_keys(n, 71).astype(np.int64))
    p = to_dev(np.arange(n, dtype=np.int64))
    cnt = fi.exchange_histogram(k, shift, g).cpu().tolist()
    guard = 1024
    cols = [(torch.full((c + guard,), -5, dtype=torch.int64, device="cuda"),
             torch.full((c + guard,), -5, dtype=torch.int64, device="cuda")) for c in cnt]
    caps = [cnt[0] - 1, cnt[1]]
    status = torch.zeros(1, dtype=torch.int32, device="cuda")
    fi.exchange_scatter(k, p, shift, g, [(c[0].data_ptr(), c[1].data_ptr(), 0, cap)
                                         for c, cap in zip(cols, caps)], status=status)
    torch.cuda.synchronize()
    assert int(status.item()) == -7
    assert bool((cols[0][0][caps[0]:] == -5).all()) and bool((cols[0][1][caps[0]:] == -5).all())
    assert bool((cols[1][0][cnt[1]:] == -5).all())
    assert int((cols[1][0][:cnt[1]] != -5).sum()) == cnt[1]


def test_exchange_validation(fi):
    k = torch.zeros(16, dtype=torch.int64, device="cuda")
    with pytest.raises(fi.SqlOpsError) as ex:
        fi.exchange_histogram(k, 0, 7)  # 128 ranks
    assert ex.value.kind == "InvalidArgument"
    k32 = torch.zeros(16, dtype=torch.int32, device="cuda")
    with pytest.raises(fi.SqlOpsError):
        fi.exchange_histogram(k32, 31, 2)  # bits [31, 33) of a 32-bit key
    with pytest.raises(fi.SqlOpsError):
        fi.exchange_scatter(k, k, 0, 1, [(0, 0, 0, 16), (0, 0, 0, 0)])  # null columns
    # empty input: nothing sent, cursors zero
    e = k[:0]
    cur = fi.exchange_scatter(e, e, 0, 1, [(k.data_ptr(), k.data_ptr(), 0, 16)] * 2)
    assert cur.cpu().tolist() == [0, 0]


def free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def ipc_worker(rank, world, port, out):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    torch.cuda.set_device(0)
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=60))
    try:
        import distributed as D
        import fi_sqlops as fi
        import oracle as O
        n = 1 << 18
        r = O.primary_keys(n, 81, np.int64)
        s = O.uniform_foreign_keys(2 * n, n, 82, np.int64)
        rk = to_dev(r[rank::world])
        sk = to_dev(s[rank::world])
        res = D.exchange_join(rk, rk, sk, sk, bits=(5, 5),
                              scheme=fi.HashingScheme.BucketChaining, exchange="peer")
        out.put((rank, res))
    except BaseException:
        import traceback
        out.put((rank, "error: " + traceback.format_exc()))
        raise
    finally:
        dist.destroy_process_group()


def test_ipc_handle_offsets(fi):
    """The handle names the whole allocation; the offset locates the tensor
    in it (a tensor of a caching-allocator block need not start it)."""
    t = torch.empty(1 << 20, dtype=torch.int64, device="cuda")
    h0, o0 = fi.ipc_handle(t)
    h1, o1 = fi.ipc_handle(t[1000:])
    assert h0 == h1 and o1 - o0 == 8000 and len(h0) == fi.IPC_HANDLE_BYTES


def test_peer_exchange_two_processes_one_gpu(oracle):
    """Two processes on one GPU: each maps the other's receive columns by
    CUDA IPC, the fused kernel stores into them, gloo orders the steps."""
    ctx = mp.get_context("spawn")
    out = ctx.Queue()
    try:
        mp.spawn(ipc_worker, args=(2, free_port(), out), nprocs=2, join=True)
    finally:
        msgs = []
        while not out.empty():
            msgs.append(out.get())
        for m in msgs:
            print("rank %d: %s" % m)
    got = sorted(msgs)
    assert len(got) == 2, got
    n = 1 << 18
    s = oracle.uniform_foreign_keys(2 * n, n, 82, np.int64)
    exp = (int(s.sum()), 2 * n)  # every S key matches; payload = key
    assert got[0][1] == got[1][1] == exp
