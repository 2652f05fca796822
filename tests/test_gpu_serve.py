"""The join server: continuous batching, admission under a memory budget,
and results that are the same alone and in the mix.

Requests of uneven sizes (batched small joins and engine-run large joins,
int32 and int64, uniform and Zipf-skewed) are submitted together; each
result must equal the same join run alone through the engine, and, for the
synthetic source, its closed form (every probe key is a foreign key, so the
count is |S| and the sum is the sum of the probe keys, payload = key).
"""
import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu

MASK = (1 << 64) - 1


def synthetic_expected(fi, tb, rn, sn, seed, zipf):
    """Closed form of a synthetic request, from the same generators."""
    dt = torch.int64 if tb == 16 else torch.int32
    sk = torch.empty(sn, dtype=dt, device="cuda")
    if zipf > 0:
        fi.gen_zipf_foreign_keys(sk, rn, zipf, seed + 1, seed)
    else:
        fi.gen_uniform_foreign_keys(sk, rn, seed + 1)
    return int(sk.to(torch.int64).sum().item()) & MASK, sn


def test_server_mixed_stream_equals_alone(fi):
    rng = np.random.default_rng(5)
    srv = fi.JoinServer(hbm_budget_bytes=60 << 30, workers=2, max_build=1 << 24,
                        probe_slice=1 << 24, batch_tuples=1 << 24)
    reqs = []
    for i in range(60):
        rn = int(np.exp(rng.uniform(np.log(64 << 10), np.log(8 << 20))))
        k = int(rng.choice([1, 2, 4, 8]))
        tb = int(rng.choice([8, 16]))
        zipf = float(rng.choice([0.0, 1.0]))
        reqs.append((tb, rn, k * rn, 1000 + i, zipf))
    tickets = [srv.submit(tuple_bytes=tb, source=fi.JoinSource.Synthetic,
                          build_len=rn, probe_len=sn, seed=seed, zipf_s=z)
               for tb, rn, sn, seed, z in reqs]
    got = [srv.wait(t) for t in tickets]
    st = srv.stats()
    srv.close()
    assert all(g["status"] == 0 for g in got)
    assert st["batches"] > 0 and st["engine_runs"] > 0
    assert st["completed"] == len(reqs)
    assert any(g["batched"] for g in got) and not all(g["batched"] for g in got)
    for (tb, rn, sn, seed, z), g in zip(reqs, got):
        assert (g["sum"] & MASK, g["count"]) == synthetic_expected(fi, tb, rn, sn, seed, z)


def test_server_automatic_workers(fi):
    """workers = 0 picks two engines when they take at most half the budget
    and one otherwise; either way the results equal the closed form."""
    shape = dict(max_build=1 << 24, probe_slice=1 << 24, batch_tuples=1 << 20)
    one = fi.JoinServer(hbm_budget_bytes=60 << 30, workers=1, **shape)
    fixed1 = one.stats()["fixed_bytes"]
    one.close()
    two = fi.JoinServer(hbm_budget_bytes=60 << 30, workers=0, **shape)
    st = two.stats()
    assert st["workers"] == 2
    engine = st["fixed_bytes"] - fixed1  # one engine's workspace
    reqs = [(16, 3 << 20, 6 << 20, 77, 0.0), (8, 5 << 20, 5 << 20, 78, 1.0)]
    got = [two.wait(two.submit(tuple_bytes=tb, source=fi.JoinSource.Synthetic,
                               build_len=rn, probe_len=sn, seed=seed, zipf_s=z))
           for tb, rn, sn, seed, z in reqs]
    two.close()
    for (tb, rn, sn, seed, z), g in zip(reqs, got):
        assert g["status"] == 0
        assert (g["sum"] & MASK, g["count"]) == synthetic_expected(fi, tb, rn, sn, seed, z)
    # a budget that holds one engine, the batch arenas and a 1 GB slab
    budget = fixed1 + (1 << 30)
    tight = fi.JoinServer(hbm_budget_bytes=budget, workers=0, **shape)
    assert tight.stats()["workers"] == (1 if 2 * engine > budget // 2 else 2)
    g = tight.wait(tight.submit(tuple_bytes=16, source=fi.JoinSource.Synthetic,
                                build_len=1 << 20, probe_len=1 << 21, seed=79))
    tight.close()
    assert g["status"] == 0
    assert (g["sum"] & MASK, g["count"]) == synthetic_expected(fi, 16, 1 << 20, 1 << 21,
                                                              79, 0.0)


def test_server_device_source_alone_vs_mix(fi, oracle):
    """Device-resident relations (with misses): the response of a request
    submitted alone equals its response inside a mix, and the engine's."""
    rng = np.random.default_rng(9)
    cols = []
    for i in range(12):
        rn = int(np.exp(rng.uniform(np.log(10_000), np.log(6 << 20))))
        sn = 2 * rn
        rk = oracle.primary_keys(rn, 40 + i, np.int64)
        sk = oracle.uniform_foreign_keys(sn, 2 * rn, 80 + i, np.int64)  # half miss
        rp = oracle.uniform_foreign_keys(rn, 1 << 40, 120 + i, np.int64)
        sp = oracle.uniform_foreign_keys(sn, 1 << 40, 160 + i, np.int64)
        cols.append(tuple(torch.from_numpy(a).cuda() for a in (rk, rp, sk, sp)))
    torch.cuda.synchronize()
    srv = fi.JoinServer(hbm_budget_bytes=40 << 30, max_build=1 << 23,
                        probe_slice=1 << 22)
    mixed = [srv.wait(t) for t in
             [srv.submit(source=fi.JoinSource.Device, columns=c) for c in cols]]
    alone = [srv.wait(srv.submit(source=fi.JoinSource.Device, columns=c)) for c in cols]
    srv.close()
    e = fi.RadixJoinEngine(1 << 23, 1 << 24, torch.int64, fi.RadixBits(7, 7),
                           fi.HashingScheme.BucketChaining)
    for c, m, a in zip(cols, mixed, alone):
        ref = e.run(*c)
        assert m["status"] == a["status"] == 0
        assert (m["sum"], m["count"]) == (a["sum"], a["count"]) == ref


def test_server_admission_budget(fi):
    """A request larger than the free budget fails with Capacity; requests
    that fit only one at a time are admitted one after another."""
    srv = fi.JoinServer(hbm_budget_bytes=0, max_build=1 << 22, probe_slice=1 << 22)
    fixed = srv.stats()["fixed_bytes"]
    srv.close()
    budget = fixed + (96 << 20)  # room for one 8M-tuple int64 request at a time
    srv = fi.JoinServer(hbm_budget_bytes=budget, max_build=1 << 22,
                        probe_slice=1 << 22)
    too_big = srv.submit(tuple_bytes=16, build_len=1 << 22, probe_len=1 << 24, seed=1)
    fits = [srv.submit(tuple_bytes=16, build_len=1 << 22, probe_len=1 << 22, seed=s)
            for s in (2, 3, 4)]
    r = srv.wait(too_big)
    assert r["status"] == -7  # FI_ERR_CAPACITY
    for t, s in zip(fits, (2, 3, 4)):
        g = srv.wait(t)
        assert g["status"] == 0
        assert (g["sum"] & MASK, g["count"]) == synthetic_expected(
            fi, 16, 1 << 22, 1 << 22, s, 0.0)
    st = srv.stats()
    assert st["peak_reserved_bytes"] <= 96 << 20
    assert st["reserved_bytes"] == 0
    srv.close()
