"""Batched small joins: many joins in one graph replay.

Every job of a batch must give the same {sum, count} as the same join run
alone through the engine and as the CPU radix join, whatever else shares
the batch (sizes, skew, bits, empty relations).
"""
import numpy as np
import pytest
import torch

from _helpers import to_dev

pytestmark = pytest.mark.gpu

MASK = (1 << 64) - 1


def make_job(oracle, rn, k, seed, ndt, miss=False):
    """R: permutation of 1..rn; S: k*rn foreign keys (uniform), drawn from
    twice R's key range when miss=True so about half the probes miss;
    payloads are independent draws."""
    sn = k * rn
    rk = oracle.primary_keys(rn, seed, ndt, base=1)
    rp = oracle.uniform_foreign_keys(rn, 1 << 30, seed + 1, ndt)
    sk = oracle.uniform_foreign_keys(sn, max(1, rn) * (2 if miss else 1), seed + 2,
                                     ndt, base=1)
    sp = oracle.uniform_foreign_keys(sn, 1 << 30, seed + 3, ndt)
    return rk, rp, sk, sp


def cpu_join(oracle, rk, rp, sk, sp):
    s, c, _, _ = oracle.cpu_radix_join(rk.astype(np.int64), rp.astype(np.int64),
                                       sk.astype(np.int64), sp.astype(np.int64),
                                       4, 4, 4, use_reference=False)
    return s & MASK, c


@pytest.mark.parametrize("ndt,tdt", [(np.int32, torch.int32), (np.int64, torch.int64)])
def test_batch_matches_cpu_join(fi, oracle, ndt, tdt):
    rng = np.random.default_rng(7)
    jobs, exp = [], []
    for i in range(40):
        rn = int(np.exp(rng.uniform(np.log(1000), np.log(200_000))))
        k = int(rng.choice([1, 2, 4, 8, 16]))
        host = make_job(oracle, rn, k, 100 + 10 * i, ndt, miss=(i % 3 == 0))
        exp.append(cpu_join(oracle, *host))
        jobs.append(tuple(to_dev(a) for a in host))
    b = fi.JoinBatch(tdt, max_jobs=64, max_tuples=1 << 25)
    got = b.run(jobs)
    assert [(g[0] & MASK, g[1]) for g in got] == exp


def test_batch_result_same_alone_and_in_mix(fi, oracle):
    """Each job alone in a batch, in a mix with others, and through the
    engine: three identical results."""
    rng = np.random.default_rng(11)
    jobs = []
    for i in range(24):
        rn = int(np.exp(rng.uniform(np.log(64 << 10), np.log(1 << 20))))
        k = int(rng.choice([1, 2, 4]))
        host = make_job(oracle, rn, k, 500 + 10 * i, np.int64, miss=(i % 2 == 0))
        jobs.append(tuple(to_dev(a) for a in host))
    b = fi.JoinBatch(torch.int64, max_jobs=32, max_tuples=1 << 26)
    mixed = b.run(jobs)
    e = fi.RadixJoinEngine(1 << 20, 4 << 20, torch.int64, fi.RadixBits(6, 6),
                           fi.HashingScheme.BucketChaining)
    for j, m in zip(jobs, mixed):
        alone = b.run([j])[0]
        assert alone == m == e.run(*j)


def test_batch_skew_bits_and_empty_jobs(fi):
    n = 1 << 18
    rk = torch.empty(n, dtype=torch.int64, device="cuda")
    sk = torch.empty(4 * n, dtype=torch.int64, device="cuda")
    fi.gen_primary_keys(rk, 3)
    fi.gen_zipf_foreign_keys(sk, n, 1.0, 4, 3)
    exp = (int(sk.sum().item()), 4 * n)
    e0 = torch.empty(0, dtype=torch.int64, device="cuda")
    b = fi.JoinBatch(torch.int64, max_jobs=16, max_tuples=1 << 24)
    jobs = [(rk, rk, sk, sk, 0), (rk, rk, sk, sk, 5), (rk, rk, sk, sk, 12),
            (rk, rk, sk, sk), (e0, e0, sk, sk), (rk, rk, e0, e0), (e0, e0, e0, e0)]
    got = b.run(jobs)
    assert got[:4] == [exp] * 4
    assert got[4:] == [(0, 0)] * 3


def test_batch_capacity_and_bits_errors(fi):
    b = fi.JoinBatch(torch.int64, max_jobs=2, max_tuples=1000)
    k = torch.arange(1, 601, dtype=torch.int64, device="cuda")
    with pytest.raises(fi.SqlOpsError) as ex:
        b.run([(k, k, k, k)])  # 1200 tuples
    assert ex.value.kind == "Capacity"
    with pytest.raises(fi.SqlOpsError) as ex:
        b.run([(k[:10], k[:10], k[:10], k[:10])] * 3)  # 3 jobs
    assert ex.value.kind == "Capacity"
    with pytest.raises(fi.SqlOpsError) as ex:
        b.run([(k[:10], k[:10], k[:10], k[:10], 13)])
    assert ex.value.kind == "Unsupported"
