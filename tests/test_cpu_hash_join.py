"""The host no-partitioning join (the reference's CpuHashJoin) against the
oracle's hash tables and sums, the reference's own compiled CPU kernels, and
the reference's sequential CPU tests (sql-ops/src/join/no_partitioning_join.rs
test_cpu_seq: primary-key build, foreign-key probe, payloads 1..n, one build
key nulled for the selective perfect join)."""
import numpy as np
import pytest


def _schemes(fi):
    return {"perfect": fi.HashingScheme.Perfect,
            "linearprobing": fi.HashingScheme.LinearProbing}


@pytest.mark.parametrize("dtype", [np.int32, np.int64])
@pytest.mark.parametrize("scheme,selective", [("perfect", False), ("perfect", True),
                                              ("linearprobing", False)])
def test_cpu_seq_like_reference(fi, oracle, dtype, scheme, selective):
    """The reference's test_cpu_seq at a quarter of its 32 MiB columns."""
    rows = (8 << 20) // np.dtype(dtype).itemsize
    ht_len = 2 * rows
    inner_key = oracle.primary_keys(rows, 11, dtype)
    outer_key = oracle.uniform_foreign_keys(rows, rows, 12, dtype)
    inner_pay = np.arange(1, rows + 1, dtype=dtype)
    outer_pay = np.arange(1, rows + 1, dtype=dtype)
    exclude = 0
    if selective:
        inner_key[np.flatnonzero(inner_key == 1)[0]] = -1
        exclude = int(outer_pay[outer_key == 1].astype(np.uint64).sum())
    ht = fi.CpuHashTable(ht_len, dtype)
    hj = fi.CpuHashJoin(_schemes(fi)[scheme], ht, is_selective=selective)
    hj.build(inner_key, inner_pay)
    got = hj.probe_sum(outer_key, outer_pay)
    assert got == rows * (rows + 1) // 2 - exclude


@pytest.mark.parametrize("dtype", [np.int32, np.int64])
@pytest.mark.parametrize("entries", [2, 7, 1000, 4099])
def test_linear_probing_table_matches_oracle(fi, oracle, dtype, entries):
    """One thread: the table equals the oracle's slot by slot (same hash,
    same probe sequence, same insertion order) and so does the sum, with
    duplicate build keys and probe keys that miss."""
    n = min(entries, 3000)
    rng = np.random.default_rng(entries)
    bk = rng.integers(0, 2 * n + 1, n).astype(dtype)
    bp = rng.integers(-2**30, 2**30, n).astype(dtype)
    pk = rng.integers(0, 2 * n + 1, 5 * n).astype(dtype)
    pp = rng.integers(-2**30, 2**30, 5 * n).astype(dtype)
    exp_sum, exp_ht = oracle.ht_linearprobing_sum(bk, bp, pk, pp, entries)
    ht = fi.CpuHashTable(entries, dtype)
    hj = fi.CpuHashJoin(fi.HashingScheme.LinearProbing, ht)
    hj.build(bk, bp)
    assert np.array_equal(ht.mem, exp_ht)
    assert hj.probe_sum(pk, pp) == exp_sum


@pytest.mark.parametrize("dtype", [np.int32, np.int64])
@pytest.mark.parametrize("selective", [False, True])
def test_perfect_table_matches_oracle(fi, oracle, dtype, selective):
    n = 20_000
    bk = oracle.primary_keys(n, 3, dtype, base=0)
    if selective:
        bk[::97] = -1  # null keys (the oracle's plain build indexes with them)
    bp = oracle.uniform_u64_keys(n, 4).astype(dtype)
    pk = oracle.uniform_foreign_keys(3 * n, n, 5, dtype, base=0)
    pp = oracle.uniform_u64_keys(3 * n, 6).astype(dtype)
    entries = n + 1
    exp_sum, exp_ht = oracle.ht_perfect_sum(bk, bp, pk, pp, entries, selective)
    ht = fi.CpuHashTable(entries, dtype)
    hj = fi.CpuHashJoin(fi.HashingScheme.Perfect, ht, is_selective=selective)
    hj.build(bk, bp)
    assert np.array_equal(ht.mem[:, 0], exp_ht[:, 0])
    keyed = exp_ht[:, 0] != -1
    assert np.array_equal(ht.mem[keyed, 1], exp_ht[keyed, 1])
    assert hj.probe_sum(pk, pp) == exp_sum


@pytest.mark.parametrize("dtype", [np.int32, np.int64])
@pytest.mark.parametrize("scheme", ["perfect", "linearprobing"])
def test_matches_reference_kernels(fi, oracle, dtype, scheme):
    if not oracle.ref_available():
        pytest.skip("reference CPU kernels not built")
    n = 50_000
    bk = oracle.primary_keys(n, 21, dtype)
    bp = oracle.uniform_u64_keys(n, 22).astype(dtype)
    pk = oracle.uniform_foreign_keys(2 * n, n, 23, dtype)
    pp = oracle.uniform_u64_keys(2 * n, 24).astype(dtype)
    entries = 2 * n
    if scheme == "perfect":
        exp_sum, exp_ht = oracle.ref_ht_perfect_sum(bk, bp, pk, pp, entries)
    else:
        exp_sum, exp_ht = oracle.ref_ht_linearprobing_sum(bk, bp, pk, pp, entries)
    ht = fi.CpuHashTable(entries, dtype)
    hj = fi.CpuHashJoin(_schemes(fi)[scheme], ht)
    hj.build(bk, bp)
    assert np.array_equal(ht.mem, exp_ht)
    assert hj.probe_sum(pk, pp) == exp_sum


@pytest.mark.parametrize("dtype", [np.int32, np.int64])
@pytest.mark.parametrize("scheme", ["perfect", "linearprobing"])
def test_threads_share_one_table(fi, oracle, dtype, scheme):
    """Threads building disjoint slices into one table: linear-probing slots
    may differ from a sequential build, but the table holds the same
    entries and every sum is identical."""
    n = 200_000
    bk = oracle.primary_keys(n, 31, dtype)
    bk[:1000] = bk[1000:2000]  # duplicate keys race for slots
    bp = oracle.uniform_u64_keys(n, 32).astype(dtype)
    pk = oracle.zipf_foreign_keys(3 * n, n, 0.8, 33, 31, dtype)
    pp = oracle.uniform_u64_keys(3 * n, 34).astype(dtype)
    entries = 2 * n + 3
    if scheme == "perfect":
        bk[:1000] = np.arange(n + 1, n + 1001, dtype=dtype)  # keep keys unique
        exp_sum, _ = oracle.ht_perfect_sum(bk, bp, pk, pp, entries)
    else:
        exp_sum, exp_ht = oracle.ht_linearprobing_sum(bk, bp, pk, pp, entries)
    for threads in (2, 5, 8):
        got = fi.cpu_hash_join_sum(bk, bp, pk, pp, _schemes(fi)[scheme], entries,
                                   threads=threads)
        assert got == exp_sum
    if scheme == "linearprobing":
        ht = fi.CpuHashTable(entries, dtype)
        hj = fi.CpuHashJoin(fi.HashingScheme.LinearProbing, ht)
        import threading
        ts = [threading.Thread(target=hj.build, args=(bk[t::4], bp[t::4]))
              for t in range(4)]
        for t in ts:
            t.start()
        for t in ts:
            t.join()
        def rows(a):
            a = a[a[:, 0] != -1]
            return a[np.lexsort((a[:, 1], a[:, 0]))]
        assert np.array_equal(rows(ht.mem), rows(exp_ht))


def test_probe_accumulates_and_wraps(fi, oracle):
    """probe_sum adds into the caller's result, wrapping mod 2^64; negative
    payloads wrap as the reference's unsigned accumulation does."""
    n = 1000
    bk = np.arange(n, dtype=np.int64)
    ht = fi.CpuHashTable(n, np.int64)
    hj = fi.CpuHashJoin(fi.HashingScheme.Perfect, ht)
    hj.build(bk, bk)
    pay = np.full(n, -3, np.int64)
    got = hj.probe_sum(bk, pay, join_result=5)
    assert got == (5 - 3 * n) % (1 << 64)
    assert hj.probe_sum(bk[:0], pay[:0], join_result=got) == got
    big = np.full(4, 2**62, np.int64)
    assert hj.probe_sum(bk[:4], big, join_result=2**63) == (2**63 + 2**64) % (1 << 64)


def test_errors(fi):
    dt = np.int64
    k = np.arange(10, dtype=dt)
    with pytest.raises(fi.SqlOpsError):
        fi.CpuHashTable(10, dt, mem_len=5)
    ht = fi.CpuHashTable(8, dt)
    with pytest.raises(fi.SqlOpsError) as ex:
        fi.CpuHashJoin(fi.HashingScheme.BucketChaining, ht)
    assert ex.value.kind == "Unsupported"
    hj = fi.CpuHashJoin(fi.HashingScheme.LinearProbing, ht, is_selective=True)
    with pytest.raises(fi.SqlOpsError) as ex:
        hj.build(k[:4], k[:4])
    assert ex.value.kind == "Unsupported"
    hj = fi.CpuHashJoin(fi.HashingScheme.LinearProbing, ht)
    with pytest.raises(fi.SqlOpsError) as ex:
        hj.build(k, k)  # 10 tuples into 8 entries
    assert ex.value.kind == "InvalidArgument"
    with pytest.raises(fi.SqlOpsError):
        hj.build(k[:4], k[:3])
    with pytest.raises(fi.SqlOpsError):
        hj.probe_sum(k.astype(np.int32), k.astype(np.int32))
    # perfect hashing skips keys outside the table instead of writing there
    hp = fi.CpuHashJoin(fi.HashingScheme.Perfect, fi.CpuHashTable(4, dt, mem_len=8))
    hp.build(np.array([1, 6, -5, 3], dt), np.array([10, 20, 30, 40], dt))
    assert hp.probe_sum(np.array([1, 3, 6, -5], dt), np.ones(4, dt)) == 2
