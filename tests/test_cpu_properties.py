"""The library's host operators on random inputs (hypothesis: sizes, chunk
counts, radix bits, full-range, negative and duplicate-heavy keys, sizes
below the chunk count): the CPU radix partitioner (the hybrid join's first
pass) equals the reference's compiled CPU partitioner slot by slot (NC) and
the oracle slot by slot (SWWC); the CPU no-partitioning join on one thread
builds the oracle's table slot by slot and returns the reference's sum."""
import numpy as np
import pytest

hypothesis = pytest.importorskip("hypothesis")
from hypothesis import given, settings, strategies as st  # noqa: E402

DTYPES = [np.int32, np.int64]
KINDS = ["full", "negative", "few"]


def draw_keys(rng, n, dt, kind):
    info = np.iinfo(dt)
    if kind == "full":
        return rng.integers(info.min, info.max, n, dtype=dt, endpoint=True)
    if kind == "negative":
        return rng.integers(-(1 << 20), 0, n).astype(dt)
    return rng.integers(0, 7, n).astype(dt)


@settings(max_examples=40, deadline=None)
@given(n=st.integers(1, 6000), chunks=st.integers(1, 8), bits=st.integers(0, 12),
       dt=st.sampled_from(DTYPES), kind=st.sampled_from(KINDS),
       algo=st.sampled_from(["NC", "SWWC"]), seed=st.integers(0, 2**32 - 1))
def test_cpu_partition_random(fi, oracle, n, chunks, bits, dt, kind, algo, seed):
    rng = np.random.default_rng(seed)
    keys = draw_keys(rng, n, dt, kind)
    pays = rng.integers(np.iinfo(dt).min, np.iinfo(dt).max, n, dtype=dt, endpoint=True)
    rel, off = fi.cpu_radix_partition(keys, pays, bits, chunks,
                                      getattr(fi.CpuRadixPartitionAlgorithm, algo))
    exp_off = oracle.chunked_prefix_sum(keys, chunks, bits)
    np.testing.assert_array_equal(off, exp_off)
    exp = oracle.chunked_radix_partition(keys, pays, exp_off, chunks, bits, 0, len(rel))
    np.testing.assert_array_equal(rel, exp)
    if algo == "NC" and oracle.ref_available():
        np.testing.assert_array_equal(off, oracle.ref_chunked_prefix_sum(keys, chunks, bits))
        np.testing.assert_array_equal(
            rel, oracle.ref_chunked_radix_partition(keys, pays, off, chunks, bits))


@settings(max_examples=40, deadline=None)
@given(n_b=st.integers(1, 3000), n_p=st.integers(1, 6000), lg=st.integers(1, 13),
       dt=st.sampled_from(DTYPES), kind=st.sampled_from(KINDS),
       seed=st.integers(0, 2**32 - 1))
def test_cpu_linear_probing_random(fi, oracle, n_b, n_p, lg, dt, kind, seed):
    size = 1 << lg
    n_b = min(n_b, size - 1)  # every build tuple finds a slot, one stays empty
    if n_b < 1:
        return
    rng = np.random.default_rng(seed)
    bk = draw_keys(rng, n_b, dt, kind)
    bk[bk == -1] = 0  # -1 is the null key of the table
    bp = rng.integers(-2**30, 2**30, n_b).astype(dt)
    pk = np.where(rng.random(n_p) < 0.5, rng.choice(bk, n_p),
                  draw_keys(rng, n_p, dt, kind)).astype(dt)
    pk[pk == -1] = 1
    pp = rng.integers(np.iinfo(dt).min, np.iinfo(dt).max, n_p, dtype=dt, endpoint=True)
    exp_sum, exp_ht = oracle.ht_linearprobing_sum(bk, bp, pk, pp, size)
    ht = fi.CpuHashTable(size, dt)
    hj = fi.CpuHashJoin(fi.HashingScheme.LinearProbing, ht)
    hj.build(bk, bp)
    np.testing.assert_array_equal(ht.mem, exp_ht)
    assert hj.probe_sum(pk, pp) == exp_sum
    if oracle.ref_available():
        ref_sum, _ = oracle.ref_ht_linearprobing_sum(bk, bp, pk, pp, size)
        assert int(exp_sum) == int(ref_sum)
