"""The oracle against the reference's compiled CPU operators on random
inputs: sizes, chunk counts, radix bits and key distributions drawn by
hypothesis (full-range keys, negative keys, a few distinct keys, ragged
sizes smaller than the chunk count).  Offsets and the NC-partitioned
relation must be identical byte for byte; the linear-probing join sums and
the bucket-chaining radix join's sum and match count equal the reference's.
Skipped where the reference library is not built."""
import numpy as np
import pytest

hypothesis = pytest.importorskip("hypothesis")
from hypothesis import given, settings, strategies as st  # noqa: E402

DTYPES = [np.int32, np.int64]


def draw_keys(rng, n, dt, kind):
    info = np.iinfo(dt)
    if kind == "full":
        return rng.integers(info.min, info.max, n, dtype=dt, endpoint=True)
    if kind == "negative":
        return rng.integers(-(1 << 20), 0, n).astype(dt)
    return rng.integers(0, 7, n).astype(dt)  # "few": heavy duplicates


@settings(max_examples=60, deadline=None)
@given(n=st.integers(1, 5000), chunks=st.integers(1, 9), bits=st.integers(0, 12),
       dt=st.sampled_from(DTYPES), kind=st.sampled_from(["full", "negative", "few"]),
       seed=st.integers(0, 2**32 - 1))
def test_partition_matches_compiled_reference(oracle, n, chunks, bits, dt, kind, seed):
    if not oracle.ref_available():
        pytest.skip("reference CPU library not built")
    rng = np.random.default_rng(seed)
    keys = draw_keys(rng, n, dt, kind)
    pays = rng.integers(np.iinfo(dt).min, np.iinfo(dt).max, n, dtype=dt, endpoint=True)
    off = oracle.chunked_prefix_sum(keys, chunks, bits)
    np.testing.assert_array_equal(off, oracle.ref_chunked_prefix_sum(keys, chunks, bits))
    pad = oracle.padding_len(dt)
    padded = n + chunks * (1 << bits) * pad
    rel = oracle.chunked_radix_partition(keys, pays, off, chunks, bits, 0, padded)
    np.testing.assert_array_equal(
        rel, oracle.ref_chunked_radix_partition(keys, pays, off, chunks, bits))


@settings(max_examples=40, deadline=None)
@given(n_b=st.integers(1, 3000), n_p=st.integers(1, 6000), lg=st.integers(1, 13),
       dt=st.sampled_from(DTYPES), kind=st.sampled_from(["full", "negative", "few"]),
       seed=st.integers(0, 2**32 - 1))
def test_linear_probing_sum_matches_compiled_reference(oracle, n_b, n_p, lg, dt, kind,
                                                       seed):
    if not oracle.ref_available():
        pytest.skip("reference CPU library not built")
    size = 1 << lg
    n_b = min(n_b, size - 1)  # every build tuple finds a slot, one stays empty
    if n_b < 1:
        return
    rng = np.random.default_rng(seed)
    r_key = draw_keys(rng, n_b, dt, kind)
    r_key[r_key == -1] = 0  # -1 is the null key of the table
    r_pay = rng.integers(-1000, 1000, n_b).astype(dt)
    # probes: half drawn from the build keys, half from the same distribution
    s_key = np.where(rng.random(n_p) < 0.5, rng.choice(r_key, n_p),
                     draw_keys(rng, n_p, dt, kind)).astype(dt)
    s_key[s_key == -1] = 1
    s_pay = rng.integers(np.iinfo(dt).min, np.iinfo(dt).max, n_p, dtype=dt,
                         endpoint=True)
    got, _ = oracle.ht_linearprobing_sum(r_key, r_pay, s_key, s_pay, size)
    exp, _ = oracle.ref_ht_linearprobing_sum(r_key, r_pay, s_key, s_pay, size)
    assert int(got) == int(exp)


@settings(max_examples=40, deadline=None)
@given(n_b=st.integers(1, 4000), n_p=st.integers(1, 8000), bits=st.integers(0, 8),
       dt=st.sampled_from(DTYPES), kind=st.sampled_from(["full", "negative", "few"]),
       seed=st.integers(0, 2**32 - 1))
def test_radix_join_matches_compiled_reference(oracle, n_b, n_p, bits, dt, kind, seed):
    """The bucket-chaining radix-join restatement (one pass, Chunked with one
    chunk, as the reference's join tests partition) against the sum and
    match count of the reference's compiled linear-probing join, which adds
    s.value once per build tuple with an equal key."""
    if not oracle.ref_available():
        pytest.skip("reference CPU library not built")
    rng = np.random.default_rng(seed)
    rk = draw_keys(rng, n_b, dt, kind)
    rk[rk == -1] = 0  # the null key stays out of the reference's table
    rp = rng.integers(np.iinfo(dt).min, np.iinfo(dt).max, n_b, dtype=dt, endpoint=True)
    sk = np.where(rng.random(n_p) < 0.5, rng.choice(rk, n_p),
                  draw_keys(rng, n_p, dt, kind)).astype(dt)
    sk[sk == -1] = 1
    sp = rng.integers(np.iinfo(dt).min, np.iinfo(dt).max, n_p, dtype=dt, endpoint=True)
    # the reference: Σ s.value over all (r, s) with equal keys, and the count
    entries = 1 << int(2 * n_b - 1).bit_length()
    exp_s, _ = oracle.ref_ht_linearprobing_sum(rk, rp, sk, sp, entries)
    exp_c, _ = oracle.ref_ht_linearprobing_sum(rk, rp, sk, np.ones_like(sp), entries)
    pad = oracle.padding_len(dt)
    F = 1 << bits
    rels = []
    for k, v in ((rk, rp), (sk, sp)):
        off = oracle.chunked_prefix_sum(k, 1, bits)
        rels.append((oracle.chunked_radix_partition(k, v, off, 1, bits, 0,
                                                    len(k) + F * pad), off))
    (b_rel, b_off), (p_rel, p_off) = rels
    s, c = oracle.radix_join("chaining", b_rel, b_off, pad, p_rel, p_off, pad, bits,
                             bits, ht_entries=1)
    assert (np.uint64(s % (1 << 64)), c) == (np.uint64(exp_s), exp_c)
