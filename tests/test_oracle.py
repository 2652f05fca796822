"""The oracle is pinned before it is trusted: against the golden fixtures made
by the reference's own compiled CPU operators (tests/golden/make_golden.py),
and, where that library is present, against it directly on more cases."""
import os

import numpy as np
import pytest

GOLDEN = os.path.join(os.path.dirname(__file__), "golden", "reference_cpu_ops.npz")


@pytest.fixture(scope="module")
def golden():
    return np.load(GOLDEN)


@pytest.mark.parametrize("name,dt", [("i32", np.int32), ("i64", np.int64)])
@pytest.mark.parametrize("chunks,bits", [(1, 0), (3, 4), (7, 6), (4, 9)])
def test_oracle_matches_golden_partition(oracle, golden, name, dt, chunks, bits):
    keys, pays = golden[name + "_keys"], golden[name + "_pays"]
    pad = oracle.padding_len(dt)
    exp_off = golden["%s_offsets_c%d_b%d" % (name, chunks, bits)]
    off = oracle.chunked_prefix_sum(keys, chunks, bits)
    np.testing.assert_array_equal(off, exp_off)
    padded = len(keys) + chunks * (1 << bits) * pad
    rel = oracle.chunked_radix_partition(keys, pays, off, chunks, bits, 0, padded)
    # the sequential NC scatter is deterministic: byte-identical
    np.testing.assert_array_equal(rel, golden["%s_nc_c%d_b%d" % (name, chunks, bits)])
    # SWWC output: same per-(chunk, partition) multisets
    swwc = golden["%s_swwc_c%d_b%d" % (name, chunks, bits)]
    a = oracle.partition_multisets(rel, off, chunks, bits, padded, pad)
    b = oracle.partition_multisets(swwc, off, chunks, bits, padded, pad)
    for x, y in zip(a, b):
        np.testing.assert_array_equal(x, y)


@pytest.mark.parametrize("name,dt", [("i32", np.int32), ("i64", np.int64)])
def test_oracle_matches_golden_hash_join(oracle, golden, name, dt):
    keys, pays = golden[name + "_keys"], golden[name + "_pays"]
    fk, fpay = golden[name + "_fk"], golden[name + "_fpay"]
    s_lp, _ = oracle.ht_linearprobing_sum(keys, pays, fk, fpay, 1 << 13)
    assert s_lp == int(golden[name + "_lp_sum"][0])
    s_pf, _ = oracle.ht_perfect_sum(keys, pays, fk, fpay, len(keys) + 1)
    assert s_pf == int(golden[name + "_perfect_sum"][0])


@pytest.mark.parametrize("dt", [np.int32, np.int64])
@pytest.mark.parametrize("n,chunks,bits", [(100, 1, 0), (100, 4, 2),
                                           (100003, 10, 6), (250000, 8, 12),
                                           (3000, 1, 13), (77, 3, 9)])
def test_oracle_matches_compiled_reference(oracle, dt, n, chunks, bits):
    if not oracle.ref_available():
        pytest.skip("reference CPU library not built")
    keys = oracle.primary_keys(n, 11, dt, base=0)
    pays = oracle.uniform_foreign_keys(n, 1000, 12, dt)
    off = oracle.chunked_prefix_sum(keys, chunks, bits)
    np.testing.assert_array_equal(off, oracle.ref_chunked_prefix_sum(keys, chunks, bits))
    pad = oracle.padding_len(dt)
    padded = n + chunks * (1 << bits) * pad
    rel = oracle.chunked_radix_partition(keys, pays, off, chunks, bits, 0, padded)
    ref = oracle.ref_chunked_radix_partition(keys, pays, off, chunks, bits)
    np.testing.assert_array_equal(rel, ref)


def test_oracle_contiguous_closed_form(oracle):
    """offsets[p] = sum_{q<p} hist[q] + (p+1)*pad (radix_partition.cu:171-198)."""
    keys = oracle.uniform_foreign_keys(50000, 1 << 20, 5, np.int64)
    bits, pad = 7, 8
    off, loc = oracle.contiguous_prefix_sum(keys, 13, bits)
    hist = np.bincount(keys & ((1 << bits) - 1), minlength=1 << bits)
    exp = np.concatenate([[0], np.cumsum(hist)[:-1]]) + (np.arange(1 << bits) + 1) * pad
    np.testing.assert_array_equal(off, exp.astype(np.uint64))
    np.testing.assert_array_equal(loc[: 1 << bits], off)
    # per-block cursors are non-decreasing down a partition
    loc2 = loc.reshape(13, 1 << bits)
    assert (np.diff(loc2.astype(np.int64), axis=0) >= 0).all()


def test_oracle_join_closed_form(oracle):
    """payload = row + 1 and FK covering PK: sum = N_s (N_s + 1) / 2
    (test_cuda_radix_join.rs:65-75,179-182)."""
    n = 40000
    r_key = oracle.primary_keys(n, 3, np.int64, base=0)
    s_key = oracle.uniform_foreign_keys(n, n, 4, np.int64, base=0)
    s_pay = np.arange(1, n + 1, dtype=np.int64)
    r_pay = np.arange(1, n + 1, dtype=np.int64)
    bits, pad = 6, 8
    b_off, _ = oracle.contiguous_prefix_sum(r_key, 1, bits)
    p_off, _ = oracle.contiguous_prefix_sum(s_key, 1, bits)
    b_rel = oracle.chunked_radix_partition(r_key, r_pay, b_off, 1, bits, 0, n + 64 * pad)
    p_rel = oracle.chunked_radix_partition(s_key, s_pay, p_off, 1, bits, 0, n + 64 * pad)
    for scheme in ("chaining", "perfect"):
        s, c = oracle.radix_join(scheme, b_rel, b_off, pad, p_rel, p_off, pad,
                                 bits, bits, ht_entries=14527)
        assert c == n
        assert s == n * (n + 1) // 2


def test_cpu_baseline_matches_oracle(oracle):
    n = 1 << 16
    r = oracle.primary_keys(n, 1, np.int64)
    s = oracle.uniform_foreign_keys(n, n, 2, np.int64)
    exp = int(s.sum())
    for use_ref in (False, True):
        if use_ref and not oracle.ref_available():
            continue
        sm, cnt, _, kind = oracle.cpu_radix_join(r, r.copy(), s, s.copy(), 5, 4,
                                                 4, use_reference=use_ref)
        assert cnt == n and sm == exp, kind


def test_datagen_shapes(oracle):
    pk = oracle.primary_keys(100003, 9, np.int64)
    assert np.array_equal(np.sort(pk), np.arange(1, 100004))
    pk32 = oracle.primary_keys(5000, 9, np.int32, base=0)
    assert np.array_equal(np.sort(pk32), np.arange(5000))
    fk = oracle.uniform_foreign_keys(200000, 1000, 3, np.int64)
    assert fk.min() >= 1 and fk.max() <= 1000
    assert abs(np.bincount(fk)[1:].mean() - 200) < 1
    z = oracle.zipf_foreign_keys(200000, 100000, 1.5, 4, 9, np.int64)
    _, cnt = np.unique(z, return_counts=True)
    # P(rank 1) = 1 / H_{N,1.5} ~ 0.383
    assert 0.37 < cnt.max() / len(z) < 0.40
    assert set(np.unique(z)) <= set(oracle.primary_keys(100000, 9, np.int64))


# --------------------------------------------------------------------------
# The radix-join restatement pinned to the reference's own join code.
# The reference's linear-probing join (no_partitioning_join.cpp:27-140) adds
# s.value once per build tuple with an equal key, which is what the radix
# join aggregates (radix_join.cu:103-311); the match count is the same join
# with every probe payload set to 1.  Cases: about half of the probe tuples
# missing, duplicate build keys, negative keys and payloads (int32 sign
# extension through key_to_partition), and all but one partition empty.
# --------------------------------------------------------------------------
import importlib.util as _ilu  # noqa: E402

_spec = _ilu.spec_from_file_location(
    "make_golden", os.path.join(os.path.dirname(__file__), "golden", "make_golden.py"))
make_golden = _ilu.module_from_spec(_spec)
_spec.loader.exec_module(make_golden)

PIN_DTYPES = [("i32", np.int32), ("i64", np.int64)]
# the perfect scheme is defined for unique, non-negative build keys
PERFECT_KINDS = ("misses", "sparse")


def _one_pass_join(oracle, scheme, rk, rp, sk, sp, bits):
    """Partition both sides into one contiguous relation (Chunked, one chunk)
    and run the oracle's per-partition join on it."""
    pad = oracle.padding_len(rk.dtype)
    F = 1 << bits
    rels = []
    for k, v in ((rk, rp), (sk, sp)):
        off = oracle.chunked_prefix_sum(k, 1, bits)
        rels.append((oracle.chunked_radix_partition(k, v, off, 1, bits, 0,
                                                    len(k) + F * pad), off))
    (b_rel, b_off), (p_rel, p_off) = rels
    entries = 1
    if scheme == "perfect":
        entries = int(max(int(rk.max()), int(sk.max()))) // F + 1
    return oracle.radix_join(scheme, b_rel, b_off, pad, p_rel, p_off, pad, bits,
                             bits, ht_entries=entries)


@pytest.mark.parametrize("kind", make_golden.JOIN_PIN_KINDS)
@pytest.mark.parametrize("name,dt", PIN_DTYPES)
@pytest.mark.parametrize("scheme", ["chaining", "perfect"])
@pytest.mark.parametrize("bits", [0, 4, 6])
def test_oracle_radix_join_matches_golden(oracle, golden, kind, name, dt, scheme,
                                          bits):
    if scheme == "perfect" and kind not in PERFECT_KINDS:
        pytest.skip("perfect hashing needs unique non-negative build keys")
    pre = "join_pin_%s_%s_" % (kind, name)
    rk, rp = golden[pre + "r_key"], golden[pre + "r_pay"]
    sk, sp = golden[pre + "s_key"], golden[pre + "s_pay"]
    s, c = _one_pass_join(oracle, scheme, rk, rp, sk, sp, bits)
    assert np.uint64(s % (1 << 64)) == golden[pre + "sum"][0]
    assert c == int(golden[pre + "count"][0])


@pytest.mark.parametrize("kind", make_golden.JOIN_PIN_KINDS)
@pytest.mark.parametrize("bits1,bits2,threads", [(3, 3, 1), (5, 4, 4), (0, 6, 3)])
def test_oracle_two_pass_join_matches_golden(oracle, golden, kind, bits1, bits2,
                                             threads):
    """The two-pass CPU radix join (pass 1, pass 2 over each first-pass
    partition, bucket-chaining join) that the engine tests compare with."""
    pre = "join_pin_%s_i64_" % kind
    rk, rp = golden[pre + "r_key"], golden[pre + "r_pay"]
    sk, sp = golden[pre + "s_key"], golden[pre + "s_pay"]
    s, c, _, _ = oracle.cpu_radix_join(rk, rp, sk, sp, bits1, bits2, threads,
                                       use_reference=False)
    assert np.uint64(s % (1 << 64)) == golden[pre + "sum"][0]
    assert c == int(golden[pre + "count"][0])


@pytest.mark.parametrize("kind", make_golden.JOIN_PIN_KINDS)
@pytest.mark.parametrize("name,dt", PIN_DTYPES)
def test_oracle_radix_join_matches_compiled_reference(oracle, kind, name, dt):
    """Larger inputs than the fixtures, against the compiled reference."""
    if not oracle.ref_available():
        pytest.skip("reference CPU library not built")
    seed = 100 * make_golden.JOIN_PIN_KINDS.index(kind) + (32 if name == "i32" else 64)
    rng = np.random.default_rng(seed)
    rk, rp, sk, sp = make_golden.join_pin_inputs(kind, dt, rng, 40000, 90001)
    exp_s, exp_c = make_golden.ref_join_sum_count(rk, rp, sk, sp)
    for scheme in ("chaining", "perfect"):
        if scheme == "perfect" and kind not in PERFECT_KINDS:
            continue
        for bits in (2, 7):
            s, c = _one_pass_join(oracle, scheme, rk, rp, sk, sp, bits)
            assert (np.uint64(s % (1 << 64)), c) == (np.uint64(exp_s), exp_c), (
                scheme, bits)
    if dt == np.int64:
        for use_ref in (False, True):
            s, c, _, _ = oracle.cpu_radix_join(rk, rp, sk, sp, 4, 5, 4,
                                               use_reference=use_ref)
            assert (np.uint64(s % (1 << 64)), c) == (np.uint64(exp_s), exp_c), use_ref


@pytest.mark.parametrize("dt", [np.int32, np.int64])
def test_oracle_linear_probing_tiny_tables(oracle, dt):
    """Tables of 1..8 slots (one slot: the reference's hash would shift by
    the whole word width, undefined; slot 0 here, as on the GPU): every
    probe key adds its payload once per equal build key."""
    for size in (1, 2, 3, 4, 8):
        slots = 1 << (size.bit_length() - 1)
        r = np.array([0, 0, 1, 5, 7, 0, 3, 1][:slots], dt)
        s = np.array([0, 1, 2, 0, 7, 9], dt)
        sp = np.array([1, 2, 3, 4, 5, 6], dt)
        got, _ = oracle.ht_linearprobing_sum(r, r + 5, s, sp, size)
        exp = sum(int(p) * int((r == k).sum()) for k, p in zip(s, sp))
        assert got == exp, size
