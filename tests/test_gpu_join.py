"""GPU parity of the joins against the oracle, through the C ABI.

Radix join: the reference's known-answer tests (test_cuda_radix_join.rs:
40-365): primary keys 0..N-1 shuffled, foreign keys over them, payload =
row + 1, so SUM(s.value) = N_s (N_s + 1) / 2; perfect hashing on 6100*2^b
build tuples and bucket chaining on 4096*2^b, grids of 1, 3 and 80 blocks.
Plus: sum and match count equal to the oracle's restated join, the task
assignments equal to the reference's greedy split, Zipf-skewed probes and
build partitions larger than shared memory.  No-partitioning join: sums equal
to the reference CPU operators' (golden-pinned oracle).  Engine: the whole
gpu_radix_join against the oracle on one- and two-pass configurations."""
import numpy as np
import pytest
import torch

from _helpers import to_dev, to_host

pytestmark = pytest.mark.gpu

DTYPES = [(np.int32, torch.int32), (np.int64, torch.int64)]


def partition_contiguous(fi, keys, pays, bits, radix_bits=None, pass_=None,
                         hist="Chunked"):
    """One contiguous relation as the reference join tests build it
    (Chunked with num_chunks = 1)."""
    tdt = keys.dtype
    radix_bits = radix_bits or fi.RadixBits(bits)
    pass_ = fi.RadixPass.First if pass_ is None else pass_
    H = getattr(fi.GpuHistogramAlgorithm, hist)
    p = fi.GpuRadixPartitioner(H, fi.GpuRadixPartitionAlgorithm.NC, radix_bits, 1, 1024)
    o = fi.PartitionOffsets(H, 1, bits, tdt)
    rel = fi.PartitionedRelation(keys.numel(), H, bits, 1, tdt, fill=-1)
    p.prefix_sum(pass_, keys, o)
    p.partition(pass_, keys, pays, o, rel)
    return rel


def gen_join(oracle, n_build, n_probe, dt, seed, zipf=None):
    r_key = oracle.primary_keys(n_build, seed, dt, base=0)
    if zipf is None:
        s_key = oracle.uniform_foreign_keys(n_probe, n_build, seed + 1, dt, base=0)
    else:
        s_key = oracle.zipf_foreign_keys(n_probe, n_build, zipf, seed + 1, seed, dt,
                                         base=0)
    r_pay = np.arange(1, n_build + 1, dtype=dt)
    s_pay = np.arange(1, n_probe + 1, dtype=dt)
    return r_key, r_pay, s_key, s_pay


JOIN_CASES = [("Perfect", 0, 6100), ("Perfect", 4, 6100 * 16), ("Perfect", 8, 6100 * 256),
              ("BucketChaining", 0, 4096), ("BucketChaining", 3, 4096 * 8),
              ("BucketChaining", 8, 4096 * 256)]


@pytest.mark.parametrize("ndt,tdt", DTYPES)
@pytest.mark.parametrize("scheme,bits,n", JOIN_CASES)
@pytest.mark.parametrize("grid,block", [(1, 128), (3, 256), (80, 1024)])
def test_radix_join_known_answer(fi, oracle, ndt, tdt, scheme, bits, n, grid, block):
    r_key, r_pay, s_key, s_pay = gen_join(oracle, n, n, ndt, 10 + bits)
    b = partition_contiguous(fi, to_dev(r_key), to_dev(r_pay), bits)
    pr = partition_contiguous(fi, to_dev(s_key), to_dev(s_pay), bits)
    result = torch.zeros(grid * block, dtype=torch.int64, device="cuda")
    tasks = torch.zeros(grid + 1, dtype=torch.int32, device="cuda")
    count = torch.zeros(1, dtype=torch.int64, device="cuda")
    j = fi.CudaRadixJoin(fi.RadixPass.First, fi.RadixBits(bits),
                         getattr(fi.HashingScheme, scheme), grid, block)
    j.join(b, pr, result, tasks, match_count=count)
    j.status()
    assert int(to_host(result).sum()) == n * (n + 1) // 2
    assert int(to_host(count)[0]) == n
    # task assignments as the reference's greedy split (radix_join.cu:58-98)
    exp_tasks = oracle.assign_tasks(to_host(pr.offsets).astype(np.uint64),
                                    pr.padded_len(), pr.padding_len(), bits, grid,
                                    ndt)
    np.testing.assert_array_equal(to_host(tasks).astype(np.uint32), exp_tasks)


@pytest.mark.parametrize("ndt,tdt", DTYPES)
@pytest.mark.parametrize("scheme", ["Perfect", "BucketChaining"])
@pytest.mark.parametrize("zipf", [None, 0.5, 1.0, 1.5])
def test_radix_join_matches_oracle(fi, oracle, ndt, tdt, scheme, zipf):
    bits, n_b, n_p = 7, 300000, 700001
    r_key, r_pay, s_key, _ = gen_join(oracle, n_b, n_p, ndt, 31, zipf=zipf)
    s_pay = oracle.uniform_foreign_keys(n_p, 1 << 30, 77, ndt) - (1 << 29)
    b = partition_contiguous(fi, to_dev(r_key), to_dev(r_pay), bits)
    pr = partition_contiguous(fi, to_dev(s_key), to_dev(s_pay.astype(ndt)), bits)
    grid, block = 148, 1024
    result = torch.zeros(grid * block, dtype=torch.int64, device="cuda")
    tasks = torch.zeros(grid + 1, dtype=torch.int32, device="cuda")
    count = torch.zeros(1, dtype=torch.int64, device="cuda")
    j = fi.CudaRadixJoin(fi.RadixPass.First, fi.RadixBits(bits),
                         getattr(fi.HashingScheme, scheme), grid, block)
    j.join(b, pr, result, tasks, match_count=count)
    j.status()
    bh, ph = to_host(b.relation), to_host(pr.relation)
    s, c = oracle.radix_join("chaining" if scheme == "BucketChaining" else "perfect",
                             bh[:b.padded_len()], to_host(b.offsets).astype(np.uint64),
                             b.padding_len(), ph[:pr.padded_len()],
                             to_host(pr.offsets).astype(np.uint64), pr.padding_len(),
                             bits, bits, ht_entries=1 << 20)
    got = int(to_host(result).astype(np.int64).sum(dtype=np.int64))
    assert got == s
    assert int(to_host(count)[0]) == c == n_p


def test_radix_join_build_larger_than_shared_memory(fi, oracle):
    """One partition of 200K build tuples: joined in shared-memory rounds
    (the reference asserts on this size, radix_join.cu:251-252)."""
    n = 200000
    r_key, r_pay, s_key, s_pay = gen_join(oracle, n, n, np.int64, 5)
    b = partition_contiguous(fi, to_dev(r_key), to_dev(r_pay), 0)
    pr = partition_contiguous(fi, to_dev(s_key), to_dev(s_pay), 0)
    result = torch.zeros(148 * 1024, dtype=torch.int64, device="cuda")
    tasks = torch.zeros(149, dtype=torch.int32, device="cuda")
    j = fi.CudaRadixJoin(fi.RadixPass.First, fi.RadixBits(0),
                         fi.HashingScheme.BucketChaining, 148, 1024)
    j.join(b, pr, result, tasks)
    j.status()
    assert int(to_host(result).sum()) == n * (n + 1) // 2


def test_radix_join_second_pass_relations(fi, oracle):
    """A join on second-pass relations (ignore bits = first + second pass
    bits, cuda_radix_join.rs:207-208)."""
    n, b1, b2 = 100000, 3, 5
    r_key, r_pay, s_key, s_pay = gen_join(oracle, n, n, np.int64, 6)
    bits = fi.RadixBits(b1, b2)
    # every key of one first-pass partition: keys with low b1 bits == 2
    rk, rp = r_key[(r_key & 7) == 2], r_pay[(r_key & 7) == 2]
    sk, sp = s_key[(s_key & 7) == 2], s_pay[(s_key & 7) == 2]
    b = partition_contiguous(fi, to_dev(rk), to_dev(rp), b2, bits, fi.RadixPass.Second)
    pr = partition_contiguous(fi, to_dev(sk), to_dev(sp), b2, bits, fi.RadixPass.Second)
    result = torch.zeros(10 * 256, dtype=torch.int64, device="cuda")
    tasks = torch.zeros(11, dtype=torch.int32, device="cuda")
    for scheme in (fi.HashingScheme.Perfect, fi.HashingScheme.BucketChaining):
        result.zero_()
        j = fi.CudaRadixJoin(fi.RadixPass.Second, bits, scheme, 10, 256)
        j.join(b, pr, result, tasks)
        j.status()
        assert int(to_host(result).sum()) == int(sp.sum())


def test_radix_join_validation(fi):
    rel = fi.PartitionedRelation(10, fi.GpuHistogramAlgorithm.Chunked, 2, 4, torch.int64)
    one = fi.PartitionedRelation(10, fi.GpuHistogramAlgorithm.Chunked, 2, 1, torch.int64)
    j = fi.CudaRadixJoin(fi.RadixPass.First, fi.RadixBits(2), fi.HashingScheme.Perfect,
                         4, 128)
    res = torch.zeros(512, dtype=torch.int64, device="cuda")
    with pytest.raises(fi.SqlOpsError, match="Chunked build relations"):
        j.join(rel, one, res, torch.zeros(5, dtype=torch.int32, device="cuda"))
    with pytest.raises(fi.SqlOpsError, match="grid size \\+ 1"):
        j.join(one, one, res, torch.zeros(4, dtype=torch.int32, device="cuda"))
    lp = fi.CudaRadixJoin(fi.RadixPass.First, fi.RadixBits(2),
                          fi.HashingScheme.LinearProbing, 4, 128)
    with pytest.raises(fi.SqlOpsError) as e:
        lp.join(one, one, res, torch.zeros(5, dtype=torch.int32, device="cuda"))
    assert e.value.kind == "Unsupported"


@pytest.mark.parametrize("ndt,tdt", DTYPES)
@pytest.mark.parametrize("scheme", ["LinearProbing", "Perfect"])
def test_hash_join(fi, oracle, ndt, tdt, scheme):
    n_b, n_p = 100003, 300007
    r_key = oracle.primary_keys(n_b, 3, ndt, base=0)
    r_pay = oracle.uniform_foreign_keys(n_b, 1000, 4, ndt)
    s_key = oracle.uniform_foreign_keys(n_p, n_b + 500, 5, ndt, base=0)
    s_pay = oracle.uniform_foreign_keys(n_p, 1 << 20, 6, ndt)
    size = (1 << 18) if scheme == "LinearProbing" else n_b + 500
    ht = fi.HashTable(size, tdt)
    hj = fi.CudaHashJoin(getattr(fi.HashingScheme, scheme), ht, (148, 512), (148, 512))
    hj.build(to_dev(r_key), to_dev(r_pay))
    res = torch.zeros(148 * 512, dtype=torch.int64, device="cuda")
    hj.probe_sum(to_dev(s_key), to_dev(s_pay), res)
    got = int(to_host(res).astype(np.uint64).sum(dtype=np.uint64))
    if scheme == "LinearProbing":
        exp, _ = oracle.ht_linearprobing_sum(r_key, r_pay, s_key, s_pay, size)
    else:
        exp, _ = oracle.ht_perfect_sum(r_key, r_pay, s_key, s_pay, size)
    assert got == exp


@pytest.mark.parametrize("ndt,tdt", DTYPES)
@pytest.mark.parametrize("size,n_b,n_p", [(1, 1, 50), (2, 2, 77), (3, 2, 64),
                                          (4, 3, 500), (8, 7, 999), (64, 60, 5000),
                                          (1024, 1000, 20011), (5000, 3000, 40009)])
def test_hash_join_linear_probing_windows(fi, oracle, ndt, tdt, size, n_b, n_p):
    """Linear probing loads a window of slots per step (4 int64 / 8 int32
    entries, the int32 window from the hash slot's aligned pair): tables of
    1..8 slots where a window wraps onto itself, nearly full tables whose
    probes cross many windows, duplicate build keys and misses; the sums
    equal the oracle's (pinned to the reference's compiled CPU join)."""
    rng = np.random.default_rng(size * 7 + n_p)
    lg = size.bit_length() - 1
    slots = 1 << lg  # the reference hashes into 2^floor(log2(size)) slots
    n_b = min(n_b, slots)  # every build tuple finds a slot
    r_key = rng.integers(0, max(2, n_b // 2 + 1), n_b).astype(ndt)  # duplicates
    r_pay = rng.integers(-1000, 1000, n_b).astype(ndt)
    s_key = rng.integers(0, n_b + 3, n_p).astype(ndt)  # some miss
    s_pay = rng.integers(-(1 << 20), 1 << 20, n_p).astype(ndt)
    ht = fi.HashTable(size, tdt)
    hj = fi.CudaHashJoin(fi.HashingScheme.LinearProbing, ht, (37, 128), (37, 128))
    hj.build(to_dev(r_key), to_dev(r_pay))
    res = torch.zeros(37 * 128, dtype=torch.int64, device="cuda")
    hj.probe_sum(to_dev(s_key), to_dev(s_pay), res)
    got = int(to_host(res).astype(np.uint64).sum(dtype=np.uint64))
    exp, _ = oracle.ht_linearprobing_sum(r_key, r_pay, s_key, s_pay, size)
    assert got == exp


@pytest.mark.parametrize("ndt,tdt", DTYPES)
@pytest.mark.parametrize("scheme", ["LinearProbing", "Perfect"])
@pytest.mark.parametrize("slice_", [1 << 27, 1_000_003])
def test_hash_join_grouped_probe(fi, oracle, ndt, tdt, scheme, slice_):
    """Tables larger than a region (8 MB) probed by at least one probe per
    slot are probed region by region (the probe side grouped slice by
    slice): the sum equals the oracle's and the ungrouped probe's, also when
    slices split the probe side, with duplicate build keys, misses, keys
    beyond a perfect table and negative payloads."""
    rng = np.random.default_rng(11 + (slice_ & 7))
    size = 1 << 21 if ndt == np.int64 else 1 << 22  # 32 MB tables
    n_b = size // 2 if scheme == "LinearProbing" else size - 7
    if scheme == "LinearProbing":
        r_key = rng.integers(0, size // 3, n_b).astype(ndt)  # duplicates
    else:
        r_key = rng.permutation(n_b).astype(ndt)
    r_pay = rng.integers(-1000, 1000, n_b).astype(ndt)
    n_p = 3 * size + 12345
    s_key = rng.integers(-5, size + 100, n_p).astype(ndt)
    s_pay = rng.integers(-(1 << 20), 1 << 20, n_p).astype(ndt)
    dk, dp = to_dev(s_key), to_dev(s_pay)
    got = []
    for grouping in (True, False):
        ht = fi.HashTable(size, tdt)
        hj = fi.CudaHashJoin(getattr(fi.HashingScheme, scheme), ht, (148, 512), (148, 512))
        hj.set_probe_grouping(grouping, slice_)
        hj.build(to_dev(r_key), to_dev(r_pay))
        res = torch.zeros(148 * 512, dtype=torch.int64, device="cuda")
        hj.probe_sum(dk, dp, res)
        hj.status()
        got.append(int(to_host(res).astype(np.uint64).sum(dtype=np.uint64)))
    if scheme == "LinearProbing":
        exp, _ = oracle.ht_linearprobing_sum(r_key, r_pay, s_key, s_pay, size)
    else:
        exp, _ = oracle.ht_perfect_sum(r_key, r_pay, s_key, s_pay, size)
    assert got[0] == got[1] == exp


@pytest.mark.parametrize("ndt,tdt", DTYPES)
@pytest.mark.parametrize("scheme", ["LinearProbing", "Perfect"])
@pytest.mark.parametrize("slice_", [1 << 27, 1_000_003])
def test_hash_join_grouped_probe_skewed(fi, oracle, ndt, tdt, scheme, slice_):
    """A probe slice whose largest table region holds more than a quarter of
    it (here half the probes are one key) is probed in input order instead
    of grouped; the sums equal the oracle's and the ungrouped probe's, also
    when slices split the probe side (unaligned slices take the per-tile
    grouping, which always groups)."""
    rng = np.random.default_rng(5 + (slice_ & 3))
    size = 1 << 21 if ndt == np.int64 else 1 << 22  # 32 MB tables
    n_b = size // 2
    r_key = rng.permutation(n_b).astype(ndt)
    r_pay = rng.integers(-1000, 1000, n_b).astype(ndt)
    n_p = 2 * size + 999
    s_key = rng.integers(-3, n_b + 10, n_p).astype(ndt)
    s_key[rng.random(n_p) < 0.5] = 12345  # the hot key
    s_pay = rng.integers(-(1 << 20), 1 << 20, n_p).astype(ndt)
    dk, dp = to_dev(s_key), to_dev(s_pay)
    got = []
    for grouping in (True, False):
        ht = fi.HashTable(size, tdt)
        hj = fi.CudaHashJoin(getattr(fi.HashingScheme, scheme), ht, (148, 512), (148, 512))
        hj.set_probe_grouping(grouping, slice_)
        hj.build(to_dev(r_key), to_dev(r_pay))
        res = torch.zeros(148 * 512, dtype=torch.int64, device="cuda")
        hj.probe_sum(dk, dp, res)
        hj.status()
        got.append(int(to_host(res).astype(np.uint64).sum(dtype=np.uint64)))
    if scheme == "LinearProbing":
        exp, _ = oracle.ht_linearprobing_sum(r_key, r_pay, s_key, s_pay, size)
    else:
        exp, _ = oracle.ht_perfect_sum(r_key, r_pay, s_key, s_pay, size)
    assert got[0] == got[1] == exp


@pytest.mark.parametrize("ndt,tdt", DTYPES)
@pytest.mark.parametrize("scheme", ["LinearProbing", "Perfect"])
def test_hash_join_grouped_probe_small_result_set(fi, oracle, ndt, tdt, scheme):
    """The grouped probe runs on the library's own grid and folds its
    threads' sums into the caller's grid * block entries (here 3 x 96, far
    fewer than its threads): their total is the oracle's sum."""
    rng = np.random.default_rng(61)
    size = 1 << 21 if ndt == np.int64 else 1 << 22  # 32 MB tables
    n_b = size // 2
    r_key = rng.permutation(size)[:n_b].astype(ndt)
    r_pay = rng.integers(-1000, 1000, n_b).astype(ndt)
    n_p = 2 * size + 5
    s_key = rng.integers(0, size + 10, n_p).astype(ndt)
    s_pay = rng.integers(-(1 << 20), 1 << 20, n_p).astype(ndt)
    ht = fi.HashTable(size, tdt)
    hj = fi.CudaHashJoin(getattr(fi.HashingScheme, scheme), ht, (3, 96), (3, 96))
    hj.build(to_dev(r_key), to_dev(r_pay))
    res = torch.zeros(3 * 96, dtype=torch.int64, device="cuda")
    hj.probe_sum(to_dev(s_key), to_dev(s_pay), res)
    hj.status()
    got = int(to_host(res).astype(np.uint64).sum(dtype=np.uint64))
    if scheme == "LinearProbing":
        exp, _ = oracle.ht_linearprobing_sum(r_key, r_pay, s_key, s_pay, size)
    else:
        exp, _ = oracle.ht_perfect_sum(r_key, r_pay, s_key, s_pay, size)
    assert got == exp


@pytest.mark.parametrize("ndt,tdt", DTYPES)
@pytest.mark.parametrize("offset", [0, 1])
def test_hash_join_grouped_probe_table_alignment(fi, oracle, ndt, tdt, offset):
    """The grouped linear-probing probe reads 32-byte windows of the table
    when its base is 32-byte aligned and slot by slot otherwise (a table one
    entry into its allocation): both give the oracle's sum, with duplicate
    build keys, misses and a nearly half-full table."""
    rng = np.random.default_rng(41 + offset)
    size = 1 << 21 if ndt == np.int64 else 1 << 22  # 32 MB tables
    n_b = size // 2
    r_key = rng.integers(0, size // 3, n_b).astype(ndt)
    r_pay = rng.integers(-1000, 1000, n_b).astype(ndt)
    n_p = 2 * size + 77
    s_key = rng.integers(-3, size // 3 + 50, n_p).astype(ndt)
    s_pay = rng.integers(-(1 << 20), 1 << 20, n_p).astype(ndt)
    ht = fi.HashTable(size, tdt, mem_len=size + 1)
    ht.mem = ht.mem[offset:offset + size]
    assert (ht.mem.data_ptr() % 32 == 0) == (offset == 0)
    hj = fi.CudaHashJoin(fi.HashingScheme.LinearProbing, ht, (148, 512), (148, 512))
    hj.build(to_dev(r_key), to_dev(r_pay))
    res = torch.zeros(148 * 512, dtype=torch.int64, device="cuda")
    hj.probe_sum(to_dev(s_key), to_dev(s_pay), res)
    hj.status()
    got = int(to_host(res).astype(np.uint64).sum(dtype=np.uint64))
    exp, _ = oracle.ht_linearprobing_sum(r_key, r_pay, s_key, s_pay, size)
    assert got == exp


@pytest.mark.parametrize("ndt,tdt", DTYPES)
@pytest.mark.parametrize("scheme,selective", [("LinearProbing", False),
                                              ("Perfect", False), ("Perfect", True)])
@pytest.mark.parametrize("slice_", [1 << 27, 333_331])
def test_hash_join_grouped_build(fi, oracle, ndt, tdt, scheme, selective, slice_):
    """Build sides of at least one tuple per 128-byte table line are inserted
    region by region (grouped slice by slice): the probe sums equal the
    oracle's and those of a build in input order, with duplicate build keys
    (linear probing), null and out-of-range build keys (perfect), misses and
    negative payloads, also when slices split the build side."""
    rng = np.random.default_rng(23 + (slice_ & 7) + 2 * selective)
    size = 1 << 21 if ndt == np.int64 else 1 << 22  # 32 MB tables
    if scheme == "LinearProbing":
        n_b = size // 2
        r_key = rng.integers(0, size // 3, n_b).astype(ndt)  # duplicates
    else:
        n_b = size - 9
        r_key = rng.permutation(n_b).astype(ndt)
        r_key[::11] = -1  # the null key: skipped by the selective build
        r_key[5::97] = size + 3  # beyond the table: skipped
    r_pay = rng.integers(-1000, 1000, n_b).astype(ndt)
    n_p = size + 4321
    s_key = rng.integers(-5, size + 100, n_p).astype(ndt)
    s_pay = rng.integers(-(1 << 20), 1 << 20, n_p).astype(ndt)
    rk, rp, dk, dp = to_dev(r_key), to_dev(r_pay), to_dev(s_key), to_dev(s_pay)
    got = []
    for grouping in (True, False):
        ht = fi.HashTable(size, tdt)
        hj = fi.CudaHashJoin(getattr(fi.HashingScheme, scheme), ht, (148, 512),
                             (148, 512), is_selective=selective)
        hj.set_build_grouping(grouping, slice_)
        hj.build(rk, rp)
        res = torch.zeros(148 * 512, dtype=torch.int64, device="cuda")
        hj.probe_sum(dk, dp, res)
        hj.status()
        got.append(int(to_host(res).astype(np.uint64).sum(dtype=np.uint64)))
    if scheme == "LinearProbing":
        exp, _ = oracle.ht_linearprobing_sum(r_key, r_pay, s_key, s_pay, size)
    else:
        exp, _ = oracle.ht_perfect_sum(r_key, r_pay, s_key, s_pay, size, selective)
    assert got[0] == got[1] == exp


def test_hash_join_selective_perfect(fi, oracle):
    n = 50000
    r_key = oracle.primary_keys(n, 3, np.int64, base=0)
    r_key[::7] = -1  # null keys are skipped by the selective build
    r_pay = np.arange(n, dtype=np.int64)
    s_key = oracle.uniform_foreign_keys(n, n, 5, np.int64, base=0)
    s_pay = np.ones(n, np.int64)
    ht = fi.HashTable(n, torch.int64)
    hj = fi.CudaHashJoin(fi.HashingScheme.Perfect, ht, (20, 256), (20, 256),
                         is_selective=True)
    hj.build(to_dev(r_key), to_dev(r_pay))
    res = torch.zeros(20 * 256, dtype=torch.int64, device="cuda")
    hj.probe_sum(to_dev(s_key), to_dev(s_pay), res)
    exp, _ = oracle.ht_perfect_sum(r_key, r_pay, s_key, s_pay, n, selective=True)
    assert int(to_host(res).sum()) == exp


@pytest.mark.parametrize("ndt,tdt", DTYPES)
@pytest.mark.parametrize("bits,scheme", [((10, None), "BucketChaining"),
                                         ((6, 6), "Perfect"),
                                         ((9, 9), "BucketChaining"),
                                         ((9, 9), "Perfect")])
def test_engine_matches_oracle(fi, oracle, ndt, tdt, bits, scheme):
    n_b, n_p = 1 << 21, (1 << 21) + 12345
    r_key = oracle.primary_keys(n_b, 41, ndt)
    r_pay = r_key.copy()
    s_key = oracle.uniform_foreign_keys(n_p, n_b, 42, ndt)
    s_pay = s_key.copy()
    e = fi.RadixJoinEngine(n_b, n_p, tdt, fi.RadixBits(*bits),
                           getattr(fi.HashingScheme, scheme))
    s, c = e.run(to_dev(r_key), to_dev(r_pay), to_dev(s_key), to_dev(s_pay))
    e.status()
    b1 = bits[0]
    b2 = bits[1] or 0
    exp_s, exp_c, _, _ = oracle.cpu_radix_join(
        r_key.astype(np.int64), r_pay.astype(np.int64), s_key.astype(np.int64),
        s_pay.astype(np.int64), b1, max(b2, 1), 8, use_reference=False)
    assert c == exp_c == n_p
    assert s == exp_s


@pytest.mark.parametrize("zipf", [0.0, 0.5, 1.0, 1.5])
def test_engine_zipf_closed_form(fi, oracle, zipf):
    """All S keys are foreign keys: count = |S|, sum = sum(S.payload)."""
    n = 1 << 22
    rk = torch.empty(n, dtype=torch.int64, device="cuda")
    sk = torch.empty(n, dtype=torch.int64, device="cuda")
    fi.gen_primary_keys(rk, 1)
    fi.gen_zipf_foreign_keys(sk, n, zipf, 2, 1)
    e = fi.RadixJoinEngine(n, n, torch.int64, fi.RadixBits(9, 9),
                           fi.HashingScheme.BucketChaining)
    s, c = e.run(rk, rk, sk, sk)
    e.status()
    assert c == n
    assert s == int(sk.sum().item())


def test_engine_int32_config1_bit_exact(fi, oracle):
    """Config 1 (16M x 16M int32, 10 bits, one pass, bucket chaining, payload
    = key) against the CPU radix join."""
    n = 16 << 20
    r_key = oracle.primary_keys(n, 101, np.int32)
    s_key = oracle.uniform_foreign_keys(n, n, 102, np.int32)
    e = fi.RadixJoinEngine(n, n, torch.int32, fi.RadixBits(10),
                           fi.HashingScheme.BucketChaining)
    s, c = e.run(to_dev(r_key), to_dev(r_key), to_dev(s_key), to_dev(s_key))
    e.status()
    exp_s, exp_c, _, _ = oracle.cpu_radix_join(
        r_key.astype(np.int64), r_key.astype(np.int64), s_key.astype(np.int64),
        s_key.astype(np.int64), 10, 1, 8, use_reference=False)
    assert (s, c) == (exp_s, exp_c)


@pytest.mark.parametrize("ndt,tdt", DTYPES)
def test_gpu_generator_matches_cpu(fi, oracle, ndt, tdt):
    n = 1 << 20
    pk = torch.empty(n, dtype=tdt, device="cuda")
    fi.gen_primary_keys(pk, 7, base=1)
    np.testing.assert_array_equal(to_host(pk), oracle.primary_keys(n, 7, ndt, base=1))
    fk = torch.empty(n, dtype=tdt, device="cuda")
    fi.gen_uniform_foreign_keys(fk, 12345, 9, base=1)
    np.testing.assert_array_equal(to_host(fk),
                                  oracle.uniform_foreign_keys(n, 12345, 9, ndt, base=1))
    if ndt == np.int64:
        u = torch.empty(n, dtype=tdt, device="cuda")
        fi.gen_uniform_u64_keys(u, 3)
        np.testing.assert_array_equal(to_host(u), oracle.uniform_u64_keys(n, 3))
    z = torch.empty(n, dtype=tdt, device="cuda")
    fi.gen_zipf_foreign_keys(z, 100000, 1.5, 4, 9)
    zc = oracle.zipf_foreign_keys(n, 100000, 1.5, 4, 9, ndt)
    assert (to_host(z) == zc).mean() > 0.999


@pytest.mark.parametrize("bits", [(7,), (6, 6)])
@pytest.mark.parametrize("scheme", ["Perfect", "BucketChaining"])
def test_engine_build_once_probe_slices(fi, oracle, bits, scheme):
    """The build side stays partitioned across probes: the slices of S,
    probed one by one, add up (wrapping) to the whole-S join."""
    n_b, n_p = 1 << 20, 3 * (1 << 20) + 777
    r_key = oracle.primary_keys(n_b, 61, np.int64)
    s_key = oracle.uniform_foreign_keys(n_p, n_b, 62, np.int64)
    s_pay = oracle.uniform_foreign_keys(n_p, 1 << 62, 63, np.int64)
    e = fi.RadixJoinEngine(n_b, 1 << 20, torch.int64, fi.RadixBits(*bits),
                           getattr(fi.HashingScheme, scheme))
    dk, dp = to_dev(s_key), to_dev(s_pay)
    e.build(to_dev(r_key), to_dev(r_key))
    tot_s, tot_c = 0, 0
    for lo in range(0, n_p, 1 << 20):
        hi = min(n_p, lo + (1 << 20))
        s, c = e.probe(dk[lo:hi], dp[lo:hi])
        tot_s = (tot_s + s) & ((1 << 64) - 1)
        tot_c += c
    e.status()
    exp_s, exp_c, _, _ = oracle.cpu_radix_join(
        r_key, r_key.copy(), s_key, s_pay, bits[0],
        bits[1] if len(bits) > 1 else 1, 8, use_reference=False)
    assert tot_c == exp_c == n_p
    assert tot_s == exp_s & ((1 << 64) - 1)


def test_engine_plans_on_one_engine(fi, oracle):
    """One engine sized for 10+10 bits runs every smaller plan (one or two
    passes, both schemes, every join block and scatter variant, int32
    tuples in an int64-sized engine) with the same result."""
    n = 1 << 20
    r_key = oracle.primary_keys(n, 71, np.int64)
    s_key = oracle.uniform_foreign_keys(2 * n, n, 72, np.int64)
    exp_s, exp_c, _, _ = oracle.cpu_radix_join(
        r_key, r_key.copy(), s_key, s_key.copy(), 6, 6, 8, use_reference=False)
    e = fi.RadixJoinEngine(n, 2 * n, torch.int64, fi.RadixBits(10, 10),
                           fi.HashingScheme.BucketChaining)
    rk, sk = to_dev(r_key), to_dev(s_key)
    rk32, sk32 = rk.to(torch.int32), sk.to(torch.int32)
    for bits in [(8,), (10,), (5, 4), (9, 9), (10, 10)]:
        for scheme in ["Perfect", "BucketChaining"]:
            for jb, sc in [(256, 0), (512, 1), (1024, 0)]:
                e.set_plan(fi.RadixBits(*bits), getattr(fi.HashingScheme, scheme),
                           join_block=jb, scatter=sc)
                assert e.run(rk, rk, sk, sk) == (exp_s, exp_c)
                s32, c32 = e.run(rk32, rk32, sk32, sk32)
                assert (s32, c32) == (exp_s, exp_c)
    with pytest.raises(fi.SqlOpsError) as ex:
        e.set_plan(fi.RadixBits(11, 10))  # above the engine's first-pass size
    assert ex.value.kind == "InvalidArgument"


def test_engine_probe_before_build(fi):
    e = fi.RadixJoinEngine(1024, 1024, torch.int64, fi.RadixBits(4),
                           fi.HashingScheme.BucketChaining)
    k = torch.arange(1024, dtype=torch.int64, device="cuda")
    with pytest.raises(fi.SqlOpsError) as ex:
        e.probe(k, k)
    assert ex.value.kind == "InvalidArgument"


# --------------------------------------------------------------------------
# The join-pinning fixtures (tests/golden/make_golden.py): misses, duplicate
# build keys, negative keys and payloads, mostly empty partitions.  The CUDA
# joins are compared with the sums and counts of the reference's own compiled
# join directly, not only with the oracle.
# --------------------------------------------------------------------------
import os  # noqa: E402

_GOLDEN = os.path.join(os.path.dirname(__file__), "golden", "reference_cpu_ops.npz")
PIN_KINDS = ("misses", "duplicates", "negative", "sparse")
PIN_PERFECT = ("misses", "sparse")
# perfect hashing indexes its shared-memory table with key >> radix bits; a
# table holds at least this many keys in every join configuration here
PIN_PERFECT_SLOTS = 8192


def _pin_case(kind, name):
    g = np.load(_GOLDEN)
    pre = "join_pin_%s_%s_" % (kind, name)
    return (g[pre + "r_key"], g[pre + "r_pay"], g[pre + "s_key"], g[pre + "s_pay"],
            int(g[pre + "sum"][0]), int(g[pre + "count"][0]))


@pytest.mark.parametrize("kind", PIN_KINDS)
@pytest.mark.parametrize("ndt,tdt", DTYPES)
@pytest.mark.parametrize("scheme", ["Perfect", "BucketChaining"])
@pytest.mark.parametrize("bits", [0, 4, 6])
def test_radix_join_pinned_to_reference(fi, kind, ndt, tdt, scheme, bits):
    if scheme == "Perfect" and kind not in PIN_PERFECT:
        pytest.skip("perfect hashing needs unique non-negative build keys")
    name = "i32" if ndt == np.int32 else "i64"
    rk, rp, sk, sp, exp_s, exp_c = _pin_case(kind, name)
    if scheme == "Perfect" and (int(rk.max()) >> bits) >= PIN_PERFECT_SLOTS:
        pytest.skip("build keys index beyond the shared-memory perfect table")
    b = partition_contiguous(fi, to_dev(rk), to_dev(rp), bits)
    pr = partition_contiguous(fi, to_dev(sk), to_dev(sp), bits)
    grid, block = 37, 512
    result = torch.zeros(grid * block, dtype=torch.int64, device="cuda")
    tasks = torch.zeros(grid + 1, dtype=torch.int32, device="cuda")
    count = torch.zeros(1, dtype=torch.int64, device="cuda")
    j = fi.CudaRadixJoin(fi.RadixPass.First, fi.RadixBits(bits),
                         getattr(fi.HashingScheme, scheme), grid, block)
    j.join(b, pr, result, tasks, match_count=count)
    j.status()
    got = int(to_host(result).astype(np.int64).sum(dtype=np.int64)) & ((1 << 64) - 1)
    assert (got, int(to_host(count)[0])) == (exp_s, exp_c)


@pytest.mark.parametrize("kind", PIN_KINDS)
@pytest.mark.parametrize("ndt,tdt", DTYPES)
@pytest.mark.parametrize("bits,scheme", [((5,), "BucketChaining"),
                                         ((3, 3), "BucketChaining"),
                                         ((3, 3), "Perfect"),
                                         ((2, 4), "BucketChaining")])
def test_engine_pinned_to_reference(fi, kind, ndt, tdt, bits, scheme):
    if scheme == "Perfect" and kind not in PIN_PERFECT:
        pytest.skip("perfect hashing needs unique non-negative build keys")
    name = "i32" if ndt == np.int32 else "i64"
    rk, rp, sk, sp, exp_s, exp_c = _pin_case(kind, name)
    e = fi.RadixJoinEngine(len(rk), len(sk), tdt, fi.RadixBits(*bits),
                           getattr(fi.HashingScheme, scheme))
    s, c = e.run(to_dev(rk), to_dev(rp), to_dev(sk), to_dev(sp))
    e.status()
    assert (s & ((1 << 64) - 1), c) == (exp_s, exp_c)
