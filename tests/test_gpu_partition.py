"""GPU parity of the radix partitioner against the oracle, through the C ABI.

Follows the reference's test matrix (sql-ops/tests/test_gpu_radix_partition.rs:
458-1550): sizes 100, 10^6 and multi-million tuples, bits 0..15, Chunked and
Contiguous histograms, every partition algorithm, one- and two-pass flows,
fewer tuples than partitions.  Offsets must be identical; every
(chunk, partition) region must hold the oracle's tuple multiset; padding
slots must stay untouched."""
import numpy as np
import pytest
import torch

from _helpers import assert_same_partitions, to_dev, to_host

pytestmark = pytest.mark.gpu

DTYPES = [(np.int32, torch.int32), (np.int64, torch.int64)]


def gen(oracle, n, dt, seed, kind="pk"):
    if kind == "pk":
        k = oracle.primary_keys(n, seed, dt, base=0)
    elif kind == "u64":
        k = oracle.uniform_u64_keys(n, seed).astype(dt)
    else:
        k = oracle.zipf_foreign_keys(n, max(n, 1), 1.5, seed, seed + 1, dt)
    p = oracle.uniform_foreign_keys(n, 1 << 20, seed + 7, dt)
    return k, p


CHUNKED_CASES = [(100, 1, 0), (100, 4, 2), (1000, 80, 9), (10**6, 8, 6),
                 (10**6, 10, 10), (1 << 20, 148, 12), (1 << 20, 148, 14),
                 (1 << 18, 3, 15), (8 * 2**20, 148, 9),
                 # fanouts above one CTA's shared-memory histogram (bin ranges)
                 (1000, 3, 17), (1 << 20, 16, 16), (1 << 19, 4, 18),
                 (1 << 20, 148, 16)]


@pytest.mark.parametrize("ndt,tdt", DTYPES)
@pytest.mark.parametrize("n,grid,bits", CHUNKED_CASES)
def test_chunked_prefix_sum(fi, oracle, ndt, tdt, n, grid, bits):
    keys, _ = gen(oracle, n, ndt, 1)
    p = fi.GpuRadixPartitioner(fi.GpuHistogramAlgorithm.Chunked,
                               fi.GpuRadixPartitionAlgorithm.SSWWCv2,
                               fi.RadixBits(bits), grid, 1024)
    o = fi.PartitionOffsets(fi.GpuHistogramAlgorithm.Chunked, grid, bits, tdt)
    p.prefix_sum(fi.RadixPass.First, to_dev(keys), o)
    p.status()
    exp = oracle.chunked_prefix_sum(keys, grid, bits)
    np.testing.assert_array_equal(to_host(o.offsets).astype(np.uint64), exp)
    assert o.len() == n


@pytest.mark.parametrize("ndt,tdt", DTYPES)
@pytest.mark.parametrize("n,grid,bits", [(100, 1, 0), (1000, 80, 9),
                                         (10**6, 10, 10), (1 << 20, 148, 12),
                                         (1 << 18, 7, 15), (1 << 20, 5, 16),
                                         (1 << 19, 3, 18)])
def test_contiguous_prefix_sum(fi, oracle, ndt, tdt, n, grid, bits):
    keys, _ = gen(oracle, n, ndt, 2)
    p = fi.GpuRadixPartitioner(fi.GpuHistogramAlgorithm.Contiguous,
                               fi.GpuRadixPartitionAlgorithm.SSWWCv2,
                               fi.RadixBits(bits), grid, 1024)
    o = fi.PartitionOffsets(fi.GpuHistogramAlgorithm.Contiguous, grid, bits, tdt)
    p.prefix_sum(fi.RadixPass.First, to_dev(keys), o)
    p.status()
    off, loc = oracle.contiguous_prefix_sum(keys, grid, bits)
    np.testing.assert_array_equal(to_host(o.offsets).astype(np.uint64), off)
    np.testing.assert_array_equal(to_host(o.local_offsets).astype(np.uint64), loc)


def test_prefix_sum_second_pass_ignore_bits(fi, oracle):
    keys, _ = gen(oracle, 300000, np.int64, 3)
    bits = fi.RadixBits(5, 7)
    p = fi.GpuRadixPartitioner(fi.GpuHistogramAlgorithm.Chunked,
                               fi.GpuRadixPartitionAlgorithm.NC, bits, 9, 512)
    o = fi.PartitionOffsets(fi.GpuHistogramAlgorithm.Chunked, 9, 7, torch.int64)
    p.prefix_sum(fi.RadixPass.Second, to_dev(keys), o)
    exp = oracle.chunked_prefix_sum(keys, 9, 7, ignore=5)
    np.testing.assert_array_equal(to_host(o.offsets).astype(np.uint64), exp)


def run_partition(fi, oracle, keys, pays, tdt, hist, algo, grid, bits,
                  radix_bits=None, radix_pass=None):
    radix_bits = radix_bits or fi.RadixBits(bits)
    radix_pass = fi.RadixPass.First if radix_pass is None else radix_pass
    n = len(keys)
    p = fi.GpuRadixPartitioner(hist, algo, radix_bits, grid, 1024)
    o = fi.PartitionOffsets(hist, grid, bits, tdt)
    rel = fi.PartitionedRelation(n, hist, bits, grid, tdt, fill=-1)
    dk, dp = to_dev(keys), to_dev(pays)
    p.prefix_sum(radix_pass, dk, o)
    p.partition(radix_pass, dk, dp, o, rel)
    p.status()
    return rel


ALGOS = ["NC", "SSWWCv2", "SSWWCv2G", "HSSWWCv4", "LASWWC"]


@pytest.mark.parametrize("ndt,tdt", DTYPES)
@pytest.mark.parametrize("algo", ALGOS)
@pytest.mark.parametrize("hist", ["Chunked", "Contiguous"])
@pytest.mark.parametrize("n,grid,bits", [(100, 1, 0), (100, 4, 2), (1000, 80, 9),
                                         (10**6, 10, 6), (10**6, 8, 10),
                                         (1 << 20, 148, 12), (1 << 19, 16, 14)])
def test_partition(fi, oracle, ndt, tdt, algo, hist, n, grid, bits):
    keys, pays = gen(oracle, n, ndt, 4)
    H = getattr(fi.GpuHistogramAlgorithm, hist)
    rel = run_partition(fi, oracle, keys, pays, tdt, H,
                        getattr(fi.GpuRadixPartitionAlgorithm, algo), grid, bits)
    pad = oracle.padding_len(ndt)
    if hist == "Chunked":
        off = oracle.chunked_prefix_sum(keys, grid, bits)
        cursors, chunks = off, grid
    else:
        off, loc = oracle.contiguous_prefix_sum(keys, grid, bits)
        cursors, chunks = loc, 1
    got_off = to_host(rel.offsets).astype(np.uint64)
    np.testing.assert_array_equal(got_off, off)
    padded = rel.padded_len()
    ref = oracle.chunked_radix_partition(keys, pays, cursors, grid, bits, 0, padded)
    got = to_host(rel.relation)[:padded]
    assert_same_partitions(got, ref, off, chunks, bits, padded, pad)
    # every tuple exactly once (tuple_loss_or_duplicates,
    # sql-ops/tests/radix_partition/mod.rs:33-87)
    valid = got[got[:, 0] != -1]
    assert len(valid) == n
    assert len(np.unique(valid[:, 0])) == n


@pytest.mark.parametrize("ndt,tdt", DTYPES)
@pytest.mark.parametrize("bits", [5, 11, 13])
def test_partition_unaligned_columns(fi, oracle, ndt, tdt, bits):
    """Columns that start off a 16-byte boundary take the register-fed scatter
    instead of the TMA-fed one; the result must be the same."""
    n, grid = 300001, 20
    keys, pays = gen(oracle, n, ndt, 12)
    dk = torch.empty(n + 1, dtype=tdt, device="cuda")[1:]
    dp = torch.empty(n + 1, dtype=tdt, device="cuda")[1:]
    dk.copy_(to_dev(keys))
    dp.copy_(to_dev(pays))
    p = fi.GpuRadixPartitioner(fi.GpuHistogramAlgorithm.Chunked,
                               fi.GpuRadixPartitionAlgorithm.SSWWCv2,
                               fi.RadixBits(bits), grid, 1024)
    o = fi.PartitionOffsets(fi.GpuHistogramAlgorithm.Chunked, grid, bits, tdt)
    rel = fi.PartitionedRelation(n, fi.GpuHistogramAlgorithm.Chunked, bits, grid, tdt,
                                 fill=-1)
    p.prefix_sum(fi.RadixPass.First, dk, o)
    p.partition(fi.RadixPass.First, dk, dp, o, rel)
    p.status()
    off = oracle.chunked_prefix_sum(keys, grid, bits)
    padded = rel.padded_len()
    ref = oracle.chunked_radix_partition(keys, pays, off, grid, bits, 0, padded)
    assert_same_partitions(to_host(rel.relation)[:padded], ref, off, grid, bits,
                           padded, oracle.padding_len(ndt))


@pytest.mark.parametrize("ndt,tdt", DTYPES)
@pytest.mark.parametrize("hist,bits,grid", [("Chunked", 15, 16), ("Chunked", 16, 16),
                                            ("Chunked", 17, 5), ("Chunked", 18, 4),
                                            ("Contiguous", 16, 8),
                                            ("Contiguous", 18, 3)])
def test_partition_hierarchical(fi, oracle, ndt, tdt, hist, bits, grid):
    """Fanouts above the tile scatter (2^15..2^18, the partition sweep's
    "hierarchical" fanouts of the reference) use the wide scatter."""
    n = 1 << 20
    keys, pays = gen(oracle, n, ndt, 5, kind="u64")
    H = getattr(fi.GpuHistogramAlgorithm, hist)
    rel = run_partition(fi, oracle, keys, pays, tdt, H,
                        fi.GpuRadixPartitionAlgorithm.HSSWWCv4, grid, bits)
    if hist == "Chunked":
        off = oracle.chunked_prefix_sum(keys, grid, bits)
        cursors, chunks = off, grid
    else:
        off, cursors = oracle.contiguous_prefix_sum(keys, grid, bits)
        chunks = 1
    np.testing.assert_array_equal(to_host(rel.offsets).astype(np.uint64), off)
    padded = rel.padded_len()
    ref = oracle.chunked_radix_partition(keys, pays, cursors, grid, bits, 0, padded)
    got = to_host(rel.relation)[:padded]
    assert_same_partitions(got, ref, off, chunks, bits, padded,
                           oracle.padding_len(ndt))
    assert (got[:, 0] != -1).sum() == n


@pytest.mark.parametrize("ndt,tdt", DTYPES)
@pytest.mark.parametrize("hist", ["Chunked", "Contiguous"])
@pytest.mark.parametrize("n,grid,bits,kind", [(5000, 37, 12, "u64"),
                                              (20000, 148, 13, "u64"),
                                              (1 << 20, 148, 12, "zipf"),
                                              (300001, 7, 18, "zipf"),
                                              (1 << 20, 148, 16, "u64"),
                                              (999999, 64, 17, "u64"),
                                              (3000, 200, 12, "u64")])
def test_partition_high_fanout(fi, oracle, ndt, tdt, hist, n, grid, bits, kind):
    """The two-level scatter above 11 bits, whose level-1 layout comes from
    the final cursors: tiles that span several small chunks (or chunks of
    length 0), Zipf-skewed keys filling a few buckets, Contiguous per-block
    cursors, up to 2^18 partitions."""
    keys, pays = gen(oracle, n, ndt, 9, kind=kind)
    H = getattr(fi.GpuHistogramAlgorithm, hist)
    rel = run_partition(fi, oracle, keys, pays, tdt, H,
                        fi.GpuRadixPartitionAlgorithm.SSWWCv2, grid, bits)
    if hist == "Chunked":
        off = oracle.chunked_prefix_sum(keys, grid, bits)
        cursors, chunks = off, grid
    else:
        off, cursors = oracle.contiguous_prefix_sum(keys, grid, bits)
        chunks = 1
    np.testing.assert_array_equal(to_host(rel.offsets).astype(np.uint64), off)
    padded = rel.padded_len()
    ref = oracle.chunked_radix_partition(keys, pays, cursors, grid, bits, 0, padded)
    assert_same_partitions(to_host(rel.relation)[:padded], ref, off, chunks, bits,
                           padded, oracle.padding_len(ndt))


@pytest.mark.parametrize("algo", ["NC", "SSWWCv2"])
def test_partition_zipf_skew(fi, oracle, algo):
    n, grid, bits = 1 << 20, 37, 9
    keys, pays = gen(oracle, n, np.int64, 6, kind="zipf")
    rel = run_partition(fi, oracle, keys, pays, torch.int64,
                        fi.GpuHistogramAlgorithm.Chunked,
                        getattr(fi.GpuRadixPartitionAlgorithm, algo), grid, bits)
    off = oracle.chunked_prefix_sum(keys, grid, bits)
    padded = rel.padded_len()
    ref = oracle.chunked_radix_partition(keys, pays, off, grid, bits, 0, padded)
    assert_same_partitions(to_host(rel.relation)[:padded], ref, off, grid, bits,
                           padded, 8)


def test_partition_uniform_64bit_keys(fi, oracle):
    """Config-2 shape: uniform 64-bit keys (negative as int64)."""
    n, grid, bits = 1 << 21, 148, 10
    keys, pays = gen(oracle, n, np.int64, 7, kind="u64")
    rel = run_partition(fi, oracle, keys, pays, torch.int64,
                        fi.GpuHistogramAlgorithm.Chunked,
                        fi.GpuRadixPartitionAlgorithm.SSWWCv2, grid, bits)
    off = oracle.chunked_prefix_sum(keys, grid, bits)
    padded = rel.padded_len()
    ref = oracle.chunked_radix_partition(keys, pays, off, grid, bits, 0, padded)
    assert_same_partitions(to_host(rel.relation)[:padded], ref, off, grid, bits,
                           padded, 8, check_padding=False)


@pytest.mark.parametrize("ndt,tdt", DTYPES)
@pytest.mark.parametrize("b1,b2", [(0, 0), (2, 2), (6, 6), (10, 10), (2, 16)])
def test_two_pass_transform_and_partition(fi, oracle, ndt, tdt, b1, b2):
    """Reference two-pass flow (test_gpu_radix_partition.rs two_pass_*):
    pass 1 Chunked, then per first-pass partition prefix_sum_and_transform and
    a Contiguous second pass."""
    n, grid1, grid2 = 200000, 10, 8
    keys, pays = gen(oracle, n, ndt, 8)
    bits = fi.RadixBits(b1, b2)
    rel1 = run_partition(fi, oracle, keys, pays, tdt, fi.GpuHistogramAlgorithm.Chunked,
                         fi.GpuRadixPartitionAlgorithm.SSWWCv2, grid1, b1,
                         radix_bits=bits)
    host_rel1 = to_host(rel1.relation)
    host_off1 = to_host(rel1.offsets).astype(np.uint64)
    pad = oracle.padding_len(ndt)
    p2 = fi.GpuRadixPartitioner(fi.GpuHistogramAlgorithm.Contiguous,
                                fi.GpuRadixPartitionAlgorithm.SSWWCv2, bits, grid2,
                                1024)
    F1 = 1 << b1
    for pid in sorted(set([0, F1 // 2, F1 - 1])):
        plen = rel1.partition_len(pid)
        ck = torch.empty(max(plen, 1), dtype=tdt, device="cuda")[:plen]
        cp = torch.empty(max(plen, 1), dtype=tdt, device="cuda")[:plen]
        o2 = fi.PartitionOffsets(fi.GpuHistogramAlgorithm.Contiguous, grid2, b2, tdt)
        p2.prefix_sum_and_transform(fi.RadixPass.Second, pid, rel1, ck, cp, o2)
        ek, ep, eoff, eloc = oracle.prefix_sum_and_transform(
            pid, host_rel1[:rel1.padded_len()], host_off1, grid1, b1, pad,
            grid2, b2, b1)
        np.testing.assert_array_equal(to_host(ck), ek)
        np.testing.assert_array_equal(to_host(cp), ep)
        np.testing.assert_array_equal(to_host(o2.offsets).astype(np.uint64), eoff)
        np.testing.assert_array_equal(to_host(o2.local_offsets).astype(np.uint64), eloc)
        rel2 = fi.PartitionedRelation(plen, fi.GpuHistogramAlgorithm.Contiguous, b2,
                                      grid2, tdt, fill=-1)
        p2.partition(fi.RadixPass.Second, ck, cp, o2, rel2)
        p2.status()
        padded = rel2.padded_len()
        ref = oracle.chunked_radix_partition(ek, ep, eloc, grid2, b2, b1, padded)
        assert_same_partitions(to_host(rel2.relation)[:padded], ref, eoff, 1, b2,
                               padded, pad)


@pytest.mark.parametrize("ndt,tdt", DTYPES)
def test_prefix_sum_and_copy_with_payload(fi, oracle, ndt, tdt):
    n, grid, bits = 300001, 12, 8
    keys, pays = gen(oracle, n, ndt, 9)
    p = fi.GpuRadixPartitioner(fi.GpuHistogramAlgorithm.Contiguous,
                               fi.GpuRadixPartitionAlgorithm.SSWWCv2,
                               fi.RadixBits(bits), grid, 1024)
    o = fi.PartitionOffsets(fi.GpuHistogramAlgorithm.Contiguous, grid, bits, tdt)
    dk = torch.empty(n, dtype=tdt, device="cuda")
    dp = torch.empty(n, dtype=tdt, device="cuda")
    p.prefix_sum_and_copy_with_payload(fi.RadixPass.First, to_dev(keys), to_dev(pays),
                                       dk, dp, o)
    np.testing.assert_array_equal(to_host(dk), keys)
    np.testing.assert_array_equal(to_host(dp), pays)
    off, loc = oracle.contiguous_prefix_sum(keys, grid, bits)
    np.testing.assert_array_equal(to_host(o.offsets).astype(np.uint64), off)
    np.testing.assert_array_equal(to_host(o.local_offsets).astype(np.uint64), loc)


def test_validation_errors(fi):
    """Argument checks of gpu_radix_partition.rs:561-1080, no launch."""
    p = fi.GpuRadixPartitioner(fi.GpuHistogramAlgorithm.Chunked,
                               fi.GpuRadixPartitionAlgorithm.NC,
                               fi.RadixBits(4), 8, 256)
    keys = torch.zeros(100, dtype=torch.int64, device="cuda")
    bad = fi.PartitionOffsets(fi.GpuHistogramAlgorithm.Chunked, 4, 4, torch.int64)
    with pytest.raises(fi.SqlOpsError, match="mismatching number of chunks"):
        p.prefix_sum(fi.RadixPass.First, keys, bad)
    wrong_bits = fi.PartitionOffsets(fi.GpuHistogramAlgorithm.Chunked, 8, 5, torch.int64)
    with pytest.raises(fi.SqlOpsError, match="mismatching radix bits"):
        p.prefix_sum(fi.RadixPass.First, keys, wrong_bits)
    with pytest.raises(fi.SqlOpsError, match="pass is not specified"):
        p.prefix_sum(fi.RadixPass.Second, keys,
                     fi.PartitionOffsets(fi.GpuHistogramAlgorithm.Chunked, 8, 4,
                                         torch.int64))
    o = fi.PartitionOffsets(fi.GpuHistogramAlgorithm.Chunked, 8, 4, torch.int64)
    rel = fi.PartitionedRelation(100, fi.GpuHistogramAlgorithm.Chunked, 4, 8, torch.int64)
    with pytest.raises(fi.SqlOpsError, match="has no length"):
        p.partition(fi.RadixPass.First, keys, keys, o, rel)
    p.prefix_sum(fi.RadixPass.First, keys, o)
    rel_bad = fi.PartitionedRelation(99, fi.GpuHistogramAlgorithm.Chunked, 4, 8,
                                     torch.int64)
    with pytest.raises(fi.SqlOpsError, match="mismatching lengths"):
        p.partition(fi.RadixPass.First, keys, keys, o, rel_bad)
    pc = fi.GpuRadixPartitioner(fi.GpuHistogramAlgorithm.Chunked,
                                fi.GpuRadixPartitionAlgorithm.NC, fi.RadixBits(4), 8, 256)
    with pytest.raises(fi.SqlOpsError, match="try using Contiguous"):
        pc.prefix_sum_and_copy_with_payload(fi.RadixPass.First, keys, keys, keys.clone(),
                                            keys.clone(), o)
