"""The CPU radix partitioner (the hybrid join's first pass; the reference's
CpuRadixPartitioner) against the oracle and the reference's own compiled CPU
partitioner: identical Chunked offsets, and relations identical slot by slot
(each chunk is scattered in input order, so even the order within a
partition matches the reference's sequential scatter)."""
import numpy as np
import pytest


@pytest.mark.parametrize("dtype", [np.int32, np.int64])
@pytest.mark.parametrize("bits", [0, 1, 6, 9, 12])
@pytest.mark.parametrize("chunks", [1, 3, 8])
@pytest.mark.parametrize("algo", ["NC", "SWWC"])
def test_cpu_partition_matches_oracle(fi, oracle, dtype, bits, chunks, algo):
    n = 100_003
    keys = oracle.uniform_u64_keys(n, 5 + bits).astype(dtype)
    pays = oracle.primary_keys(n, 6, dtype)
    rel, off = fi.cpu_radix_partition(keys, pays, bits, chunks,
                                      getattr(fi.CpuRadixPartitionAlgorithm, algo))
    exp_off = oracle.chunked_prefix_sum(keys, chunks, bits)
    assert np.array_equal(off, exp_off)
    exp = oracle.chunked_radix_partition(keys, pays, exp_off, chunks, bits, 0, len(rel))
    assert np.array_equal(rel, exp)


@pytest.mark.parametrize("dtype", [np.int32, np.int64])
def test_cpu_partition_matches_reference(fi, oracle, dtype):
    if not oracle.ref_available():
        pytest.skip("reference CPU partitioner not built")
    n, bits, chunks = 77_777, 7, 5
    keys = oracle.uniform_u64_keys(n, 9).astype(dtype)
    pays = oracle.uniform_u64_keys(n, 10).astype(dtype)
    rel, off = fi.cpu_radix_partition(keys, pays, bits, chunks,
                                      fi.CpuRadixPartitionAlgorithm.NC)
    assert np.array_equal(off, oracle.ref_chunked_prefix_sum(keys, chunks, bits))
    ref_rel = oracle.ref_chunked_radix_partition(keys, pays, off, chunks, bits)
    assert np.array_equal(rel, ref_rel)


def test_cpu_second_pass_bits_and_empty(fi, oracle):
    """ignore_bits selects the second-pass digit; empty inputs work."""
    n, chunks = 50_000, 4
    keys = oracle.uniform_u64_keys(n, 3)
    pays = keys.copy()
    F, pad = 1 << 5, fi.padding_len(fi.torch.int64)
    off = np.zeros(chunks * F, np.uint64)
    rel = np.full((n + chunks * F * pad, 2), -1, np.int64)
    p = fi.CpuRadixPartitioner(fi.CpuHistogramAlgorithm.Chunked,
                               fi.CpuRadixPartitionAlgorithm.SWWC, 5)
    for c in range(chunks):
        o = off[c * F:(c + 1) * F]
        p.prefix_sum(keys, c, chunks, o, ignore_bits=9)
        p.partition(keys, pays, c, chunks, o, rel, ignore_bits=9)
    assert np.array_equal(off, oracle.chunked_prefix_sum(keys, chunks, 5, ignore=9))
    exp = oracle.chunked_radix_partition(keys, pays, off, chunks, 5, 9, len(rel))
    assert np.array_equal(rel, exp)
    e = np.zeros(0, np.int64)
    r0, o0 = fi.cpu_radix_partition(e, e, 4, 2)
    assert r0.shape == (2 * 16 * pad, 2) and (r0 == -1).all()


def test_cpu_partition_errors(fi, oracle):
    with pytest.raises(fi.SqlOpsError):
        fi.CpuRadixPartitioner(fi.CpuHistogramAlgorithm.Chunked,
                               fi.CpuRadixPartitionAlgorithm.NC, 17)
    p = fi.CpuRadixPartitioner(fi.CpuHistogramAlgorithm.Chunked,
                               fi.CpuRadixPartitionAlgorithm.NC, 4)
    keys = np.arange(1000, dtype=np.int64)
    off = np.zeros(16, np.uint64)
    with pytest.raises(fi.SqlOpsError) as ex:
        p.prefix_sum(keys, 3, 3, off)
    assert ex.value.kind == "InvalidArgument"
    p.prefix_sum(keys, 0, 1, off)
    small = np.zeros((100, 2), np.int64)  # far too short for 1000 tuples
    with pytest.raises(fi.SqlOpsError) as ex:
        p.partition(keys, keys, 0, 1, off, small)
    assert ex.value.kind == "Capacity"


@pytest.mark.parametrize("dtype", [np.int32, np.int64])
def test_cpu_swwc_unaligned_relation(fi, oracle, dtype):
    """A relation whose base is not aligned to the tuple size takes the
    plain-copy write-combining path; its slots equal the oracle's too, as do
    those of the line-aligned streaming path on an aligned relation."""
    n, bits, chunks = 50_001, 6, 3
    keys = oracle.uniform_u64_keys(n, 17).astype(dtype)
    pays = oracle.uniform_u64_keys(n, 18).astype(dtype)
    F, pad = 1 << bits, fi.padding_len(fi.torch.int32 if dtype == np.int32 else fi.torch.int64)
    tsz = 2 * np.dtype(dtype).itemsize
    total = n + chunks * F * pad
    raw = np.zeros(total * tsz + 64, np.uint8)
    base = raw.ctypes.data
    skew = (tsz // 2 - base % tsz) % tsz or tsz // 2  # element-aligned, not tuple-aligned
    rel = raw[skew:skew + total * tsz].view(dtype).reshape(total, 2)
    assert rel.ctypes.data % tsz != 0 and rel.ctypes.data % np.dtype(dtype).itemsize == 0
    rel[:] = -1
    off = np.zeros(chunks * F, np.uint64)
    p = fi.CpuRadixPartitioner(fi.CpuHistogramAlgorithm.Chunked,
                               fi.CpuRadixPartitionAlgorithm.SWWC, bits)
    for c in range(chunks):
        o = off[c * F:(c + 1) * F]
        p.prefix_sum(keys, c, chunks, o)
        p.partition(keys, pays, c, chunks, o, rel)
    exp = oracle.chunked_radix_partition(keys, pays, off, chunks, bits, 0, total)
    assert np.array_equal(rel, exp)
