"""The reference's own GPU kernels, compiled for sm_100a from its sources and
launched as its Rust host code launches them (baseline/refgpu), against this
repository's kernels on the same inputs:

* gpu_chunked_prefix_sum_*: offsets identical element by element;
* the NC and LASWWC scatters: identical per-(chunk, partition) multisets;
* gpu_radix_join_assign_tasks + gpu_join_aggregate_smem_{perfect,chaining}_*:
  the same sum as this repository's join and as the golden sums of the
  reference's compiled CPU join (tests/golden/make_golden.py).

Each reference launch is checked on the host first, so its device asserts
cannot fire; requests the reference kernels cannot take are refused before
any launch (checked here too)."""
import os
import sys

import numpy as np
import pytest
import torch

from _helpers import assert_same_partitions, to_dev, to_host

sys.path.insert(0, os.path.join(os.path.dirname(os.path.dirname(
    os.path.abspath(__file__))), "baseline", "refgpu"))
import refgpu  # noqa: E402

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not refgpu.available(),
                                 reason="reference GPU kernels not built")]

DTYPES = [(np.int32, torch.int32), (np.int64, torch.int64)]
GOLDEN = os.path.join(os.path.dirname(__file__), "golden", "reference_cpu_ops.npz")


def our_chunked(fi, dk, dp, chunks, bits, algo="SSWWCv2"):
    p = fi.GpuRadixPartitioner(fi.GpuHistogramAlgorithm.Chunked,
                               getattr(fi.GpuRadixPartitionAlgorithm, algo),
                               fi.RadixBits(bits), chunks, 1024)
    o = fi.PartitionOffsets(fi.GpuHistogramAlgorithm.Chunked, chunks, bits, dk.dtype)
    rel = fi.PartitionedRelation(dk.numel(), fi.GpuHistogramAlgorithm.Chunked, bits,
                                 chunks, dk.dtype, fill=-1)
    p.prefix_sum(fi.RadixPass.First, dk, o)
    p.partition(fi.RadixPass.First, dk, dp, o, rel)
    p.status()
    return rel


@pytest.mark.parametrize("ndt,tdt", DTYPES)
@pytest.mark.parametrize("n,chunks,bits", [(1000, 1, 0), (100003, 7, 6),
                                           (1 << 20, 148, 10), (777777, 16, 14),
                                           (300000, 3, 15)])
def test_reference_prefix_sum_identical(fi, oracle, ndt, tdt, n, chunks, bits):
    keys = oracle.uniform_u64_keys(n, 17).astype(ndt)
    dk = to_dev(keys)
    ref = to_host(refgpu.chunked_prefix_sum(dk, chunks, bits)).astype(np.uint64)
    p = fi.GpuRadixPartitioner(fi.GpuHistogramAlgorithm.Chunked,
                               fi.GpuRadixPartitionAlgorithm.SSWWCv2,
                               fi.RadixBits(bits), chunks, 1024)
    o = fi.PartitionOffsets(fi.GpuHistogramAlgorithm.Chunked, chunks, bits, tdt)
    p.prefix_sum(fi.RadixPass.First, dk, o)
    ours = to_host(o.offsets).astype(np.uint64)
    np.testing.assert_array_equal(ours, ref)
    np.testing.assert_array_equal(ref, oracle.chunked_prefix_sum(keys, chunks, bits))


@pytest.mark.parametrize("ndt,tdt", DTYPES)
@pytest.mark.parametrize("variant", [refgpu.NC, refgpu.LASWWC])
@pytest.mark.parametrize("n,chunks,bits", [(5000, 1, 3), (1 << 20, 148, 9),
                                           (654321, 10, 12), (1 << 19, 8, 14)])
def test_reference_scatter_same_partitions(fi, oracle, ndt, tdt, variant, n,
                                           chunks, bits):
    keys = oracle.uniform_u64_keys(n, 23).astype(ndt)
    pays = oracle.uniform_u64_keys(n, 24).astype(ndt)
    dk, dp = to_dev(keys), to_dev(pays)
    off = refgpu.chunked_prefix_sum(dk, chunks, bits)
    pad = refgpu.padding_len(tdt)
    padded = n + (chunks << bits) * pad
    rel = torch.full((padded, 2), -1, dtype=tdt, device="cuda")
    part = refgpu.Partition(variant, dk, dp, chunks, bits, off, rel)
    part.launch()
    ref_rel = to_host(rel)
    ours = our_chunked(fi, dk, dp, chunks, bits)
    off_h = to_host(off).astype(np.uint64)
    np.testing.assert_array_equal(to_host(ours.offsets).astype(np.uint64), off_h)
    assert_same_partitions(to_host(ours.relation)[:padded], ref_rel, off_h, chunks,
                           bits, padded, pad)
    # the reference's scatter leaves the padding as it found it, too
    assert_same_partitions(ref_rel, ref_rel, off_h, chunks, bits, padded, pad)


def test_reference_scatter_refuses_foreign_offsets(fi, oracle):
    """Offsets that are not the prefix sum of the keys are refused before
    any launch (they could send tuples outside their regions)."""
    n, chunks, bits = 4096, 2, 4
    dk = to_dev(oracle.uniform_u64_keys(n, 1))
    off = refgpu.chunked_prefix_sum(dk, chunks, bits)
    off[3] += 1
    rel = torch.full((n + (chunks << bits) * 8, 2), -1, dtype=torch.int64, device="cuda")
    with pytest.raises(refgpu.RefGpuError):
        refgpu.Partition(refgpu.NC, dk, dk, chunks, bits, off, rel)


def contiguous(fi, keys, pays, bits):
    p = fi.GpuRadixPartitioner(fi.GpuHistogramAlgorithm.Chunked,
                               fi.GpuRadixPartitionAlgorithm.NC, fi.RadixBits(bits), 1,
                               1024)
    o = fi.PartitionOffsets(fi.GpuHistogramAlgorithm.Chunked, 1, bits, keys.dtype)
    rel = fi.PartitionedRelation(keys.numel(), fi.GpuHistogramAlgorithm.Chunked, bits, 1,
                                 keys.dtype, fill=-1)
    p.prefix_sum(fi.RadixPass.First, keys, o)
    p.partition(fi.RadixPass.First, keys, pays, o, rel)
    p.status()
    return rel


def both_joins(fi, scheme, rk, rp, sk, sp, bits, grid=148, block=512):
    """(reference join sum, this repository's join sum) on the same relations."""
    b = contiguous(fi, to_dev(rk), to_dev(rp), bits)
    pr = contiguous(fi, to_dev(sk), to_dev(sp), bits)
    j = refgpu.Join(scheme, b.relation, b.offsets, b.padded_len(), pr.relation,
                    pr.offsets, pr.padded_len(), bits, bits, grid, block)
    j.launch()
    ref = j.sum()
    result = torch.zeros(grid * block, dtype=torch.int64, device="cuda")
    tasks = torch.zeros(grid + 1, dtype=torch.int32, device="cuda")
    ours = fi.CudaRadixJoin(fi.RadixPass.First, fi.RadixBits(bits),
                            fi.HashingScheme.Perfect if scheme == refgpu.PERFECT
                            else fi.HashingScheme.BucketChaining, grid, block)
    ours.join(b, pr, result, tasks)
    ours.status()
    # identical task split (radix_join.cu:58-98)
    np.testing.assert_array_equal(to_host(tasks), to_host(j.tasks))
    return ref, int(to_host(result).sum()) & ((1 << 64) - 1)


@pytest.mark.parametrize("kind", ["misses", "duplicates", "negative", "sparse"])
@pytest.mark.parametrize("ndt,tdt", DTYPES)
@pytest.mark.parametrize("scheme", [refgpu.PERFECT, refgpu.CHAINING])
@pytest.mark.parametrize("bits", [0, 4])
def test_reference_join_pinned(fi, kind, ndt, tdt, scheme, bits):
    g = np.load(GOLDEN)
    pre = "join_pin_%s_%s_" % (kind, "i32" if ndt == np.int32 else "i64")
    rk, rp, sk, sp = (g[pre + x] for x in ("r_key", "r_pay", "s_key", "s_pay"))
    exp = int(g[pre + "sum"][0])
    if scheme == refgpu.PERFECT:
        if kind in ("duplicates", "negative"):
            pytest.skip("perfect hashing needs unique non-negative build keys")
        # the reference's perfect table: 227 KB of shared memory / 2K - 1
        slots = 29055 if ndt == np.int32 else 14527
        if max(int(rk.max()), int(sk.max())) >> bits >= slots:
            # the reference would index shared memory out of bounds: refused
            with pytest.raises(refgpu.RefGpuError) as e:
                both_joins(fi, scheme, rk, rp, sk, sp, bits)
            assert e.value.code == -7
            return
    ref, ours = both_joins(fi, scheme, rk, rp, sk, sp, bits)
    assert ref == ours == exp


@pytest.mark.parametrize("ndt,tdt", DTYPES)
@pytest.mark.parametrize("scheme", [refgpu.PERFECT, refgpu.CHAINING])
def test_reference_join_known_answer(fi, oracle, ndt, tdt, scheme):
    """Unique primary keys 1..N, uniform foreign keys, payload = row + 1:
    SUM = N (N + 1) / 2 (test_cuda_radix_join.rs:179-182), 6 radix bits so
    a partition holds ~16K tuples (within both reference tables)."""
    n = 1 << 20
    rk = oracle.primary_keys(n, 3, ndt)
    sk = oracle.uniform_foreign_keys(n, n, 4, ndt)
    pay = np.arange(1, n + 1, dtype=ndt)
    # int64: the chaining table holds 12458 tuples and the perfect table
    # indexes key >> bits below 14527, so 7 bits; int32: 22425 and 29055
    bits = 7 if ndt == np.int64 else 6
    ref, ours = both_joins(fi, scheme, rk, pay, sk, pay, bits)
    assert ref == ours == (n * (n + 1) // 2) & ((1 << 64) - 1)
