"""The allocation-free chunked prefix sum.

Callers that cannot allocate device memory (an engine that owns all device
memory through its own pool, a host that forbids cudaMalloc on its threads)
use fi_gpu_chunked_prefix_sum_noalloc_int64, whose scratch counters live in
a fixed array inside the library.  Its offsets must equal those of the
handle-based fi_gpu_prefix_sum_int64, call after call: the array keeps the
previous call's contents, so two different calls in a row check that each
call clears what it needs.  This file is collected last so that a run that
stops at the first failure has run every other test first.
"""
import ctypes as C

import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu

MAX_COUNTERS = 524288  # 2 MiB of u32 counters


def reference_offsets(fi, keys, chunks, bits, ignore):
    """Offsets from the existing entry point (a Chunked partitioner)."""
    rb = fi.RadixBits(ignore, bits) if ignore else fi.RadixBits(bits)
    pas = fi.RadixPass.Second if ignore else fi.RadixPass.First
    p = fi.GpuRadixPartitioner(fi.GpuHistogramAlgorithm.Chunked,
                               fi.GpuRadixPartitionAlgorithm.SSWWCv2, rb, chunks, 1024)
    o = fi.PartitionOffsets(fi.GpuHistogramAlgorithm.Chunked, chunks, bits, torch.int64)
    p.prefix_sum(pas, keys, o)
    torch.cuda.synchronize()
    return o.offsets.cpu().numpy()


def noalloc_offsets(fi, keys, chunks, bits, ignore):
    out = torch.full(((chunks << bits),), -7, dtype=torch.int64, device="cuda")
    fi._check(fi.lib().fi_gpu_chunked_prefix_sum_noalloc_int64(
        C.c_void_p(keys.data_ptr()), C.c_uint64(keys.numel()), C.c_uint32(chunks),
        C.c_uint32(bits), C.c_uint32(ignore), C.c_void_p(out.data_ptr()),
        C.c_void_p(torch.cuda.current_stream().cuda_stream)))
    torch.cuda.synchronize()
    return out.cpu().numpy()


def test_noalloc_prefix_sum_matches_partitioner(fi, oracle):
    # two calls in a row with different inputs and shapes; both use the
    # shared scratch (few chunks, so several CTAs add into each chunk's
    # counters)
    # 16 bits: two 2^15-bin range passes; 2 chunks x 18 bits: exactly the
    # array's 524288 counters, filled by the thread-block-cluster histogram
    cases = [(1_000_003, 8, 10, 0, 1), (777_777, 5, 7, 3, 2),
             (600_001, 4, 16, 0, 3), (900_007, 2, 18, 0, 4),
             (333_333, 3, 12, 5, 5)]
    for n, chunks, bits, ignore, seed in cases:
        assert (chunks << bits) <= MAX_COUNTERS
        keys = torch.from_numpy(oracle.uniform_u64_keys(n, seed)).cuda()
        got = noalloc_offsets(fi, keys, chunks, bits, ignore)
        exp = reference_offsets(fi, keys, chunks, bits, ignore)
        np.testing.assert_array_equal(got, exp)
        np.testing.assert_array_equal(
            got.astype(np.uint64),
            oracle.chunked_prefix_sum(keys.cpu().numpy(), chunks, bits, ignore))


def test_noalloc_rejects_oversized_requests(fi):
    keys = torch.zeros(16, dtype=torch.int64, device="cuda")
    out = torch.zeros(1, dtype=torch.int64, device="cuda")
    chunks, bits = 64, 14  # 64 * 16384 counters > the fixed array
    assert (chunks << bits) > MAX_COUNTERS
    rc = fi.lib().fi_gpu_chunked_prefix_sum_noalloc_int64(
        C.c_void_p(keys.data_ptr()), C.c_uint64(16), C.c_uint32(chunks),
        C.c_uint32(bits), C.c_uint32(0), C.c_void_p(out.data_ptr()),
        C.c_void_p(torch.cuda.current_stream().cuda_stream))
    assert rc == -1  # FI_ERR_INVALID_ARGUMENT
    assert b"exceeds the fixed scratch array" in fi.lib().fi_last_error()
    # more radix bits than any prefix sum supports: FI_ERR_UNSUPPORTED
    rc = fi.lib().fi_gpu_chunked_prefix_sum_noalloc_int64(
        C.c_void_p(keys.data_ptr()), C.c_uint64(16), C.c_uint32(1),
        C.c_uint32(19), C.c_uint32(0), C.c_void_p(out.data_ptr()),
        C.c_void_p(torch.cuda.current_stream().cuda_stream))
    assert rc == -6
