"""Shared helpers of the GPU parity tests (host-side comparisons only)."""
import numpy as np
import torch


def to_dev(a):
    return torch.from_numpy(np.ascontiguousarray(a)).cuda()


def to_host(t):
    torch.cuda.synchronize()
    return t.cpu().numpy()


def region_index(offsets, chunks, bits, padded_len, pad):
    """Slots and region ids of every non-padding slot of a partitioned
    relation (index rule of partitioned_relation.rs:510-537)."""
    offsets = np.asarray(offsets, dtype=np.int64)
    n = chunks << bits
    ends = np.empty(n, np.int64)
    ends[:-1] = offsets[1:] - pad
    ends[-1] = padded_len
    lens = ends - offsets
    assert (lens >= 0).all(), "offsets are not monotone"
    total = int(lens.sum())
    rid = np.repeat(np.arange(n), lens)
    starts = np.repeat(offsets - np.concatenate([[0], np.cumsum(lens)[:-1]]), lens)
    slots = starts + np.arange(total)
    return slots, rid


def canonical_runs(rel, slots, rid):
    """Tuples of every (chunk, partition) region, sorted inside the region."""
    t = rel[slots]
    order = np.lexsort((t[:, 1], t[:, 0], rid))
    return t[order], rid[order]


def assert_same_partitions(rel_gpu, rel_ref, offsets, chunks, bits, padded_len,
                           pad, check_padding=True, null=-1):
    slots, rid = region_index(offsets, chunks, bits, padded_len, pad)
    a, ra = canonical_runs(rel_gpu, slots, rid)
    b, rb = canonical_runs(rel_ref, slots, rid)
    np.testing.assert_array_equal(ra, rb)
    np.testing.assert_array_equal(a, b)
    if check_padding:
        mask = np.ones(padded_len, bool)
        mask[slots] = False
        pads = rel_gpu[:padded_len][mask]
        assert (pads == null).all(), "a padding slot was written"
