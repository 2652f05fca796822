"""Out-of-core join: the first radix pass streamed from host memory.

The relations stay in (pinned) host memory and the first pass copies them
block by block over the host link.  The result must equal the in-HBM engine
and the CPU radix join on the same seeded inputs, for any block size,
including a ragged last block and a single block.
"""
import numpy as np
import pytest
import torch

from _helpers import to_dev

pytestmark = pytest.mark.gpu

DTYPES = [(np.int32, torch.int32), (np.int64, torch.int64)]


def pinned(a):
    return torch.from_numpy(np.ascontiguousarray(a)).pin_memory()


@pytest.mark.parametrize("ndt,tdt", DTYPES)
@pytest.mark.parametrize("bits,block", [((6, 6), 1 << 18), ((9, 9), 3 << 16),
                                        ((9, 9), 0), ((4, 10), 1 << 20)])
def test_streamed_matches_oracle(fi, oracle, ndt, tdt, bits, block):
    n_b, n_p = 1 << 21, (1 << 21) + 12345
    r_key = oracle.primary_keys(n_b, 51, ndt)
    r_pay = oracle.uniform_foreign_keys(n_b, 1 << 30, 53, ndt)
    s_key = oracle.uniform_foreign_keys(n_p, n_b, 52, ndt)
    s_pay = oracle.uniform_foreign_keys(n_p, 1 << 30, 54, ndt)
    e = fi.RadixJoinEngine(n_b, n_p, tdt, fi.RadixBits(*bits),
                           fi.HashingScheme.BucketChaining)
    got = e.run_streamed(pinned(r_key), pinned(r_pay), pinned(s_key),
                         pinned(s_pay), block_tuples=block)
    e.status()
    dev = e.run(to_dev(r_key), to_dev(r_pay), to_dev(s_key), to_dev(s_pay))
    exp_s, exp_c, _, _ = oracle.cpu_radix_join(
        r_key.astype(np.int64), r_pay.astype(np.int64), s_key.astype(np.int64),
        s_pay.astype(np.int64), bits[0], bits[1], 8, use_reference=False)
    mask = (1 << 64) - 1
    assert (got[0] & mask, got[1]) == (dev[0] & mask, dev[1]) == (exp_s & mask, exp_c)
    assert exp_c == n_p


@pytest.mark.parametrize("scheme", ["Perfect", "BucketChaining"])
def test_streamed_zipf_closed_form(fi, scheme):
    """Zipf-skewed foreign keys: every S key matches, so count = |S| and
    sum = sum of S payloads (payload = key)."""
    n = 1 << 22
    rk = torch.empty(n, dtype=torch.int64, device="cuda")
    sk = torch.empty(n, dtype=torch.int64, device="cuda")
    fi.gen_primary_keys(rk, 5)
    fi.gen_zipf_foreign_keys(sk, n, 1.0, 6, 5)
    exp = int(sk.sum().item())
    hr, hs = rk.cpu().pin_memory(), sk.cpu().pin_memory()
    e = fi.RadixJoinEngine(n, n, torch.int64, fi.RadixBits(8, 9),
                           getattr(fi.HashingScheme, scheme))
    s, c = e.run_streamed(hr, hr, hs, hs, block_tuples=1 << 19)
    e.status()
    assert (s, c) == (exp, n)
    # a second run on the same engine reuses the staging slots
    assert e.run_streamed(hr, hr, hs, hs, block_tuples=1 << 20) == (exp, n)


def test_streamed_validation(fi):
    n = 1 << 16
    k = torch.arange(1, n + 1, dtype=torch.int64).pin_memory()
    one = fi.RadixJoinEngine(n, n, torch.int64, fi.RadixBits(8),
                             fi.HashingScheme.BucketChaining)
    with pytest.raises(fi.SqlOpsError) as ex:
        one.run_streamed(k, k, k, k)
    assert ex.value.kind == "Unsupported"
    big = 1 << 24
    two = fi.RadixJoinEngine(big, big, torch.int64, fi.RadixBits(6, 6),
                             fi.HashingScheme.BucketChaining)
    kb = torch.arange(1, big + 1, dtype=torch.int64).pin_memory()
    with pytest.raises(fi.SqlOpsError) as ex:
        two.run_streamed(kb, kb, kb, kb, block_tuples=1 << 16)  # 256 blocks
    assert ex.value.kind == "InvalidArgument"
    empty = torch.empty(0, dtype=torch.int64).pin_memory()
    assert two.run_streamed(empty, empty, kb, kb) == (0, 0)


@pytest.mark.parametrize("bits", [(9,), (5, 7)])
def test_run_host_one_and_two_passes(fi, bits):
    """The host entry point: one pass copies the columns whole, two passes
    stream them (here over two blocks of 2^26 tuples, the second ragged);
    the same closed-form result either way, and for empty relations."""
    n_b, n_p = 1 << 20, (1 << 26) + 54321
    rk = torch.empty(n_b, dtype=torch.int32, device="cuda")
    sk = torch.empty(n_p, dtype=torch.int32, device="cuda")
    fi.gen_primary_keys(rk, 7)
    fi.gen_uniform_foreign_keys(sk, n_b, 8)
    exp = (int(sk.to(torch.int64).sum().item()), n_p)
    hr, hs = rk.cpu().pin_memory(), sk.cpu().pin_memory()
    del rk, sk
    e = fi.RadixJoinEngine(n_b, n_p, torch.int32, fi.RadixBits(*bits),
                           fi.HashingScheme.BucketChaining)
    assert e.run_host(hr, hr, hs, hs) == exp
    e.status()
    assert e.run_host(hr[:0], hr[:0], hs, hs) == (0, 0)
    assert e.run_host(hr, hr, hs, hs) == exp
