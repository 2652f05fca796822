"""Hybrid join: CPU first pass (cpu_partition.cu) + GPU second pass and join,
against the device-resident join and the closed form."""
import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu


def wrap64(x):
    return (int(x) + (1 << 63)) % (1 << 64) - (1 << 63)


@pytest.mark.parametrize("dt,ndt", [(torch.int32, np.int32), (torch.int64, np.int64)])
@pytest.mark.parametrize("threads", [1, 5, 0, 1000])
@pytest.mark.parametrize("zipf", [0.0, 1.0])
def test_hybrid_matches_device_join(fi, oracle, dt, ndt, threads, zipf):
    n_b, n_p = (1 << 20) + 5, (3 << 20) + 11
    rk = torch.from_numpy(oracle.primary_keys(n_b, 31, ndt))
    sk = torch.from_numpy(oracle.zipf_foreign_keys(n_p, n_b, zipf, 32, 31, ndt))
    rp, sp = rk * 3, sk - 7
    e = fi.RadixJoinEngine(n_b, n_p, dt, fi.RadixBits(7, 6),
                           fi.HashingScheme.BucketChaining)
    got = e.run_hybrid(rk, rp, sk, sp, threads=threads)
    exp = (wrap64(sp.to(torch.int64).sum().item()), n_p)
    assert got == exp
    assert e.run(rk.cuda(), rp.cuda(), sk.cuda(), sp.cuda()) == exp
    e.status()


def test_hybrid_needs_two_passes_and_empty(fi):
    k = torch.arange(1, 1001, dtype=torch.int64)
    e = fi.RadixJoinEngine(1000, 1000, torch.int64, fi.RadixBits(6),
                           fi.HashingScheme.BucketChaining)
    with pytest.raises(fi.SqlOpsError) as ex:
        e.run_hybrid(k, k, k, k)
    assert ex.value.kind == "Unsupported"
    e2 = fi.RadixJoinEngine(1000, 1000, torch.int64, fi.RadixBits(4, 4),
                            fi.HashingScheme.BucketChaining)
    assert e2.run_hybrid(k, k, k, k) == (int(k.sum()), 1000)
    z = torch.empty(0, dtype=torch.int64)
    assert e2.run_hybrid(k, k, z, z) == (0, 0)
