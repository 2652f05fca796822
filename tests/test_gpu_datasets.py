"""Named data sets with join selectivity, and joins of relations loaded from
relation files, on the GPU against the oracle."""
import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu


def wrap64(x):
    return (int(x) + (1 << 63)) % (1 << 64) - (1 << 63)


@pytest.mark.parametrize("dt,ndt", [(torch.int32, np.int32), (torch.int64, np.int64)])
@pytest.mark.parametrize("sel", [0, 37, 100])
def test_null_keys_match_oracle(fi, oracle, dt, ndt, sel):
    n = (1 << 20) + 3
    keys = torch.empty(n, dtype=dt, device="cuda")
    fi.gen_primary_keys(keys, 5)
    exp = oracle.null_keys(oracle.primary_keys(n, 5, ndt), sel, 77)
    fi.null_keys(keys, sel, 77)
    assert np.array_equal(keys.cpu().numpy(), exp)


@pytest.mark.parametrize("dataset,dt", [("Test", torch.int64), ("Test", torch.int32),
                                        ("Blanas4MB", torch.int64)])
@pytest.mark.parametrize("sel", [100, 50])
def test_dataset_join_with_selectivity(fi, oracle, dataset, dt, sel):
    """A foreign key matches iff its primary key survived the selectivity
    draw; payload = key, so the sum is that of the matching foreign keys."""
    ds = getattr(fi.Dataset, dataset)
    rk, rp, sk, sp = fi.gen_dataset(ds, dt, selectivity=sel, seed=3)
    nb, npr = fi.dataset_shape(ds, dt)
    assert rk.numel() == nb and sk.numel() == npr
    s_np = sk.cpu().numpy()
    kept = oracle.null_keys(s_np.copy(), sel, 3 + 7) != -1
    exp = (wrap64(s_np[kept].astype(np.int64).sum()), int(kept.sum()))
    plan = fi.autotune_plan(8 if dt == torch.int32 else 16, nb, npr)
    bits = plan["bits"] if plan["bits"][0] > 0 else (1,)
    e = fi.RadixJoinEngine(nb, npr, dt, fi.RadixBits(*bits),
                           fi.HashingScheme.BucketChaining)
    assert e.run(rk, rp, sk, sp) == exp
    e.status()


@pytest.mark.parametrize("dt,ndt", [(torch.int32, np.int32), (torch.int64, np.int64)])
def test_join_from_relation_files(fi, oracle, tmp_path, dt, ndt):
    """build_with_files: both relations read from text files (the outer one
    gzip-compressed), joined through the host entry point."""
    import gzip
    n_b, n_p = 40_000, 100_000
    rk = oracle.primary_keys(n_b, 21, ndt)
    rp = (rk * 2).astype(ndt)
    sk = oracle.uniform_foreign_keys(n_p, n_b, 22, ndt)
    sp = (sk - 5).astype(ndt)
    inner, outer = tmp_path / "r.tsv", tmp_path / "s.tsv.gz"
    inner.write_text("key value\n" + "".join("%d %d\n" % t for t in zip(rk.tolist(), rp.tolist())))
    with gzip.open(outer, "wt") as f:
        f.write("key value\n" + "".join("%d %d\n" % t for t in zip(sk.tolist(), sp.tolist())))
    cols = fi.load_join_data(str(inner), str(outer), dt)
    assert all(c.is_pinned() for c in cols)
    e = fi.RadixJoinEngine(n_b, n_p, dt, fi.RadixBits(6, 5),
                           fi.HashingScheme.BucketChaining)
    got = e.run_host(*cols)
    exp = (wrap64(sp.astype(np.int64).sum()), n_p)
    assert got == exp
