"""Relation files (data-store/src/join_data.rs:173-280, build_with_files)
and the named data set shapes (datagen/src/popular.rs, the data sets of
radix-join/src/main.rs:657-760), through the C ABI on the CPU: no GPU is
touched by the loader or the shape table."""
import gzip

import numpy as np
import pytest
import torch


def write_relation(path, keys, pays, header="key payload", newline="\n"):
    text = header + newline + "".join(
        "%d %d%s" % (k, v, newline) for k, v in zip(keys.tolist(), pays.tolist()))
    if str(path).endswith("gz"):
        with gzip.open(path, "wt", newline="") as f:
            f.write(text)
    else:
        with open(path, "w", newline="") as f:
            f.write(text)


@pytest.mark.parametrize("dtype", [np.int32, np.int64])
@pytest.mark.parametrize("name", ["r.tsv", "r.tsv.gz"])
def test_read_relation_file(fi, oracle, tmp_path, dtype, name):
    n = 5000
    keys = oracle.primary_keys(n, 11, dtype)
    pays = oracle.uniform_foreign_keys(n, 1 << 20, 12, dtype) - (1 << 19)
    info = np.iinfo(dtype)
    keys[:2] = [info.min, info.max]  # the whole range parses
    path = tmp_path / name
    write_relation(path, keys, pays)
    assert fi.relation_file_len(str(path)) == n
    tdt = torch.int32 if dtype == np.int32 else torch.int64
    k, v = fi.read_relation_file(str(path), tdt, pin=False)
    assert k.dtype == tdt and np.array_equal(k.numpy(), keys)
    assert np.array_equal(v.numpy(), pays)


def test_load_join_data_crlf_and_blank_lines(fi, tmp_path):
    r = tmp_path / "inner.tsv"
    s = tmp_path / "outer.tsv.gz"
    write_relation(r, np.arange(1, 4), np.arange(10, 13), newline="\r\n")
    with open(s, "wb") as f:
        f.write(gzip.compress(b"k v\n\n1 7\n\n3 -9\n"))
    rk, rp, sk, sp = fi.load_join_data(str(r), str(s), torch.int64, pin=False)
    assert rk.tolist() == [1, 2, 3] and rp.tolist() == [10, 11, 12]
    assert sk.tolist() == [1, 3] and sp.tolist() == [7, -9]


def test_empty_and_header_only_files(fi, tmp_path):
    for text in ["", "key payload\n"]:
        p = tmp_path / "e.tsv"
        p.write_text(text)
        assert fi.relation_file_len(str(p)) == 0
        k, v = fi.read_relation_file(str(p), torch.int64, pin=False)
        assert k.numel() == 0 and v.numel() == 0


@pytest.mark.parametrize("body,dtype,what", [
    ("1 2 3\n", torch.int64, "two fields"),
    ("1\n", torch.int64, "two fields"),
    ("1  2\n", torch.int64, "two fields"),
    ("1 x\n", torch.int64, "integer"),
    ("1 2.5\n", torch.int64, "integer"),
    ("2147483648 1\n", torch.int32, "32-bit"),
    ("9223372036854775808 1\n", torch.int64, "64-bit"),
    ("-9223372036854775809 1\n", torch.int64, "64-bit"),
])
def test_malformed_lines_are_errors(fi, tmp_path, body, dtype, what):
    p = tmp_path / "bad.tsv"
    p.write_text("key payload\n1 1\n" + body)
    with pytest.raises(fi.SqlOpsError) as ex:
        fi.read_relation_file(str(p), dtype, pin=False)
    assert ex.value.kind == "InvalidArgument"
    assert what in str(ex.value) and "bad.tsv:3" in str(ex.value)


def test_file_errors(fi, tmp_path):
    with pytest.raises(fi.SqlOpsError) as ex:
        fi.relation_file_len(str(tmp_path / "missing.tsv"))
    assert "cannot open" in str(ex.value)
    p = tmp_path / "plain.gz"  # the name promises gzip data
    p.write_text("key payload\n1 2\n")
    with pytest.raises(fi.SqlOpsError) as ex:
        fi.relation_file_len(str(p))
    assert "not gzip" in str(ex.value)
    q = tmp_path / "short.tsv"
    q.write_text("key payload\n1 2\n3 4\n")
    k = torch.empty(1, dtype=torch.int64)
    rc = fi.lib().fi_relation_file_read_int64(str(q).encode(), fi.C.c_void_p(k.data_ptr()),
                                              fi.C.c_void_p(k.data_ptr()),
                                              fi.C.c_uint64(1))
    assert rc != 0 and "more than 1" in fi.lib().fi_last_error().decode()


def test_dataset_shapes(fi):
    D = fi.Dataset
    assert fi.dataset_shape(D.Blanas, torch.int64) == (16 << 20, 256 << 20)
    assert fi.dataset_shape(D.Blanas4MB, torch.int64) == (512 << 10, 256 << 20)
    assert fi.dataset_shape(D.Kim, torch.int32) == (128 * 10**6, 128 * 10**6)
    assert fi.dataset_shape(D.Test, torch.int32) == (1000, 1000)
    assert fi.dataset_shape(D.Lutz2Gv32G, torch.int64) == ((2 << 30) // 16, (32 << 30) // 16)
    assert fi.dataset_shape(D.Lutz32Gv32G, torch.int32) == ((32 << 30) // 8, (32 << 30) // 8)
    with pytest.raises(fi.SqlOpsError):
        fi.dataset_shape(17, torch.int64)


def test_oracle_null_keys_selectivity(oracle):
    """The oracle's selectivity draw keeps (s + 1) / 101 of the keys, and the
    same keys whatever their order."""
    n = 200_000
    k = oracle.primary_keys(n, 4, np.int64)
    for sel in (0, 25, 50, 99):
        kk = oracle.null_keys(k.copy(), sel, 9)
        kept = (kk != -1).mean()
        assert abs(kept - (sel + 1) / 101) < 0.01
        shuffled = oracle.null_keys(k[::-1].copy(), sel, 9)
        assert np.array_equal(shuffled[::-1], kk)
    assert np.array_equal(oracle.null_keys(k.copy(), 100, 9), k)
