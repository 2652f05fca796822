"""CPU checks of the C ABI: the library loads, exports every symbol
include/fi_sqlops.h declares, and its host-side helpers (no GPU needed) keep
the reference's layout rules."""
import ctypes as C
import os
import re

import pytest

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(REPO, "include", "fi_sqlops.h")


def declared_symbols():
    text = open(HEADER).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(fi_[a-z0-9_]+)\s*\(", text)))


def test_library_exports_every_declared_symbol(fi):
    syms = declared_symbols()
    assert len(syms) >= 45
    missing = [s for s in syms if not hasattr(fi.lib(), s)]
    assert missing == []


def test_version(fi):
    assert b"sm_100a" in fi.lib().fi_version()


def test_input_chunk_size(fi, oracle):
    # partition_input_chunk.rs:24-35
    for n, c, kb in [(0, 1, 8), (100, 3, 4), (10**6, 148, 8), (2**29, 148, 8),
                     (2**30 + 7, 148, 4), (77, 80, 8)]:
        assert fi.input_chunk_size(n, c, kb) == oracle.input_chunk_size(n, c, kb)
    with pytest.raises(fi.SqlOpsError) as e:
        fi.input_chunk_size(2**33, 1, 8)
    assert e.value.kind == "IntegerOverflow"


def test_padding_len(fi):
    assert fi.lib().fi_padding_len(8) == 16
    assert fi.lib().fi_padding_len(16) == 8


def test_partitioned_relation_helpers(fi):
    lib = fi.lib()
    rel = fi._RelationC()
    # Chunked, 4 chunks, 2 bits, int64 tuples: 100 + 4*4*8 padding tuples
    n_alloc = lib.fi_partitioned_relation_alloc_len(C.c_uint64(100), 0, 2, 4, 16)
    assert n_alloc == 100 + 4 * 4 * 8
    with pytest.raises(fi.SqlOpsError):
        fi._check(lib.fi_partitioned_relation_init(
            C.byref(rel), C.c_uint64(100), 0, 2, 4, 16, C.c_void_p(1),
            C.c_uint64(n_alloc - 1), C.c_void_p(2)))
    fi._check(lib.fi_partitioned_relation_init(
        C.byref(rel), C.c_uint64(100), 0, 2, 4, 16, C.c_void_p(1),
        C.c_uint64(n_alloc), C.c_void_p(2)))
    assert rel.chunks == 4 and rel.len == 100
    # partition_len over host offsets (partitioned_relation.rs:409-437)
    import numpy as np
    pad = 8
    sizes = np.array([[3, 5, 0, 17], [9, 1, 1, 4], [0, 0, 30, 0], [10, 10, 5, 5]])
    offs, pos = [], 0
    for c in range(4):
        for p in range(4):
            pos += pad
            offs.append(pos)
            pos += sizes[c, p]
    offs = np.array(offs, np.uint64)
    rel.len = int(sizes.sum())
    for p in range(4):
        out = C.c_uint64(0)
        fi._check(lib.fi_partition_len(C.byref(rel), C.c_void_p(offs.ctypes.data),
                                       p, C.byref(out)))
        assert out.value == sizes[:, p].sum()
    with pytest.raises(fi.SqlOpsError) as e:
        fi._check(lib.fi_partition_len(C.byref(rel), C.c_void_p(offs.ctypes.data),
                                       4, C.byref(C.c_uint64())))
    assert "Invalid partition ID" in str(e.value)
    # resize (partitioned_relation.rs:383-395)
    fi._check(lib.fi_partitioned_relation_resize(C.byref(rel), C.c_uint64(100)))
    with pytest.raises(fi.SqlOpsError):
        fi._check(lib.fi_partitioned_relation_resize(C.byref(rel), C.c_uint64(101)))


def test_partition_offsets_init(fi):
    o = fi._OffsetsC()
    fi._check(fi.lib().fi_partition_offsets_init(C.byref(o), 1, 148, 9, 16,
                                                 C.c_void_p(8), C.c_void_p(16)))
    assert o.chunks == 1 and o.max_chunks == 148 and o.local_offsets == 16
    fi._check(fi.lib().fi_partition_offsets_init(C.byref(o), 0, 148, 9, 16,
                                                 C.c_void_p(8), C.c_void_p(16)))
    assert o.chunks == 148 and o.local_offsets is None


def test_errors_without_launch(fi):
    """Argument validation happens on the host before any launch."""
    with pytest.raises(fi.SqlOpsError) as e:
        fi.CudaRadixJoin(fi.RadixPass.Second, fi.RadixBits(5), fi.HashingScheme.Perfect,
                         4, 128)
    assert e.value.kind == "InvalidArgument"
    assert "pass is not specified" in str(e.value)


def test_hash_join_grouping_arguments(fi):
    """The grouping switches of CudaHashJoin validate their slices on the
    host; the status of a handle that never grouped is FI_OK (no device
    work).  The handle is made on a placeholder table address: nothing here
    touches the device."""
    L = fi.lib()
    h = C.c_void_p()
    table = C.c_void_p(0x100000)
    fi._check(L.fi_cuda_hash_join_new(C.c_int(int(fi.HashingScheme.LinearProbing)),
                                      C.c_int(0), table, C.c_uint64(1 << 20),
                                      C.c_uint64(1 << 20), C.c_uint32(148),
                                      C.c_uint32(256), C.c_uint32(148),
                                      C.c_uint32(256), C.byref(h)))
    try:
        for setter in (L.fi_cuda_hash_join_set_build_grouping,
                       L.fi_cuda_hash_join_set_probe_grouping):
            with pytest.raises(fi.SqlOpsError) as e:
                fi._check(setter(h, C.c_int(1), C.c_uint64(0)))
            assert e.value.kind == "InvalidArgument" and "at least 1" in str(e.value)
            with pytest.raises(fi.SqlOpsError) as e:
                fi._check(setter(h, C.c_int(1), C.c_uint64(1 << 32)))
            assert e.value.kind == "InvalidArgument" and "below 2^32" in str(e.value)
            fi._check(setter(h, C.c_int(1), C.c_uint64(1_000_003)))
            fi._check(setter(h, C.c_int(0), C.c_uint64(0)))  # off: the slice is unused
        fi._check(L.fi_cuda_hash_join_status(h))
        with pytest.raises(fi.SqlOpsError) as e:
            fi._check(L.fi_cuda_hash_join_status(None))
        assert e.value.kind == "InvalidArgument"
    finally:
        L.fi_cuda_hash_join_free(h)


def test_autotune_model_and_table(fi, tmp_path):
    """The autotuner's model (no table) and a loaded table (no GPU needed)."""
    fi.autotune_load(None)
    p = fi.autotune_plan(16, 1 << 21, 1 << 22)
    assert p["bits"] == (9,) and not p["batched"]          # 2^21 / 4096
    p = fi.autotune_plan(16, 1 << 30, 1 << 30)
    assert p["bits"] == (9, 9)                              # the 1024M join
    p = fi.autotune_plan(8, 100_000, 400_000)
    assert p["batched"] and p["bits"][0] <= 12              # below 4M tuples
    assert not fi.autotune_plan(8, 100_000, 400_000, small_tuples=1000)["batched"]
    table = tmp_path / "table.txt"
    table.write_text("# tb log2r log2k skew b1 b2 scheme block scatter\n"
                     "16 30 0 0 10 8 2 1024 1\n")
    fi.autotune_load(str(table))
    p = fi.autotune_plan(16, 1 << 30, 1 << 30)
    assert p["bits"] == (10, 8) and p["join_block"] == 1024 and p["scatter"] == 1
    assert fi.autotune_plan(16, 1 << 21, 1 << 22)["bits"] == (9,)  # too far
    assert fi.autotune_plan(8, 1 << 30, 1 << 30)["bits"] == (9, 9)  # other type
    table.write_text("16 30 0 0 10 8 2 333 1\n")
    with pytest.raises(fi.SqlOpsError) as ex:
        fi.autotune_load(str(table))
    assert ex.value.kind == "InvalidArgument"
    fi.autotune_load(None)


def test_reference_gpu_harness_exports():
    """The launch harness of the reference's own GPU kernels
    (baseline/refgpu) loads without a GPU and exports its entry points."""
    import ctypes as C
    import os
    import sys
    sys.path.insert(0, os.path.join(os.path.dirname(os.path.dirname(
        os.path.abspath(__file__))), "baseline", "refgpu"))
    import refgpu
    if not refgpu.available():
        pytest.skip("reference GPU kernels not built (no reference tree)")
    lib = refgpu.lib()
    for name in ("rg_chunked_prefix_sum", "rg_partition_prepare", "rg_partition",
                 "rg_join_prepare", "rg_join", "rg_last_error", "rg_padding_len"):
        assert hasattr(lib, name), name
    assert lib.rg_padding_len(C.c_int(4)) == 16
    assert lib.rg_padding_len(C.c_int(8)) == 8


def test_cpp_host_api_builds():
    """The C++ host API (include/fi_sqlops.hpp) and its test program compile
    and link against the library (run on a GPU by test_gpu_host_api.py)."""
    import subprocess
    import os
    here = os.path.dirname(os.path.abspath(__file__))
    r = subprocess.run(["make", "-s", "-C", os.path.join(here, "cpp")],
                       capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    assert os.path.exists(os.path.join(here, "cpp", "_build", "host_api_test"))
