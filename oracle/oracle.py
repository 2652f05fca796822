"""ctypes/numpy face of the CPU oracle.  TEST INFRASTRUCTURE ONLY.

Only tests/, the smoke check and bench.py's CPU-baseline leg import this
module.  It wraps two libraries:

* ``oracle/_build/liboracle.so`` -- the restatement of the reference's
  algorithms (``oracle.c``), the seeded generator (``datagen.c``) and the
  multi-threaded CPU baseline (``cpu_baseline.c``);
* ``oracle/_ref/libref_cpu.so`` -- the reference's own CPU operators compiled
  from its sources by ``oracle/build_ref.sh`` (optional: absent where the
  reference tree was never available).

Relations are numpy arrays of shape (n, 2) (columns key, value), which is the
memory layout of the reference's ``Tuple<K, V>`` (sql-ops/src/partition.rs:
144-147).  Offsets are uint64 arrays.
"""
import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "_build", "liboracle.so")
REF_PATH = os.path.join(HERE, "_ref", "libref_cpu.so")

PADDING_BYTES = 128  # sql-ops/build.rs:58
ALIGN_BYTES = 128  # sql-ops/build.rs:46

_lib = None
_ref = None

u64p = C.POINTER(C.c_uint64)
u32p = C.POINTER(C.c_uint32)


def build():
    """Compiles the oracle (and the reference library when its sources exist)."""
    subprocess.run(["make", "-s", "-C", HERE], check=True)


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            build()
        _lib = C.CDLL(LIB_PATH)
    return _lib


def ref_available():
    return os.path.exists(REF_PATH)


def ref():
    global _ref
    if _ref is None:
        _ref = C.CDLL(REF_PATH)
    return _ref


def _p(a):
    return C.c_void_p(a.ctypes.data)


def _sfx(dtype):
    return "i32" if np.dtype(dtype) == np.int32 else "i64"


def padding_len(dtype):
    """PADDING_BYTES / sizeof(Tuple<K, K>) (partitioned_relation.rs:27-29)."""
    return PADDING_BYTES // (2 * np.dtype(dtype).itemsize)


def input_chunk_size(n, chunks, key_bytes):
    f = lib().or_input_chunk_size
    f.restype = C.c_uint64
    return f(C.c_uint64(n), C.c_uint32(chunks), C.c_uint32(key_bytes))


def chunked_prefix_sum(keys, chunks, bits, ignore=0, pad=None):
    pad = padding_len(keys.dtype) if pad is None else pad
    out = np.zeros(chunks << bits, np.uint64)
    getattr(lib(), "or_chunked_prefix_sum_" + _sfx(keys.dtype))(
        _p(keys), C.c_uint64(len(keys)), C.c_uint32(chunks), C.c_uint32(bits),
        C.c_uint32(ignore), C.c_uint32(pad), _p(out))
    return out


def contiguous_prefix_sum(keys, grid, bits, ignore=0, pad=None):
    pad = padding_len(keys.dtype) if pad is None else pad
    off = np.zeros(1 << bits, np.uint64)
    loc = np.zeros(grid << bits, np.uint64)
    getattr(lib(), "or_contiguous_prefix_sum_" + _sfx(keys.dtype))(
        _p(keys), C.c_uint64(len(keys)), C.c_uint32(grid), C.c_uint32(bits),
        C.c_uint32(ignore), C.c_uint32(pad), _p(off), _p(loc))
    return off, loc


def chunked_radix_partition(keys, pays, chunk_offsets, chunks, bits, ignore,
                            padded_len, fill=-1):
    """Sequential scatter; padding slots keep `fill` (the null key)."""
    out = np.full((padded_len, 2), fill, keys.dtype)
    getattr(lib(), "or_chunked_radix_partition_" + _sfx(keys.dtype))(
        _p(keys), _p(pays), C.c_uint64(len(keys)), _p(chunk_offsets),
        C.c_uint32(chunks), C.c_uint32(bits), C.c_uint32(ignore), _p(out))
    return out


def prefix_sum_and_transform(pid, src, src_offsets, src_chunks, src_bits, pad,
                             grid, bits, ignore):
    dt = src.dtype
    n_max = len(src)
    dk = np.zeros(n_max, dt)
    dp = np.zeros(n_max, dt)
    off = np.zeros(1 << bits, np.uint64)
    loc = np.zeros(grid << bits, np.uint64)
    f = getattr(lib(), "or_prefix_sum_and_transform_" + _sfx(dt))
    f.restype = C.c_uint64
    n = f(C.c_uint32(pid), _p(src), _p(src_offsets), C.c_uint32(src_chunks),
          C.c_uint32(src_bits), C.c_uint64(len(src)), C.c_uint32(pad),
          C.c_uint32(grid), C.c_uint32(bits), C.c_uint32(ignore), _p(dk),
          _p(dp), _p(off), _p(loc))
    return dk[:n].copy(), dp[:n].copy(), off, loc


def assign_tasks(probe_offsets, probe_len, probe_pad, bits, grid, dtype):
    tasks = np.zeros(grid + 1, np.uint32)
    getattr(lib(), "or_assign_tasks_" + _sfx(dtype))(
        _p(probe_offsets), C.c_uint32(probe_len), C.c_uint32(probe_pad),
        C.c_uint32(bits), C.c_uint32(grid), _p(tasks))
    return tasks


def radix_join(scheme, build, build_off, build_pad, probe, probe_off,
               probe_pad, bits, ignore, ht_entries=None):
    """Returns (wrapping i64 sum, match count).  scheme: 'chaining'|'perfect'."""
    cnt = C.c_uint64(0)
    sfx = _sfx(build.dtype)
    if scheme == "chaining":
        f = getattr(lib(), "or_radix_join_chaining_" + sfx)
        f.restype = C.c_int64
        s = f(_p(build), _p(build_off), C.c_uint64(len(build)),
              C.c_uint32(build_pad), _p(probe), _p(probe_off),
              C.c_uint64(len(probe)), C.c_uint32(probe_pad), C.c_uint32(bits),
              C.c_uint32(ignore), C.byref(cnt))
    else:
        f = getattr(lib(), "or_radix_join_perfect_" + sfx)
        f.restype = C.c_int64
        s = f(_p(build), _p(build_off), C.c_uint64(len(build)),
              C.c_uint32(build_pad), _p(probe), _p(probe_off),
              C.c_uint64(len(probe)), C.c_uint32(probe_pad), C.c_uint32(bits),
              C.c_uint32(ignore), C.c_uint64(ht_entries), C.byref(cnt))
    return s, cnt.value


def ht_linearprobing_sum(build_key, build_pay, probe_key, probe_pay, entries):
    dt = build_key.dtype
    ht = np.full((entries, 2), -1, dt)
    sfx = _sfx(dt)
    getattr(lib(), "or_ht_build_linearprobing_" + sfx)(
        _p(ht), C.c_uint64(entries), _p(build_key), _p(build_pay),
        C.c_uint64(len(build_key)))
    f = getattr(lib(), "or_ht_probe_aggregate_linearprobing_" + sfx)
    f.restype = C.c_uint64
    return f(_p(ht), C.c_uint64(entries), _p(probe_key), _p(probe_pay),
             C.c_uint64(len(probe_key))), ht


def ht_perfect_sum(build_key, build_pay, probe_key, probe_pay, entries,
                   selective=False):
    dt = build_key.dtype
    ht = np.full((entries, 2), -1, dt)
    sfx = _sfx(dt)
    getattr(lib(), "or_ht_build_perfect_" + sfx)(
        _p(ht), C.c_uint64(entries), _p(build_key), _p(build_pay),
        C.c_uint64(len(build_key)), C.c_int(1 if selective else 0))
    f = getattr(lib(), "or_ht_probe_aggregate_perfect_" + sfx)
    f.restype = C.c_uint64
    return f(_p(ht), C.c_uint64(entries), _p(probe_key), _p(probe_pay),
             C.c_uint64(len(probe_key))), ht


# --------------------------------------------------------------------------
# Seeded generator (datagen.c)
# --------------------------------------------------------------------------
def primary_keys(n, seed, dtype=np.int64, base=1):
    out = np.empty(n, dtype)
    ct = C.c_int32 if np.dtype(dtype) == np.int32 else C.c_int64
    getattr(lib(), "dg_primary_keys_" + _sfx(dtype))(
        _p(out), C.c_uint64(n), C.c_uint64(seed), ct(base))
    return out


def uniform_foreign_keys(n, pk_n, seed, dtype=np.int64, base=1):
    out = np.empty(n, dtype)
    ct = C.c_int32 if np.dtype(dtype) == np.int32 else C.c_int64
    getattr(lib(), "dg_uniform_foreign_keys_" + _sfx(dtype))(
        _p(out), C.c_uint64(n), C.c_uint64(pk_n), C.c_uint64(seed), ct(base))
    return out


def zipf_foreign_keys(n, pk_n, s, seed, pk_seed, dtype=np.int64, base=1):
    out = np.empty(n, dtype)
    ct = C.c_int32 if np.dtype(dtype) == np.int32 else C.c_int64
    getattr(lib(), "dg_zipf_foreign_keys_" + _sfx(dtype))(
        _p(out), C.c_uint64(n), C.c_uint64(pk_n), C.c_double(s),
        C.c_uint64(seed), C.c_uint64(pk_seed), ct(base))
    return out


def null_keys(keys, selectivity, seed, base=1):
    """In place: keys whose seeded draw exceeds `selectivity` percent become
    the null key (datagen.c dg_null_keys, the selectivity of
    datagen/src/relation.rs:85-151)."""
    ct = C.c_int32 if keys.dtype == np.int32 else C.c_int64
    getattr(lib(), "dg_null_keys_" + _sfx(keys.dtype))(
        _p(keys), C.c_uint64(len(keys)), C.c_uint32(selectivity), C.c_uint64(seed),
        ct(base))
    return keys


def uniform_u64_keys(n, seed):
    out = np.empty(n, np.int64)
    lib().dg_uniform_u64_keys(_p(out), C.c_uint64(n), C.c_uint64(seed))
    return out


# --------------------------------------------------------------------------
# CPU baseline (cpu_baseline.c)
# --------------------------------------------------------------------------
def cpu_radix_join(r_key, r_pay, s_key, s_pay, bits1, bits2, threads,
                   use_reference=True):
    """Returns (sum, count, [prefix_s, partition_s, pass2_join_s], kind)."""
    path = REF_PATH.encode() if (use_reference and ref_available()) else None
    s = C.c_int64(0)
    c = C.c_uint64(0)
    t = (C.c_double * 3)()
    rc = lib().cb_cpu_radix_join_i64(
        _p(r_key), _p(r_pay), C.c_uint64(len(r_key)), _p(s_key), _p(s_pay),
        C.c_uint64(len(s_key)), C.c_uint32(bits1), C.c_uint32(bits2),
        C.c_uint32(threads), path, C.byref(s), C.byref(c), t)
    if rc != 0:
        raise RuntimeError("cpu baseline failed: %d" % rc)
    return s.value, c.value, list(t), ("reference" if path else "port")


# --------------------------------------------------------------------------
# The reference's own CPU operators (libref_cpu.so), called per chunk the way
# sql-ops/src/partition/cpu_radix_partition.rs:466-633 does.
# --------------------------------------------------------------------------
class _RefPrefixSumArgs(C.Structure):
    # sql-ops/cpputils/radix_partition.cpp:91-105
    _fields_ = [("partition_attr", C.c_void_p), ("data_length", C.c_size_t),
                ("canonical_chunk_length", C.c_size_t),
                ("padding_length", C.c_uint32), ("radix_bits", C.c_uint32),
                ("ignore_bits", C.c_uint32),
                ("tmp_partition_offsets", C.c_void_p),
                ("partition_offsets", C.c_void_p)]


class _RefPartitionArgs(C.Structure):
    # sql-ops/cpputils/radix_partition.cpp:107-124
    _fields_ = [("join_attr_data", C.c_void_p),
                ("payload_attr_data", C.c_void_p), ("data_length", C.c_size_t),
                ("padding_length", C.c_size_t), ("radix_bits", C.c_uint32),
                ("ignore_bits", C.c_uint32),
                ("partition_offsets", C.c_void_p),
                ("tmp_partition_offsets", C.c_void_p),
                ("write_combine_buffer", C.c_void_p),
                ("partitioned_relation", C.c_void_p)]


def ref_chunked_prefix_sum(keys, chunks, bits):
    kb = keys.dtype.itemsize
    sfx = "int32" if kb == 4 else "int64"
    pad = padding_len(keys.dtype)
    F = 1 << bits
    clen = input_chunk_size(len(keys), chunks, kb)
    out = np.zeros(chunks * F, np.uint64)
    tmp = np.zeros(F, np.uint32)
    for c in range(chunks):
        b = clen * c
        e = len(keys) if c + 1 == chunks else b + clen
        a = _RefPrefixSumArgs(keys.ctypes.data + b * kb, e - b, clen, pad, bits,
                              0, tmp.ctypes.data, out.ctypes.data + c * F * 8)
        getattr(ref(), "cpu_chunked_prefix_sum_" + sfx)(
            C.byref(a), C.c_uint32(c), C.c_uint32(chunks))
    return out


def ref_chunked_radix_partition(keys, pays, offsets, chunks, bits, swwc=False):
    kb = keys.dtype.itemsize
    sfx = "int32_int32" if kb == 4 else "int64_int64"
    pad = padding_len(keys.dtype)
    F = 1 << bits
    clen = input_chunk_size(len(keys), chunks, kb)
    padded = len(keys) + chunks * F * pad
    # 128-byte aligned output buffer, prefilled with the null key
    raw = np.full(padded * 2 + 64, -1, keys.dtype)
    shift = (-raw.ctypes.data % 128) // kb
    out = raw[shift:shift + padded * 2].reshape(padded, 2)
    wcb = ref().cpu_swwc_buffer_bytes
    wcb.restype = C.c_size_t
    wc_raw = np.zeros(F * wcb() + 64, np.uint8)
    wc = wc_raw[(-wc_raw.ctypes.data) % 64:]
    tmp = np.zeros(F, np.uint64)
    fn = getattr(ref(), ("cpu_chunked_radix_partition_swwc_" if swwc else
                         "cpu_chunked_radix_partition_") + sfx)
    for c in range(chunks):
        b = clen * c
        e = len(keys) if c + 1 == chunks else b + clen
        off = offsets[c * F:(c + 1) * F]
        base = int(off[0]) - pad
        a = _RefPartitionArgs(keys.ctypes.data + b * kb,
                              pays.ctypes.data + b * kb, e - b, pad, bits, 0,
                              off.ctypes.data, tmp.ctypes.data,
                              wc.ctypes.data,
                              out.ctypes.data + base * 2 * kb)
        fn(C.byref(a))
    return out.copy()


def ref_ht_linearprobing_sum(build_key, build_pay, probe_key, probe_pay,
                             entries):
    dt = build_key.dtype
    sfx = "int32" if dt == np.int32 else "int64"
    ht = np.full((entries, 2), -1, dt)
    getattr(ref(), "cpu_ht_build_linearprobing_" + sfx)(
        _p(ht), C.c_uint64(entries), _p(build_key), _p(build_pay),
        C.c_uint64(len(build_key)))
    res = C.c_uint64(0)
    getattr(ref(), "cpu_ht_probe_aggregate_linearprobing_" + sfx)(
        _p(ht), C.c_uint64(entries), _p(probe_key), _p(probe_pay),
        C.c_uint64(len(probe_key)), C.byref(res))
    return res.value, ht


def ref_ht_perfect_sum(build_key, build_pay, probe_key, probe_pay, entries,
                       selective=False):
    dt = build_key.dtype
    sfx = "int32" if dt == np.int32 else "int64"
    ht = np.full((entries, 2), -1, dt)
    getattr(ref(), ("cpu_ht_build_selective_perfect_" if selective else
                    "cpu_ht_build_perfect_") + sfx)(
        _p(ht), C.c_uint64(entries), _p(build_key), _p(build_pay),
        C.c_uint64(len(build_key)))
    res = C.c_uint64(0)
    getattr(ref(), "cpu_ht_probe_aggregate_perfect_" + sfx)(
        _p(ht), C.c_uint64(entries), _p(probe_key), _p(probe_pay),
        C.c_uint64(len(probe_key)), C.byref(res))
    return res.value, ht


def partition_multisets(rel, offsets, chunks, bits, padded_len, pad):
    """Per-(chunk, partition) sorted tuple runs, padding excluded
    (index rule of sql-ops/src/partition/partitioned_relation.rs:510-537)."""
    F = 1 << bits
    res = []
    n = chunks * F
    for i in range(n):
        b = int(offsets[i])
        e = int(offsets[i + 1]) - pad if i + 1 < n else padded_len
        run = rel[b:e]
        order = np.lexsort((run[:, 1], run[:, 0]))
        res.append(run[order])
    return res
