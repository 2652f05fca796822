"""Python face of the B200 sql-ops operators: a ctypes binding of the C ABI in
include/fi_sqlops.h, shaped like the reference's Rust API (sql-ops/src/...):

* ``RadixBits``, ``RadixPass``, ``GpuHistogramAlgorithm``,
  ``GpuRadixPartitionAlgorithm``, ``HashingScheme`` (partition.rs:35-134,
  gpu_radix_partition.rs:192-293, join/hashing_scheme.rs:18-43);
* ``PartitionOffsets`` and ``PartitionedRelation`` (partitioned_relation.rs)
  holding torch tensors as memory;
* ``GpuRadixPartitioner`` (gpu_radix_partition.rs:314-555), ``CudaRadixJoin``
  (join/cuda_radix_join.rs:116-164), ``CudaHashJoin`` / ``HashTable``
  (join/no_partitioning_join.rs:153-304);
* ``RadixJoinEngine``: the gpu_radix_join execution method
  (radix-join/src/execution_methods/gpu_radix_join.rs:90-565);
* the seeded generator (``gen_*``).

Every call goes through the compiled library ``libfi_sqlops.so`` next to this
file; there is no other code path.  Errors raise ``SqlOpsError`` whose ``kind``
names the reference's ErrorKind (sql-ops/src/error.rs:20-29).
"""
import ctypes as C
import enum
import os

import torch

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libfi_sqlops.so")
TUNING_TABLE = os.path.join(HERE, "tuning_table.txt")

PADDING_BYTES = 128
ALIGN_BYTES = 128
RADIX_JOIN_BUCKET_CHAINING_ENTRIES = 2048

_ERR_KIND = {
    -1: "InvalidArgument",
    -2: "IntegerOverflow",
    -3: "CudaError",
    -4: "RuntimeError",
    -5: "Timeout",
    -6: "Unsupported",
    -7: "Capacity",
    -8: "OutOfMemory",
}


class SqlOpsError(RuntimeError):
    def __init__(self, code, message):
        self.code = code
        self.kind = _ERR_KIND.get(code, "Unknown")
        super().__init__("%s: %s" % (self.kind, message))


_lib = None


def lib():
    """The compiled library; raises if it has not been built."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise OSError(
                "libfi_sqlops.so is missing; build it with "
                "`make -C fast-interconnects_b200` (or __graft_entry__.build())")
        _lib = C.CDLL(LIB_PATH)
        _lib.fi_last_error.restype = C.c_char_p
        _lib.fi_version.restype = C.c_char_p
        _lib.fi_padding_len.restype = C.c_uint32
        _lib.fi_partitioned_relation_alloc_len.restype = C.c_uint64
        _lib.fi_radix_join_engine_workspace_bytes.restype = C.c_uint64
        _lib.fi_gpu_prefix_sum_state_len.restype = C.c_uint64
        # the autotuner's measured table (autotune.py), when it exists
        if os.path.exists(TUNING_TABLE):
            _check(_lib.fi_autotune_load(TUNING_TABLE.encode()))
    return _lib


def _check(rc):
    if rc != 0:
        raise SqlOpsError(rc, lib().fi_last_error().decode())


# ---------------------------------------------------------------------------
# vocabulary
# ---------------------------------------------------------------------------
class GpuHistogramAlgorithm(enum.IntEnum):
    Chunked = 0
    Contiguous = 1


HistogramAlgorithmType = GpuHistogramAlgorithm


class GpuRadixPartitionAlgorithm(enum.IntEnum):
    NC = 0
    LASWWC = 1
    SSWWCv2 = 2
    SSWWCv2G = 3
    HSSWWCv4 = 4


class RadixPass(enum.IntEnum):
    First = 0
    Second = 1
    Third = 2


class HashingScheme(enum.IntEnum):
    Perfect = 0
    LinearProbing = 1
    BucketChaining = 2


class _RadixBitsC(C.Structure):
    _fields_ = [("pass_bits", C.c_int32 * 3)]


class RadixBits:
    """RadixBits (partition.rs:64-110)."""

    def __init__(self, first=None, second=None, third=None):
        self.pass_bits = [first, second, third]

    def c(self):
        return _RadixBitsC((C.c_int32 * 3)(
            *[-1 if b is None else b for b in self.pass_bits]))

    def pass_radix_bits(self, p):
        return self.pass_bits[int(p)]

    def pass_fanout(self, p):
        b = self.pass_bits[int(p)]
        return None if b is None else 1 << b

    def pass_ignore_bits(self, p):
        return sum(b or 0 for b in self.pass_bits[:int(p)])

    def radix_bits(self):
        return sum(b or 0 for b in self.pass_bits)


class _OffsetsC(C.Structure):
    _fields_ = [("offsets", C.c_void_p), ("local_offsets", C.c_void_p),
                ("chunks", C.c_uint32), ("max_chunks", C.c_uint32),
                ("radix_bits", C.c_uint32), ("histogram_type", C.c_uint32),
                ("data_len", C.c_uint64), ("has_data_len", C.c_uint32),
                ("tuple_bytes", C.c_uint32)]


class _RelationC(C.Structure):
    _fields_ = [("relation", C.c_void_p), ("relation_len", C.c_uint64),
                ("offsets", C.c_void_p), ("len", C.c_uint64),
                ("chunks", C.c_uint32), ("radix_bits", C.c_uint32),
                ("tuple_bytes", C.c_uint32), ("reserved", C.c_uint32)]


class _JoinResultC(C.Structure):
    _fields_ = [("sum", C.c_int64), ("count", C.c_uint64)]


class _JoinPlanC(C.Structure):
    _fields_ = [("radix_bits", _RadixBitsC), ("hashing_scheme", C.c_int),
                ("join_block", C.c_uint32), ("scatter", C.c_uint32)]


def _ptr(t):
    return C.c_void_p(t.data_ptr()) if t is not None else C.c_void_p(0)


def _stream(stream):
    if stream is None:
        stream = torch.cuda.current_stream()
    return C.c_void_p(stream.cuda_stream)


def _tuple_bytes(dtype):
    return 8 if dtype == torch.int32 else 16


def _sfx(dtype):
    if dtype == torch.int32:
        return "int32"
    if dtype == torch.int64:
        return "int64"
    raise TypeError("keys must be int32 or int64 (gpu_radix_partition.rs:1245)")


def padding_len(dtype):
    return lib().fi_padding_len(_tuple_bytes(dtype))


def input_chunk_size(data_len, num_chunks, key_bytes):
    out = C.c_uint64(0)
    _check(lib().fi_input_chunk_size(C.c_uint64(data_len), C.c_uint32(num_chunks),
                                     C.c_uint32(key_bytes), C.byref(out)))
    return out.value


# ---------------------------------------------------------------------------
# PartitionOffsets / PartitionedRelation
# ---------------------------------------------------------------------------
class PartitionOffsets:
    """PartitionOffsets<Tuple<K,K>> (partitioned_relation.rs:62-201).

    Memory: u64 tensors on `device` (pass 'cpu' with pin=True for pinned host
    memory the GPU can address, like the reference's CudaPinnedMem)."""

    def __init__(self, histogram_type, max_chunks, radix_bits, dtype,
                 device="cuda", pin=False):
        F = 1 << radix_bits
        chunks = max_chunks if histogram_type == GpuHistogramAlgorithm.Chunked else 1
        self.dtype = dtype
        self.offsets = _alloc_u64(chunks * F, device, pin)
        self.local_offsets = (_alloc_u64(max_chunks * F, device, pin)
                              if histogram_type == GpuHistogramAlgorithm.Contiguous
                              else None)
        self.c = _OffsetsC()
        _check(lib().fi_partition_offsets_init(
            C.byref(self.c), C.c_int(int(histogram_type)), C.c_uint32(max_chunks),
            C.c_uint32(radix_bits), C.c_uint32(_tuple_bytes(dtype)),
            _ptr(self.offsets), _ptr(self.local_offsets)))

    def _sync_ptrs(self):
        self.c.offsets = self.offsets.data_ptr()

    def num_chunks(self):
        return self.c.chunks

    def radix_bits(self):
        return self.c.radix_bits

    def fanout(self):
        return 1 << self.c.radix_bits

    def len(self):
        return self.c.data_len if self.c.has_data_len else None

    def padding_len(self):
        return padding_len(self.dtype)


def _alloc_u64(n, device, pin):
    t = torch.empty(max(n, 1), dtype=torch.int64,
                    device=device if not pin else "cpu",
                    pin_memory=pin)
    return t


class PartitionedRelation:
    """PartitionedRelation<Tuple<K,K>> (partitioned_relation.rs:323-497).
    `relation` is an (alloc_len, 2) tensor; `offsets` a u64 tensor."""

    def __init__(self, length, histogram_type, radix_bits, max_chunks, dtype,
                 device="cuda", fill=None):
        alloc = lib().fi_partitioned_relation_alloc_len(
            C.c_uint64(length), C.c_int(int(histogram_type)),
            C.c_uint32(radix_bits), C.c_uint32(max_chunks),
            C.c_uint32(_tuple_bytes(dtype)))
        self.dtype = dtype
        if fill is None:
            self.relation = torch.empty((max(alloc, 1), 2), dtype=dtype, device=device)
        else:
            self.relation = torch.full((max(alloc, 1), 2), fill, dtype=dtype,
                                       device=device)
        chunks = max_chunks if histogram_type == GpuHistogramAlgorithm.Chunked else 1
        self.offsets = torch.zeros(chunks << radix_bits, dtype=torch.int64,
                                   device=device)
        self.c = _RelationC()
        _check(lib().fi_partitioned_relation_init(
            C.byref(self.c), C.c_uint64(length), C.c_int(int(histogram_type)),
            C.c_uint32(radix_bits), C.c_uint32(max_chunks),
            C.c_uint32(_tuple_bytes(dtype)), _ptr(self.relation),
            C.c_uint64(alloc), _ptr(self.offsets)))

    def _sync_ptrs(self):
        self.c.offsets = self.offsets.data_ptr()

    def len(self):
        return self.c.len

    def num_chunks(self):
        return self.c.chunks

    def radix_bits(self):
        return self.c.radix_bits

    def fanout(self):
        return 1 << self.c.radix_bits

    def padding_len(self):
        return padding_len(self.dtype)

    def padded_len(self):
        return self.c.len + (self.c.chunks << self.c.radix_bits) * self.padding_len()

    def resize(self, new_len):
        _check(lib().fi_partitioned_relation_resize(C.byref(self.c),
                                                    C.c_uint64(new_len)))

    def partition_len(self, partition_id):
        host = self.offsets.cpu().contiguous()
        out = C.c_uint64(0)
        _check(lib().fi_partition_len(C.byref(self.c), _ptr(host),
                                      C.c_uint32(partition_id), C.byref(out)))
        return out.value


# ---------------------------------------------------------------------------
# GpuRadixPartitioner
# ---------------------------------------------------------------------------
class GpuRadixPartitioner:
    """GpuRadixPartitioner (gpu_radix_partition.rs:314-555)."""

    def __init__(self, prefix_sum_algorithm, partition_algorithm, radix_bits,
                 grid_size, block_size, dmem_buffer_bytes=8192):
        self.h = C.c_void_p()
        self.radix_bits = radix_bits
        _check(lib().fi_gpu_radix_partitioner_new(
            C.c_int(int(prefix_sum_algorithm)), C.c_int(int(partition_algorithm)),
            radix_bits.c(), C.c_uint32(grid_size), C.c_uint32(block_size),
            C.c_uint64(dmem_buffer_bytes), C.byref(self.h)))

    def __del__(self):
        if getattr(self, "h", None) and _lib is not None:
            _lib.fi_gpu_radix_partitioner_free(self.h)
            self.h = None

    def status(self):
        _check(lib().fi_gpu_radix_partitioner_status(self.h))

    def prefix_sum(self, radix_pass, partition_attr, partition_offsets,
                   stream=None):
        f = getattr(lib(), "fi_gpu_prefix_sum_" + _sfx(partition_attr.dtype))
        _check(f(self.h, C.c_int(int(radix_pass)), _ptr(partition_attr),
                 C.c_uint64(partition_attr.numel()),
                 C.byref(partition_offsets.c), _stream(stream)))

    def prefix_sum_and_copy_with_payload(self, radix_pass, src_key, src_pay,
                                         dst_key, dst_pay, partition_offsets,
                                         stream=None):
        f = getattr(lib(), "fi_gpu_prefix_sum_and_copy_with_payload_" +
                    _sfx(src_key.dtype))
        _check(f(self.h, C.c_int(int(radix_pass)), _ptr(src_key), _ptr(src_pay),
                 C.c_uint64(src_key.numel()), _ptr(dst_key), _ptr(dst_pay),
                 C.c_uint64(dst_key.numel()), C.byref(partition_offsets.c),
                 _stream(stream)))

    def prefix_sum_and_transform(self, radix_pass, partition_id, src_relation,
                                 dst_key, dst_pay, partition_offsets,
                                 stream=None):
        f = getattr(lib(), "fi_gpu_prefix_sum_and_transform_" + _sfx(dst_key.dtype))
        _check(f(self.h, C.c_int(int(radix_pass)), C.c_uint32(partition_id),
                 C.byref(src_relation.c), _ptr(dst_key), _ptr(dst_pay),
                 C.c_uint64(dst_key.numel()), C.byref(partition_offsets.c),
                 _stream(stream)))

    def preallocate_partition_state(self, radix_pass, dtype=torch.int64):
        f = getattr(lib(), "fi_gpu_preallocate_partition_state_" + _sfx(dtype))
        _check(f(self.h, C.c_int(int(radix_pass))))

    def partition(self, radix_pass, partition_attr, payload_attr,
                  partition_offsets, partitioned_relation, stream=None):
        """Partitions and swaps the offsets into the relation
        (gpu_radix_partition.rs:1113-1121)."""
        if partition_attr.numel() != payload_attr.numel():
            raise SqlOpsError(-1, "Partition and payload attributes have "
                                  "different sizes")
        f = getattr(lib(), "fi_gpu_partition_" + _sfx(partition_attr.dtype))
        before = partition_offsets.c.offsets
        _check(f(self.h, C.c_int(int(radix_pass)), _ptr(partition_attr),
                 _ptr(payload_attr), C.c_uint64(partition_attr.numel()),
                 C.byref(partition_offsets.c), C.byref(partitioned_relation.c),
                 _stream(stream)))
        if partitioned_relation.c.offsets == before:
            partition_offsets.offsets, partitioned_relation.offsets = (
                partitioned_relation.offsets, partition_offsets.offsets)


# ---------------------------------------------------------------------------
# CudaRadixJoin
# ---------------------------------------------------------------------------
def prefix_sum_state_len(grid_size, block_size):
    """GpuPrefixSum::state_len: scan-state entries (32 bytes each)."""
    return lib().fi_gpu_prefix_sum_state_len(C.c_uint32(grid_size), C.c_uint32(block_size))


def block_exclusive_prefix_sum(data, padding, grid_size, block_size, stream=None):
    """host_block_exclusive_prefix_sum_uint64 on a device u64 (int64) tensor,
    in place: each block scans its len/grid_size items."""
    _check(lib().fi_block_exclusive_prefix_sum_uint64(
        _ptr(data), C.c_uint64(data.numel()), C.c_uint64(padding),
        C.c_uint32(grid_size), C.c_uint32(block_size), _stream(stream)))


def device_exclusive_prefix_sum(data, padding, grid_size, block_size, stream=None):
    """host_device_exclusive_prefix_sum[_initialize]_uint64 on a device u64
    (int64) tensor, in place, with freshly initialised state."""
    n = prefix_sum_state_len(grid_size, block_size)
    state = torch.empty(4 * n, dtype=torch.int64, device=data.device)
    status = torch.zeros(1, dtype=torch.int32, device=data.device)
    _check(lib().fi_device_exclusive_prefix_sum_initialize_uint64(
        _ptr(state), C.c_uint32(grid_size), C.c_uint32(block_size), _stream(stream)))
    _check(lib().fi_device_exclusive_prefix_sum_uint64(
        _ptr(data), C.c_uint64(data.numel()), C.c_uint64(padding), _ptr(state),
        C.c_uint32(grid_size), C.c_uint32(block_size), _ptr(status), _stream(stream)))
    if int(status.item()) != 0:
        _check(int(status.item()))


class CpuHistogramAlgorithm(enum.IntEnum):
    Chunked = 0
    ChunkedSimd = 1


class CpuRadixPartitionAlgorithm(enum.IntEnum):
    NC = 0
    SWWC = 1
    SWWCSimd = 2


class CpuRadixPartitioner:
    """CpuRadixPartitioner (cpu_radix_partition.rs): per-chunk prefix sum and
    partition on the host, one partitioner per thread.  Arrays are numpy
    arrays or CPU tensors; `relation` is a (padded_len, 2) array of the key
    type."""

    def __init__(self, histogram_algorithm, partition_algorithm, radix_bits):
        self.radix_bits = radix_bits
        self.h = C.c_void_p()
        _check(lib().fi_cpu_radix_partitioner_new(
            C.c_int(int(histogram_algorithm)), C.c_int(int(partition_algorithm)),
            C.c_uint32(radix_bits), C.byref(self.h)))

    def __del__(self):
        if getattr(self, "h", None) and _lib is not None:
            _lib.fi_cpu_radix_partitioner_free(self.h)
            self.h = None

    @staticmethod
    def _addr(a):
        return C.c_void_p(a.data_ptr() if isinstance(a, torch.Tensor) else a.ctypes.data)

    @staticmethod
    def _sfx(a):
        return "int32" if a.dtype in (torch.int32, np_int32()) else "int64"

    def prefix_sum(self, keys, chunk_id, num_chunks, chunk_offsets, ignore_bits=0):
        f = getattr(lib(), "fi_cpu_prefix_sum_" + self._sfx(keys))
        _check(f(self.h, self._addr(keys), C.c_uint64(len(keys)), C.c_uint32(chunk_id),
                 C.c_uint32(num_chunks), C.c_uint32(ignore_bits),
                 self._addr(chunk_offsets)))

    def partition(self, keys, pays, chunk_id, num_chunks, chunk_offsets, relation,
                  ignore_bits=0):
        f = getattr(lib(), "fi_cpu_partition_" + self._sfx(keys))
        _check(f(self.h, self._addr(keys), self._addr(pays), C.c_uint64(len(keys)),
                 C.c_uint32(chunk_id), C.c_uint32(num_chunks), C.c_uint32(ignore_bits),
                 self._addr(chunk_offsets), self._addr(relation),
                 C.c_uint64(len(relation))))


def np_int32():
    import numpy as np
    return np.dtype(np.int32)


def cpu_radix_partition(keys, pays, radix_bits, num_chunks,
                        algorithm=CpuRadixPartitionAlgorithm.SWWC, fill=-1):
    """Chunked partition of numpy columns on num_chunks host threads (one
    partitioner each, as the reference's rayon scope): returns (relation of
    len + chunks*F*pad tuples, offsets of chunks*F entries)."""
    import threading
    import numpy as np
    F = 1 << radix_bits
    pad = padding_len(torch.int32 if keys.dtype == np.int32 else torch.int64)
    offsets = np.zeros(num_chunks * F, np.uint64)
    rel = np.full((len(keys) + num_chunks * F * pad, 2), fill, keys.dtype)
    errors = []

    def run(c):
        try:
            p = CpuRadixPartitioner(CpuHistogramAlgorithm.Chunked, algorithm, radix_bits)
            off = offsets[c * F:(c + 1) * F]
            p.prefix_sum(keys, c, num_chunks, off)
            p.partition(keys, pays, c, num_chunks, off, rel)
        except Exception as e:  # reported after the join
            errors.append(e)

    ts = [threading.Thread(target=run, args=(c,)) for c in range(num_chunks)]
    for t in ts:
        t.start()
    for t in ts:
        t.join()
    if errors:
        raise errors[0]
    return rel, offsets


class CudaRadixJoin:
    """CudaRadixJoin (cuda_radix_join.rs:116-164)."""

    def __init__(self, radix_pass, radix_bits, hashing_scheme, grid_size,
                 block_size):
        self.h = C.c_void_p()
        self.grid_size, self.block_size = grid_size, block_size
        _check(lib().fi_cuda_radix_join_new(
            C.c_int(int(radix_pass)), radix_bits.c(), C.c_int(int(hashing_scheme)),
            C.c_uint32(grid_size), C.c_uint32(block_size), C.byref(self.h)))

    def __del__(self):
        if getattr(self, "h", None) and _lib is not None:
            _lib.fi_cuda_radix_join_free(self.h)
            self.h = None

    def status(self):
        _check(lib().fi_cuda_radix_join_status(self.h))

    def join(self, build_rel, probe_rel, result_set, task_assignments,
             match_count=None, stream=None):
        f = getattr(lib(), "fi_cuda_radix_join_" + _sfx(build_rel.dtype))
        _check(f(self.h, C.byref(build_rel.c), C.byref(probe_rel.c),
                 _ptr(result_set), C.c_uint64(result_set.numel()),
                 _ptr(task_assignments), C.c_uint64(task_assignments.numel()),
                 _ptr(match_count), _stream(stream)))


# ---------------------------------------------------------------------------
# CudaHashJoin (no partitioning)
# ---------------------------------------------------------------------------
class HashTable:
    """HashTable::new_on_gpu (no_partitioning_join.rs:579-625)."""

    def __init__(self, size, dtype, mem_len=None, stream=None):
        mem_len = size if mem_len is None else mem_len
        self.dtype = dtype
        self.size = size
        self.mem = torch.empty((max(mem_len, 1), 2), dtype=dtype, device="cuda")
        f = getattr(lib(), "fi_hash_table_init_" + _sfx(dtype))
        _check(f(_ptr(self.mem), C.c_uint64(mem_len), _stream(stream)))


class CudaHashJoin:
    """CudaHashJoin built like CudaHashJoinBuilder (no_partitioning_join.rs)."""

    def __init__(self, hashing_scheme, hash_table, build_dim=(1, 1),
                 probe_dim=(1, 1), is_selective=False):
        self.ht = hash_table
        self.h = C.c_void_p()
        _check(lib().fi_cuda_hash_join_new(
            C.c_int(int(hashing_scheme)), C.c_int(1 if is_selective else 0),
            _ptr(hash_table.mem), C.c_uint64(hash_table.mem.shape[0]),
            C.c_uint64(hash_table.size), C.c_uint32(build_dim[0]),
            C.c_uint32(build_dim[1]), C.c_uint32(probe_dim[0]),
            C.c_uint32(probe_dim[1]), C.byref(self.h)))

    def __del__(self):
        if getattr(self, "h", None) and _lib is not None:
            _lib.fi_cuda_hash_join_free(self.h)
            self.h = None

    def build(self, join_attr, payload_attr, stream=None):
        f = getattr(lib(), "fi_cuda_hash_join_build_" + _sfx(join_attr.dtype))
        _check(f(self.h, _ptr(join_attr), _ptr(payload_attr),
                 C.c_uint64(join_attr.numel()), _stream(stream)))

    def set_probe_grouping(self, enable=True, slice_tuples=1 << 27):
        """Probe-side grouping by table region (fi_cuda_hash_join_set_probe_grouping;
        no counterpart in the reference): on by default."""
        _check(lib().fi_cuda_hash_join_set_probe_grouping(
            self.h, C.c_int(1 if enable else 0), C.c_uint64(slice_tuples)))

    def set_build_grouping(self, enable=True, slice_tuples=1 << 27):
        """Build-side grouping by table region (fi_cuda_hash_join_set_build_grouping;
        no counterpart in the reference): on by default."""
        _check(lib().fi_cuda_hash_join_set_build_grouping(
            self.h, C.c_int(1 if enable else 0), C.c_uint64(slice_tuples)))

    def status(self):
        """Raises the device-side error (a bounded wait that gave up) of the
        grouped build and probe since the last call
        (fi_cuda_hash_join_status)."""
        _check(lib().fi_cuda_hash_join_status(self.h))

    def probe_sum(self, join_attr, payload_attr, result_set, stream=None):
        f = getattr(lib(), "fi_cuda_hash_join_probe_sum_" + _sfx(join_attr.dtype))
        _check(f(self.h, _ptr(join_attr), _ptr(payload_attr),
                 C.c_uint64(join_attr.numel()), _ptr(result_set),
                 C.c_uint64(result_set.numel()), _stream(stream)))


class CpuHashTable:
    """HashTable::new_on_cpu (no_partitioning_join.rs:568-581): `mem_len`
    host entries of {key, value} (a (mem_len, 2) numpy array of the key
    type) whose keys are the null key; `size` is the size used for hashing."""

    def __init__(self, size, dtype, mem_len=None):
        import numpy as np
        mem_len = size if mem_len is None else mem_len
        if mem_len < size:
            raise SqlOpsError(-1, "Provided memory must be larger than hash table size")
        self.dtype = np.dtype(dtype)
        self.size = size
        self.mem = np.empty((max(mem_len, 1), 2), self.dtype)
        f = getattr(lib(), "fi_cpu_hash_table_init_" + _cpu_sfx(self.mem))
        _check(f(C.c_void_p(self.mem.ctypes.data), C.c_uint64(mem_len)))
        self.mem_len = mem_len


def _cpu_sfx(a):
    import numpy as np
    return "int32" if a.dtype == np.int32 else "int64"


class CpuHashJoin:
    """CpuHashJoin built like CpuHashJoinBuilder (no_partitioning_join.rs:
    153-304, 740-772): build and probe_sum of numpy columns on the host.
    Several threads may build (or probe) disjoint slices through one join."""

    def __init__(self, hashing_scheme, hash_table, is_selective=False):
        self.ht = hash_table
        self.h = C.c_void_p()
        _check(lib().fi_cpu_hash_join_new(
            C.c_int(int(hashing_scheme)), C.c_int(1 if is_selective else 0),
            C.c_void_p(hash_table.mem.ctypes.data), C.c_uint64(hash_table.mem_len),
            C.c_uint64(hash_table.size), C.byref(self.h)))

    def __del__(self):
        if getattr(self, "h", None) and _lib is not None:
            _lib.fi_cpu_hash_join_free(self.h)
            self.h = None

    def _cols(self, join_attr, payload_attr):
        import numpy as np
        if len(join_attr) != len(payload_attr):
            raise SqlOpsError(-1, "Join and payload attributes have different sizes")
        if join_attr.dtype != self.ht.dtype or payload_attr.dtype != self.ht.dtype:
            raise SqlOpsError(-1, "attributes must have the hash table's key type")
        return (np.ascontiguousarray(join_attr), np.ascontiguousarray(payload_attr))

    def build(self, join_attr, payload_attr):
        k, p = self._cols(join_attr, payload_attr)
        f = getattr(lib(), "fi_cpu_hash_join_build_" + _cpu_sfx(k))
        _check(f(self.h, C.c_void_p(k.ctypes.data), C.c_void_p(p.ctypes.data),
                 C.c_uint64(len(k))))

    def probe_sum(self, join_attr, payload_attr, join_result=0):
        """Returns join_result plus (wrapping mod 2^64) the payloads of all
        matching probe tuples."""
        k, p = self._cols(join_attr, payload_attr)
        f = getattr(lib(), "fi_cpu_hash_join_probe_sum_" + _cpu_sfx(k))
        acc = C.c_uint64(int(join_result) & 0xFFFFFFFFFFFFFFFF)
        _check(f(self.h, C.c_void_p(k.ctypes.data), C.c_void_p(p.ctypes.data),
                 C.c_uint64(len(k)), C.byref(acc)))
        return acc.value


def cpu_hash_join_sum(build_key, build_pay, probe_key, probe_pay, hashing_scheme,
                      size, threads=1, is_selective=False, mem_len=None):
    """Whole no-partitioning join on `threads` host threads, as the
    reference's cpu_hash_join benchmark runs it: the threads build disjoint
    slices into one shared table, then probe disjoint slices; returns the
    u64 sum of the matched probe payloads."""
    import threading
    ht = CpuHashTable(size, build_key.dtype, mem_len)
    hj = CpuHashJoin(hashing_scheme, ht, is_selective)
    sums, errors = [0] * threads, []

    def slices(n):
        return [(n * t // threads, n * (t + 1) // threads) for t in range(threads)]

    def run(fn):
        ts = [threading.Thread(target=fn, args=(t,)) for t in range(threads)]
        for t in ts:
            t.start()
        for t in ts:
            t.join()
        if errors:
            raise errors[0]

    def build(t):
        try:
            b, e = slices(len(build_key))[t]
            hj.build(build_key[b:e], build_pay[b:e])
        except Exception as ex:  # reported after the join
            errors.append(ex)

    def probe(t):
        try:
            b, e = slices(len(probe_key))[t]
            sums[t] = hj.probe_sum(probe_key[b:e], probe_pay[b:e])
        except Exception as ex:
            errors.append(ex)

    run(build)
    run(probe)
    return sum(sums) & 0xFFFFFFFFFFFFFFFF


# ---------------------------------------------------------------------------
# Radix exchange between GPUs (exchange.cu)
# ---------------------------------------------------------------------------
EXCHANGE_MAX_RANKS = 64
IPC_HANDLE_BYTES = 64


class ExchangeDest(C.Structure):
    """fi_exchange_dest: one destination's receive columns (device or peer
    pointers), the sender's first slot there and the columns' length."""
    _fields_ = [("key", C.c_void_p), ("pay", C.c_void_p), ("base", C.c_uint64),
                ("cap", C.c_uint64)]


def exchange_histogram(keys, shift, exchange_bits, counts=None, stream=None):
    """counts[d] = number of keys whose bits [shift, shift + exchange_bits)
    equal d (an int64 device tensor of 2^exchange_bits entries)."""
    F = 1 << exchange_bits
    if counts is None:
        counts = torch.empty(F, dtype=torch.int64, device=keys.device)
    f = getattr(lib(), "fi_exchange_histogram_" + _sfx(keys.dtype))
    _check(f(_ptr(keys), C.c_uint64(keys.numel()), C.c_uint32(shift),
             C.c_uint32(exchange_bits), _ptr(counts), _stream(stream)))
    return counts


def exchange_scatter(keys, pays, shift, exchange_bits, dests, cursors=None,
                     status=None, stream=None):
    """Fused partition + send: dests is a list of 2^exchange_bits tuples
    (key_ptr, pay_ptr, base, cap) -- device or peer pointers as ints.
    Returns the cursors workspace (per destination: tuples sent)."""
    F = 1 << exchange_bits
    if len(dests) != F:
        raise SqlOpsError(-1, "need %d destinations, got %d" % (F, len(dests)))
    arr = (ExchangeDest * F)(*[ExchangeDest(int(k), int(p), int(b), int(c))
                               for k, p, b, c in dests])
    if cursors is None:
        cursors = torch.empty(F, dtype=torch.int64, device=keys.device)
    f = getattr(lib(), "fi_exchange_scatter_" + _sfx(keys.dtype))
    _check(f(_ptr(keys), _ptr(pays), C.c_uint64(keys.numel()), C.c_uint32(shift),
             C.c_uint32(exchange_bits), arr, _ptr(cursors), _ptr(status),
             _stream(stream)))
    return cursors


def ipc_handle(t):
    """(handle bytes, byte offset of t in its allocation): the CUDA IPC
    handle of the whole allocation holding tensor t."""
    buf = C.create_string_buffer(IPC_HANDLE_BYTES)
    off = C.c_uint64(0)
    _check(lib().fi_ipc_get_handle(_ptr(t), buf, C.byref(off)))
    return buf.raw, off.value


def ipc_open(handle):
    """Opens another process's IPC handle; returns the allocation's base
    device pointer (open each allocation once per process)."""
    out = C.c_void_p()
    _check(lib().fi_ipc_open_handle(C.create_string_buffer(bytes(handle),
                                                           IPC_HANDLE_BYTES),
                                    C.byref(out)))
    return out.value


def ipc_close(ptr):
    _check(lib().fi_ipc_close_handle(C.c_void_p(ptr)))


# ---------------------------------------------------------------------------
# gpu_radix_join execution method
# ---------------------------------------------------------------------------
class RadixJoinEngine:
    """Whole radix join (pass 1, optional pass 2, per-partition join)."""

    def __init__(self, max_build, max_probe, dtype, radix_bits,
                 hashing_scheme=HashingScheme.BucketChaining):
        self.dtype = dtype
        self.h = C.c_void_p()
        _check(lib().fi_radix_join_engine_new(
            C.c_uint64(max_build), C.c_uint64(max_probe),
            C.c_uint32(_tuple_bytes(dtype)), radix_bits.c(),
            C.c_int(int(hashing_scheme)), C.byref(self.h)))
        self.result = torch.zeros(2, dtype=torch.int64, device="cuda")

    def __del__(self):
        if getattr(self, "h", None) and _lib is not None:
            _lib.fi_radix_join_engine_free(self.h)
            self.h = None

    def workspace_bytes(self):
        return lib().fi_radix_join_engine_workspace_bytes(self.h)

    PHASE_EVENTS = 11

    def set_events(self, events):
        """Records torch.cuda.Event objects at the phase boundaries of every
        run (see fi_radix_join_engine_set_events); None stops recording."""
        if events is None:
            _check(lib().fi_radix_join_engine_set_events(self.h, None, 0))
            self._events = None
            return
        for e in events:  # torch creates an event's handle at its first record
            if not e.cuda_event:
                e.record()
        arr = (C.c_void_p * len(events))(*[e.cuda_event for e in events])
        self._events = (events, arr)
        _check(lib().fi_radix_join_engine_set_events(self.h, arr, len(events)))

    def last_launches(self):
        return lib().fi_radix_join_engine_last_launches(self.h)

    def status(self):
        _check(lib().fi_radix_join_engine_status(self.h))

    def run_async(self, build_key, build_pay, probe_key, probe_pay, stream=None):
        """Enqueues the join; the device tensor self.result = [sum, count]."""
        f = getattr(lib(), "fi_radix_join_engine_run_" + _sfx(build_key.dtype))
        _check(f(self.h, _ptr(build_key), _ptr(build_pay),
                 C.c_uint64(build_key.numel()), _ptr(probe_key), _ptr(probe_pay),
                 C.c_uint64(probe_key.numel()), _ptr(self.result), _stream(stream)))
        return self.result

    def run(self, build_key, build_pay, probe_key, probe_pay, stream=None):
        self.run_async(build_key, build_pay, probe_key, probe_pay, stream)
        r = self.result.cpu()
        return int(r[0]), int(r[1]) & ((1 << 64) - 1)

    def run_host(self, build_key, build_pay, probe_key, probe_pay, stream=None):
        """Host (pinned) columns in, (sum, count) out; synchronous."""
        res = _JoinResultC()
        f = getattr(lib(), "fi_radix_join_engine_run_host_" + _sfx(build_key.dtype))
        _check(f(
            self.h, _ptr(build_key), _ptr(build_pay),
            C.c_uint64(build_key.numel()), _ptr(probe_key), _ptr(probe_pay),
            C.c_uint64(probe_key.numel()), C.byref(res), _stream(stream)))
        return res.sum, res.count

    def run_hybrid(self, build_key, build_pay, probe_key, probe_pay, threads=0,
                   stream=None):
        """Hybrid join: host columns in; the first pass on `threads` host
        threads (0 = all), the second pass and the join on the GPU;
        (sum, count) out; synchronous."""
        res = _JoinResultC()
        f = getattr(lib(), "fi_radix_join_engine_run_hybrid_" + _sfx(build_key.dtype))
        _check(f(self.h, _ptr(build_key), _ptr(build_pay), C.c_uint64(build_key.numel()),
                 _ptr(probe_key), _ptr(probe_pay), C.c_uint64(probe_key.numel()),
                 C.c_uint32(threads), C.byref(res), _stream(stream)))
        return res.sum, res.count

    def set_plan(self, radix_bits, hashing_scheme=HashingScheme.BucketChaining,
                 join_block=0, scatter=0):
        """Plan of the following runs, within the engine's creation bits
        (fi_radix_join_engine_set_plan)."""
        plan = _JoinPlanC(radix_bits.c(), int(hashing_scheme), join_block, scatter)
        _check(lib().fi_radix_join_engine_set_plan(self.h, C.byref(plan)))

    def build(self, build_key, build_pay, stream=None):
        """Partitions the build relation; it stays resident until the next
        build or plan."""
        f = getattr(lib(), "fi_radix_join_engine_build_" + _sfx(build_key.dtype))
        _check(f(self.h, _ptr(build_key), _ptr(build_pay),
                 C.c_uint64(build_key.numel()), _stream(stream)))

    def probe_async(self, probe_key, probe_pay, result=None, stream=None):
        """Joins a probe relation (or a slice) against the resident build
        side; result (device int64[2]) = [sum, count] of this probe."""
        result = self.result if result is None else result
        f = getattr(lib(), "fi_radix_join_engine_probe_" + _sfx(probe_key.dtype))
        _check(f(self.h, _ptr(probe_key), _ptr(probe_pay),
                 C.c_uint64(probe_key.numel()), _ptr(result), _stream(stream)))
        return result

    def probe(self, probe_key, probe_pay, stream=None):
        r = self.probe_async(probe_key, probe_pay, stream=stream).cpu()
        return int(r[0]), int(r[1]) & ((1 << 64) - 1)

    def run_streamed(self, build_key, build_pay, probe_key, probe_pay,
                     block_tuples=0, stream=None):
        """Out-of-core join: host (pinned) columns, the first pass streamed
        over the host link in blocks of block_tuples (0 = library default);
        (sum, count) out; synchronous."""
        res = _JoinResultC()
        f = getattr(lib(), "fi_radix_join_engine_run_streamed_" + _sfx(build_key.dtype))
        _check(f(self.h, _ptr(build_key), _ptr(build_pay),
                 C.c_uint64(build_key.numel()), _ptr(probe_key), _ptr(probe_pay),
                 C.c_uint64(probe_key.numel()), C.c_uint64(block_tuples),
                 C.byref(res), _stream(stream)))
        return res.sum, res.count


class _BatchJobC(C.Structure):
    _fields_ = [("build_key", C.c_void_p), ("build_pay", C.c_void_p),
                ("probe_key", C.c_void_p), ("probe_pay", C.c_void_p),
                ("build_len", C.c_uint64), ("probe_len", C.c_uint64),
                ("radix_bits", C.c_int32)]


class JoinBatch:
    """Many small joins of one tuple type run at once (fi_join_batch_*)."""

    def __init__(self, dtype, max_jobs=256, max_tuples=1 << 24):
        self.dtype = dtype
        self.h = C.c_void_p()
        _check(lib().fi_join_batch_new(C.c_uint32(_tuple_bytes(dtype)),
                                       C.c_uint32(max_jobs), C.c_uint64(max_tuples),
                                       C.byref(self.h)))

    def __del__(self):
        if getattr(self, "h", None) and _lib is not None:
            _lib.fi_join_batch_free(self.h)
            self.h = None

    def device_bytes(self):
        lib().fi_join_batch_device_bytes.restype = C.c_uint64
        return lib().fi_join_batch_device_bytes(self.h)

    def run(self, jobs):
        """jobs: list of (build_key, build_pay, probe_key, probe_pay[, bits])
        device tensors; returns [(sum, count)] per job."""
        arr = (_BatchJobC * max(len(jobs), 1))()
        for i, j in enumerate(jobs):
            bk, bp, pk, pp = j[:4]
            bits = j[4] if len(j) > 4 else -1
            arr[i] = _BatchJobC(_ptr(bk).value, _ptr(bp).value, _ptr(pk).value,
                                _ptr(pp).value, bk.numel(), pk.numel(), bits)
        res = (_JoinResultC * max(len(jobs), 1))()
        _check(lib().fi_join_batch_run(self.h, arr, C.c_uint32(len(jobs)), res))
        return [(res[i].sum, res[i].count) for i in range(len(jobs))]


class _ServerConfigC(C.Structure):
    _fields_ = [("hbm_budget_bytes", C.c_uint64), ("workers", C.c_uint32),
                ("small_tuples", C.c_uint64), ("max_batch_jobs", C.c_uint32),
                ("batch_tuples", C.c_uint64), ("batch_wait_us", C.c_uint32),
                ("max_build", C.c_uint64), ("probe_slice", C.c_uint64)]


class _RequestC(C.Structure):
    _fields_ = [("tuple_bytes", C.c_uint32), ("source", C.c_uint32),
                ("build_len", C.c_uint64), ("probe_len", C.c_uint64),
                ("build_key", C.c_void_p), ("build_pay", C.c_void_p),
                ("probe_key", C.c_void_p), ("probe_pay", C.c_void_p),
                ("seed", C.c_uint64), ("zipf_s", C.c_double)]


class _ResponseC(C.Structure):
    _fields_ = [("status", C.c_int32), ("batched", C.c_uint32),
                ("result", _JoinResultC), ("batch_jobs", C.c_uint32),
                ("reserved", C.c_uint32), ("queue_us", C.c_double),
                ("latency_us", C.c_double)]


class _ServerStatsC(C.Structure):
    _fields_ = [(n, C.c_uint64) for n in (
        "submitted", "completed", "batches", "batched_jobs", "engine_runs",
        "reserved_bytes", "peak_reserved_bytes", "fixed_bytes", "arena_bytes")] + [
        (n, C.c_double) for n in ("engine_busy_us", "batch_busy_us", "enqueue_us")] + [
        ("workers", C.c_uint64)]


class JoinSource(enum.IntEnum):
    Device = 0
    Host = 1
    Synthetic = 2


class JoinServer:
    """Continuous-batching join server (fi_join_server_*).  submit() returns
    a ticket at once; wait()/poll() hand over a dict with status, sum,
    count, batched, batch_jobs, queue_us and latency_us."""

    def __init__(self, hbm_budget_bytes=0, workers=0, small_tuples=0,
                 max_batch_jobs=0, batch_tuples=0, batch_wait_us=0, max_build=0,
                 probe_slice=0):
        cfg = _ServerConfigC(hbm_budget_bytes, workers, small_tuples, max_batch_jobs,
                             batch_tuples, batch_wait_us, max_build, probe_slice)
        self.h = C.c_void_p()
        self._keep = {}
        _check(lib().fi_join_server_new(C.byref(cfg), C.byref(self.h)))

    def close(self):
        if getattr(self, "h", None) and _lib is not None:
            _lib.fi_join_server_free(self.h)
            self.h = None

    def __del__(self):
        self.close()

    def submit(self, tuple_bytes=16, source=JoinSource.Synthetic, build_len=0,
               probe_len=0, columns=None, seed=0, zipf_s=0.0):
        """columns: (build_key, build_pay, probe_key, probe_pay) tensors for
        the device and host sources (kept alive until the response)."""
        ptrs = [None] * 4
        if columns is not None:
            ptrs = [c.data_ptr() for c in columns]
            build_len, probe_len = columns[0].numel(), columns[2].numel()
        req = _RequestC(tuple_bytes, int(source), build_len, probe_len, *ptrs, seed,
                        zipf_s)
        t = C.c_uint64()
        _check(lib().fi_join_server_submit(self.h, C.byref(req), C.byref(t)))
        if columns is not None:
            self._keep[t.value] = columns
        return t.value

    @staticmethod
    def _resp(r):
        return {"status": r.status, "sum": r.result.sum, "count": r.result.count,
                "batched": bool(r.batched), "batch_jobs": r.batch_jobs,
                "queue_us": r.queue_us, "latency_us": r.latency_us}

    def wait(self, ticket):
        r = _ResponseC()
        _check(lib().fi_join_server_wait(self.h, C.c_uint64(ticket), C.byref(r)))
        self._keep.pop(ticket, None)
        return self._resp(r)

    def poll(self, ticket):
        r = _ResponseC()
        done = C.c_int()
        _check(lib().fi_join_server_poll(self.h, C.c_uint64(ticket), C.byref(done),
                                         C.byref(r)))
        if not done.value:
            return None
        self._keep.pop(ticket, None)
        return self._resp(r)

    def stats(self):
        st = _ServerStatsC()
        _check(lib().fi_join_server_stats_get(self.h, C.byref(st)))
        return {n: getattr(st, n) for n, _ in _ServerStatsC._fields_}


class _TunedPlanC(C.Structure):
    _fields_ = [("batched", C.c_uint32), ("radix_bits", _RadixBitsC),
                ("hashing_scheme", C.c_int), ("join_block", C.c_uint32),
                ("scatter", C.c_uint32)]


def autotune_plan(tuple_bytes, build_len, probe_len, skew=0, small_tuples=0):
    """The autotuner's plan as a dict (fi_autotune_plan)."""
    p = _TunedPlanC()
    _check(lib().fi_autotune_plan(C.c_uint32(tuple_bytes), C.c_uint64(build_len),
                                  C.c_uint64(probe_len), C.c_uint32(skew),
                                  C.c_uint64(small_tuples), C.byref(p)))
    bits = [b for b in p.radix_bits.pass_bits if b >= 0]
    return {"batched": bool(p.batched), "bits": tuple(bits),
            "scheme": HashingScheme(p.hashing_scheme), "join_block": p.join_block,
            "scatter": p.scatter}


def autotune_load(path):
    _check(lib().fi_autotune_load(None if path is None else path.encode()))


# ---------------------------------------------------------------------------
# seeded generator
# ---------------------------------------------------------------------------
def _ctype(dtype):
    return C.c_int32 if dtype == torch.int32 else C.c_int64


def gen_primary_keys(t, seed, base=1, stream=None):
    f = getattr(lib(), "fi_datagen_primary_keys_" + _sfx(t.dtype))
    _check(f(_ptr(t), C.c_uint64(t.numel()), C.c_uint64(seed),
             _ctype(t.dtype)(base), _stream(stream)))
    return t


def gen_uniform_foreign_keys(t, pk_n, seed, base=1, stream=None):
    f = getattr(lib(), "fi_datagen_uniform_foreign_keys_" + _sfx(t.dtype))
    _check(f(_ptr(t), C.c_uint64(t.numel()), C.c_uint64(pk_n), C.c_uint64(seed),
             _ctype(t.dtype)(base), _stream(stream)))
    return t


def gen_zipf_foreign_keys(t, pk_n, s, seed, pk_seed, base=1, stream=None):
    f = getattr(lib(), "fi_datagen_zipf_foreign_keys_" + _sfx(t.dtype))
    _check(f(_ptr(t), C.c_uint64(t.numel()), C.c_uint64(pk_n), C.c_double(s),
             C.c_uint64(seed), C.c_uint64(pk_seed), _ctype(t.dtype)(base),
             _stream(stream)))
    return t


def gen_uniform_u64_keys(t, seed, stream=None):
    _check(lib().fi_datagen_uniform_u64_keys(_ptr(t), C.c_uint64(t.numel()),
                                             C.c_uint64(seed), _stream(stream)))
    return t


def null_keys(t, selectivity, seed, base=1, stream=None):
    """Join selectivity in percent (fi_datagen_null_keys): each key of `t`
    stays with probability (selectivity+1)/101, a function of (seed, key -
    base), and becomes the null key (-1) otherwise; selectivity 100 keeps
    all keys.  Apply it to primary keys base..base+n-1."""
    f = getattr(lib(), "fi_datagen_null_keys_" + _sfx(t.dtype))
    _check(f(_ptr(t), C.c_uint64(t.numel()), C.c_uint32(selectivity),
             C.c_uint64(seed), _ctype(t.dtype)(base), _stream(stream)))
    return t


# ---------------------------------------------------------------------------
# data sets and relation files
# ---------------------------------------------------------------------------
class Dataset(enum.IntEnum):
    """The reference's named data sets (radix-join/src/main.rs:657-760)."""
    Blanas = 0
    Blanas4MB = 1
    Kim = 2
    Test = 3
    Lutz2Gv32G = 4
    Lutz32Gv32G = 5


def dataset_shape(dataset, dtype):
    """(|R|, |S|) of a named data set for tuples of two `dtype` values."""
    b, p = C.c_uint64(), C.c_uint64()
    _check(lib().fi_dataset_shape(int(dataset), _tuple_bytes(dtype), C.byref(b),
                                  C.byref(p)))
    return b.value, p.value


def gen_dataset(dataset, dtype, selectivity=100, seed=0, stream=None):
    """Device columns (build_key, build_pay, probe_key, probe_pay) of a named
    data set: primary keys a seeded permutation of 1..|R| with
    (100 - selectivity)% nulled, foreign keys uniform over 1..|R|, payload =
    key (the reference leaves the payload columns unset for these sets)."""
    nb, npr = dataset_shape(dataset, dtype)
    rk = torch.empty(nb, dtype=dtype, device="cuda")
    sk = torch.empty(npr, dtype=dtype, device="cuda")
    gen_primary_keys(rk, seed, base=1, stream=stream)
    null_keys(rk, selectivity, seed + 7, base=1, stream=stream)
    gen_uniform_foreign_keys(sk, nb, seed + 1, base=1, stream=stream)
    return rk, rk.clone(), sk, sk.clone()


def relation_file_len(path):
    """Tuples in a relation file (fi_relation_file_len)."""
    n = C.c_uint64()
    _check(lib().fi_relation_file_len(os.fsencode(path), C.byref(n)))
    return n.value


def read_relation_file(path, dtype=torch.int64, pin=None):
    """(keys, payloads) of a relation file as host tensors, pinned when a GPU
    is present (pin=None) so that the engine's host entry points copy them
    directly."""
    if pin is None:
        pin = torch.cuda.is_available()
    n = relation_file_len(path)
    keys = torch.empty(n, dtype=dtype, pin_memory=pin)
    pays = torch.empty(n, dtype=dtype, pin_memory=pin)
    f = getattr(lib(), "fi_relation_file_read_" + _sfx(dtype))
    _check(f(os.fsencode(path), C.c_void_p(keys.data_ptr() if n else 0),
             C.c_void_p(pays.data_ptr() if n else 0), C.c_uint64(n)))
    return keys, pays


def load_join_data(inner_path, outer_path, dtype=torch.int64, pin=None):
    """build_with_files (data-store/src/join_data.rs:173-280): the inner
    (build) and outer (probe) relations as host columns (build_key,
    build_pay, probe_key, probe_pay)."""
    rk, rp = read_relation_file(inner_path, dtype, pin)
    sk, sp = read_relation_file(outer_path, dtype, pin)
    return rk, rp, sk, sp
