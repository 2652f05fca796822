"""ctypes wrapper of _build/libref_gpu.so: the reference's own GPU kernels
(sql-ops/cudautils/radix_partition.cu, radix_join.cu), compiled for sm_100a
from the reference sources and launched with the reference's argument
structs, grids and shared-memory sizes (harness.cu).

Benchmark and test infrastructure only: it measures the reference's kernels
beside this repository's on the same B200 and gives the join parity tests a
further pin.  Every launch is checked first (``*_prepare`` in harness.cu) so
that none of the reference's device asserts can fire and no unchecked
shared-memory index leaves its array; a request that fails a check raises
RefGpuError without launching anything.

Tensors are torch CUDA tensors; relations are [n, 2] AoS tuples; offsets are
int64 tensors holding the u64 offsets.
"""
import ctypes as C
import os

import torch

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "_build", "libref_gpu.so")

NC, LASWWC = 0, 1
PERFECT, CHAINING = 0, 1

_lib = None


class RefGpuError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__("%s (%d)" % (msg, code))
        self.code = code


def available():
    return os.path.exists(LIB_PATH)


def lib():
    global _lib
    if _lib is None:
        if not available():
            raise RefGpuError(-4, "reference GPU library not built: " + LIB_PATH)
        L = C.CDLL(LIB_PATH)
        L.rg_last_error.restype = C.c_char_p
        L.rg_padding_len.restype = C.c_uint32
        _lib = L
    return _lib


def _check(rc):
    if rc != 0:
        raise RefGpuError(rc, lib().rg_last_error().decode())


def _p(t):
    return C.c_void_p(t.data_ptr())


def _stream(stream):
    s = stream if stream is not None else torch.cuda.current_stream()
    return C.c_void_p(s.cuda_stream)


def _kb(t):
    if t.dtype not in (torch.int32, torch.int64):
        raise RefGpuError(-1, "keys must be int32 or int64")
    return t.element_size()


def padding_len(dtype):
    return int(lib().rg_padding_len(C.c_int(4 if dtype == torch.int32 else 8)))


def chunked_prefix_sum(keys, chunks, bits, ignore=0, block=1024, out=None,
                       stream=None):
    """gpu_chunked_prefix_sum_*: offsets[c * 2^bits + p] (u64 in int64)."""
    n = chunks << bits
    if out is None:
        out = torch.empty(n, dtype=torch.int64, device=keys.device)
    if out.numel() < n or out.dtype != torch.int64:
        raise RefGpuError(-1, "offsets need %d int64 slots" % n)
    _check(lib().rg_chunked_prefix_sum(
        C.c_int(_kb(keys)), _p(keys), C.c_uint64(keys.numel()), C.c_uint32(chunks),
        C.c_uint32(bits), C.c_uint32(ignore), _p(out), C.c_uint32(block),
        _stream(stream)))
    return out


class Partition:
    """One checked scatter call (NC or LASWWC) of `keys`/`pays` into
    `relation` with the reference prefix-sum `offsets` of the same keys."""

    def __init__(self, variant, keys, pays, chunks, bits, offsets, relation,
                 ignore=0, block=1024):
        kb = _kb(keys)
        if relation.dim() != 2 or relation.shape[1] != 2 or relation.dtype != keys.dtype:
            raise RefGpuError(-1, "relation must be [n, 2] of the key type")
        if offsets.numel() < (chunks << bits):
            raise RefGpuError(-1, "offsets too short")
        self.args = (C.c_int(variant), C.c_int(kb), _p(keys), _p(pays),
                     C.c_uint64(keys.numel()), C.c_uint32(chunks), C.c_uint32(bits),
                     C.c_uint32(ignore), _p(offsets), _p(relation),
                     C.c_uint64(relation.shape[0]), C.c_uint32(block))
        torch.cuda.synchronize()
        _check(lib().rg_partition_prepare(*self.args))

    def launch(self, stream=None):
        _check(lib().rg_partition(*self.args, _stream(stream)))


class Join:
    """One checked reference join (assign_tasks + the shared-memory join) of
    two contiguous partitioned relations; `result` (grid * block int64) is
    accumulated with += as in the reference, `tasks` gets grid + 1 u32."""

    def __init__(self, scheme, build_rel, build_off, build_len, probe_rel,
                 probe_off, probe_len, bits, ignore, grid, block):
        kb = _kb(build_rel)
        if probe_rel.dtype != build_rel.dtype:
            raise RefGpuError(-1, "build and probe types differ")
        dev = build_rel.device
        self.result = torch.zeros(grid * block, dtype=torch.int64, device=dev)
        self.tasks = torch.zeros(grid + 1, dtype=torch.int32, device=dev)
        self.args = (C.c_int(scheme), C.c_int(kb), _p(build_rel), _p(build_off),
                     C.c_uint64(build_len), _p(probe_rel), _p(probe_off),
                     C.c_uint64(probe_len), C.c_uint32(bits), C.c_uint32(ignore),
                     C.c_uint32(grid), C.c_uint32(block), _p(self.result),
                     _p(self.tasks))
        torch.cuda.synchronize()
        _check(lib().rg_join_prepare(*self.args))

    def launch(self, stream=None):
        _check(lib().rg_join(*self.args, _stream(stream)))

    def sum(self):
        """Wrapping u64 sum of the per-thread results."""
        torch.cuda.synchronize()
        return int(self.result.sum().item()) & ((1 << 64) - 1)
