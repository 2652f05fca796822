// C ABI of the B200 radix-partition / hash-join operators (include/fi_sqlops.h).
//
// Host side of the drop-in boundary: argument validation with the reference's
// error kinds and messages (sql-ops/src/partition/gpu_radix_partition.rs,
// sql-ops/src/join/cuda_radix_join.rs, sql-ops/src/join/no_partitioning_join.rs),
// device scratch owned by the handles, and the kernel launches.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <string>

#include "../../include/fi_sqlops.h"
#include "api_internal.h"
#include "common.cuh"
#include "kernels.h"

namespace fi {

static thread_local std::string g_last_error;

int set_error(int code, const char *fmt, ...) {
  char buf[512];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(buf, sizeof(buf), fmt, ap);
  va_end(ap);
  g_last_error = buf;
  return code;
}

int cuda_error(cudaError_t e, const char *what) {
  if (e == cudaErrorMemoryAllocation)
    return set_error(FI_ERR_OUT_OF_MEMORY, "%s: %s", what, cudaGetErrorString(e));
  return set_error(FI_ERR_CUDA, "%s: %s", what, cudaGetErrorString(e));
}

int device_sm_count() {
  int dev = 0, v = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&v, cudaDevAttrMultiProcessorCount, dev);
  return v > 0 ? v : 1;
}

int device_max_smem_optin() {
  int dev = 0, v = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&v, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
  return v > 0 ? v : 48 * 1024;
}

// Grows a device buffer to at least `bytes` (contents discarded).
int DevBuf::reserve(size_t bytes, bool zero) {
  if (bytes <= size) return FI_OK;
  if (ptr) cudaFree(ptr);
  ptr = nullptr;
  size = 0;
  cudaError_t e = cudaMalloc(&ptr, bytes);
  if (e != cudaSuccess) {
    ptr = nullptr;
    return cuda_error(e, "device allocation");
  }
  size = bytes;
  if (zero) {
    e = cudaMemset(ptr, 0, bytes);
    if (e != cudaSuccess) return cuda_error(e, "device memset");
  }
  return FI_OK;
}

void DevBuf::release() {
  if (ptr) cudaFree(ptr);
  ptr = nullptr;
  size = 0;
}

int read_and_clear_status(DevBuf &status) {
  if (!status.ptr) return FI_OK;
  cudaError_t e = cudaDeviceSynchronize();
  if (e != cudaSuccess) return cuda_error(e, "device synchronize");
  int v = 0;
  e = cudaMemcpy(&v, status.ptr, sizeof(int), cudaMemcpyDeviceToHost);
  if (e != cudaSuccess) return cuda_error(e, "status read");
  if (v != 0) {
    cudaMemset(status.ptr, 0, sizeof(int));
    if (v == FI_ERR_TIMEOUT)
      return set_error(v, "a bounded device-side wait gave up");
    if (v == FI_ERR_CAPACITY)
      return set_error(v, "a kernel met a capacity limit (partition cursors "
                          "outside the relation or a key outside the hash "
                          "table)");
    return set_error(FI_ERR_RUNTIME, "device-side error %d", v);
  }
  return FI_OK;
}

uint32_t padding_len(uint32_t tuple_bytes) {
  return kPaddingBytes / tuple_bytes;
}

}  // namespace fi

using namespace fi;

// ---------------------------------------------------------------------------
// errors, version, host-side helpers
// ---------------------------------------------------------------------------
extern "C" const char *fi_last_error(void) { return g_last_error.c_str(); }

extern "C" const char *fi_version(void) { return "fi_sqlops 0.1.0 (sm_100a)"; }

extern "C" int fi_input_chunk_size(uint64_t data_len, uint32_t num_chunks,
                                   uint32_t key_bytes, uint64_t *chunk_len) {
  if (num_chunks == 0 || (key_bytes != 4 && key_bytes != 8) || !chunk_len)
    return set_error(FI_ERR_INVALID_ARGUMENT, "invalid chunking arguments");
  const uint64_t mask = ~((uint64_t)(kAlignBytes / key_bytes) - 1ull);
  const uint64_t len = ((data_len + num_chunks - 1) / num_chunks) & mask;
  if (len >= 0xffffffffull)
    return set_error(FI_ERR_INTEGER_OVERFLOW,
                     "Relation is too large and causes an integer overflow. Try "
                     "using more chunks by setting a higher CUDA grid size");
  *chunk_len = len;
  return FI_OK;
}

extern "C" uint32_t fi_padding_len(uint32_t tuple_bytes) {
  return tuple_bytes ? kPaddingBytes / tuple_bytes : 0;
}

static bool valid_tuple_bytes(uint32_t t) { return t == 8 || t == 16; }

extern "C" int fi_partition_offsets_init(fi_partition_offsets *o,
                                         fi_histogram_algorithm histogram_type,
                                         uint32_t max_chunks,
                                         uint32_t radix_bits,
                                         uint32_t tuple_bytes,
                                         uint64_t *offsets,
                                         uint64_t *local_offsets) {
  if (!o || !valid_tuple_bytes(tuple_bytes) || max_chunks == 0 ||
      radix_bits > 31)
    return set_error(FI_ERR_INVALID_ARGUMENT, "invalid PartitionOffsets arguments");
  memset(o, 0, sizeof(*o));
  o->offsets = offsets;
  o->local_offsets =
      histogram_type == FI_HISTOGRAM_CONTIGUOUS ? local_offsets : nullptr;
  o->chunks = histogram_type == FI_HISTOGRAM_CONTIGUOUS ? 1u : max_chunks;
  o->max_chunks = max_chunks;
  o->radix_bits = radix_bits;
  o->histogram_type = (uint32_t)histogram_type;
  o->tuple_bytes = tuple_bytes;
  return FI_OK;
}

extern "C" uint64_t fi_partitioned_relation_alloc_len(
    uint64_t len, fi_histogram_algorithm histogram_type, uint32_t radix_bits,
    uint32_t max_chunks, uint32_t tuple_bytes) {
  const uint64_t chunks =
      histogram_type == FI_HISTOGRAM_CONTIGUOUS ? 1u : max_chunks;
  return len + (chunks << radix_bits) * fi_padding_len(tuple_bytes);
}

extern "C" int fi_partitioned_relation_init(
    fi_partitioned_relation *r, uint64_t len,
    fi_histogram_algorithm histogram_type, uint32_t radix_bits,
    uint32_t max_chunks, uint32_t tuple_bytes, void *relation,
    uint64_t relation_len, uint64_t *offsets) {
  if (!r || !valid_tuple_bytes(tuple_bytes) || max_chunks == 0 || radix_bits > 31)
    return set_error(FI_ERR_INVALID_ARGUMENT,
                     "invalid PartitionedRelation arguments");
  const uint64_t need = fi_partitioned_relation_alloc_len(
      len, histogram_type, radix_bits, max_chunks, tuple_bytes);
  if (relation_len < need)
    return set_error(FI_ERR_INVALID_ARGUMENT,
                     "relation memory holds %llu tuples; %llu are needed",
                     (unsigned long long)relation_len,
                     (unsigned long long)need);
  memset(r, 0, sizeof(*r));
  r->relation = relation;
  r->relation_len = relation_len;
  r->offsets = offsets;
  r->len = len;
  r->chunks = histogram_type == FI_HISTOGRAM_CONTIGUOUS ? 1u : max_chunks;
  r->radix_bits = radix_bits;
  r->tuple_bytes = tuple_bytes;
  return FI_OK;
}

static uint64_t rel_padded_len(const fi_partitioned_relation *r) {
  return r->len + ((uint64_t)r->chunks << r->radix_bits) *
                      fi_padding_len(r->tuple_bytes);
}

extern "C" int fi_partition_len(const fi_partitioned_relation *r,
                                const uint64_t *host_offsets,
                                uint32_t partition_id, uint64_t *len) {
  if (!r || !host_offsets || !len)
    return set_error(FI_ERR_INVALID_ARGUMENT, "null argument");
  const uint32_t F = 1u << r->radix_bits;
  if (partition_id >= F)
    return set_error(FI_ERR_INVALID_ARGUMENT, "Invalid partition ID");
  const uint64_t pad = fi_padding_len(r->tuple_bytes);
  const uint64_t n_off = (uint64_t)r->chunks * F;
  uint64_t total = 0;
  for (uint32_t c = 0; c < r->chunks; ++c) {
    const uint64_t ofi = (uint64_t)c * F + partition_id;
    const uint64_t b = host_offsets[ofi];
    const uint64_t e =
        (ofi + 1 < n_off) ? host_offsets[ofi + 1] - pad : rel_padded_len(r);
    total += e - b;
  }
  *len = total;
  return FI_OK;
}

extern "C" int fi_partitioned_relation_resize(fi_partitioned_relation *r,
                                              uint64_t new_len) {
  if (!r) return set_error(FI_ERR_INVALID_ARGUMENT, "null argument");
  const uint64_t pad_total =
      ((uint64_t)r->chunks << r->radix_bits) * fi_padding_len(r->tuple_bytes);
  const uint64_t capacity = r->relation_len - pad_total;
  if (new_len > capacity)
    return set_error(FI_ERR_INVALID_ARGUMENT,
                     "Insufficient capacity to resize to new length");
  r->len = new_len;
  return FI_OK;
}

// ---------------------------------------------------------------------------
// GpuRadixPartitioner
// ---------------------------------------------------------------------------
struct fi_gpu_radix_partitioner {
  fi_histogram_algorithm hist;
  fi_partition_algorithm algo;
  int32_t bits[3];
  uint32_t grid, block;
  uint64_t dmem_buffer_bytes;
  DevBuf hist_buf, tile_state, counter, status;
  DevBuf tmp_rel, tmp_cursors;  // hierarchical scatter

  int pass_bits(fi_radix_pass pass, uint32_t *b, uint32_t *ignore) const {
    if ((int)pass < 0 || (int)pass > 2 || bits[pass] < 0)
      return set_error(FI_ERR_INVALID_ARGUMENT,
                       "The requested partitioning pass is not specified");
    *b = (uint32_t)bits[pass];
    uint32_t ig = 0;
    for (int i = 0; i < (int)pass; ++i) ig += bits[i] > 0 ? (uint32_t)bits[i] : 0u;
    *ignore = ig;
    return FI_OK;
  }

  int scratch(uint32_t F, uint32_t chunks) {
    int rc = hist_buf.reserve((size_t)chunks * F * sizeof(uint32_t), true);
    if (rc) return rc;
    rc = tile_state.reserve(((size_t)F / kScanTile + 2) * sizeof(uint64_t), true);
    if (rc) return rc;
    rc = counter.reserve(sizeof(uint32_t) * 4, true);
    if (rc) return rc;
    return status.reserve(sizeof(int) * 4, true);
  }

  HistScratch hs() {
    return HistScratch{(uint32_t *)hist_buf.ptr, (uint64_t *)tile_state.ptr,
                       (uint32_t *)counter.ptr, (int *)status.ptr};
  }
};

extern "C" int fi_gpu_radix_partitioner_new(
    fi_histogram_algorithm prefix_sum_algorithm,
    fi_partition_algorithm partition_algorithm, fi_radix_bits radix_bits,
    uint32_t grid_size, uint32_t block_size, uint64_t dmem_buffer_bytes,
    fi_gpu_radix_partitioner **out) {
  if (!out) return set_error(FI_ERR_INVALID_ARGUMENT, "null output handle");
  *out = nullptr;
  if ((int)prefix_sum_algorithm < 0 || (int)prefix_sum_algorithm > 1 ||
      (int)partition_algorithm < 0 || (int)partition_algorithm > 4)
    return set_error(FI_ERR_INVALID_ARGUMENT, "unknown algorithm");
  if (grid_size == 0 || block_size == 0)
    return set_error(FI_ERR_INVALID_ARGUMENT, "grid and block must be non-zero");
  for (int i = 0; i < 3; ++i)
    if (radix_bits.pass_bits[i] > (int)kMaxRadixBits)
      return set_error(FI_ERR_UNSUPPORTED,
                       "at most %u radix bits per pass are supported",
                       kMaxRadixBits);
  auto *p = new fi_gpu_radix_partitioner();
  p->hist = prefix_sum_algorithm;
  p->algo = partition_algorithm;
  for (int i = 0; i < 3; ++i) p->bits[i] = radix_bits.pass_bits[i];
  p->grid = grid_size;
  p->block = block_size;
  p->dmem_buffer_bytes = dmem_buffer_bytes;
  // prefix-scan state, allocated eagerly like the reference
  // (gpu_radix_partition.rs:337-345)
  uint32_t fmax = 1;
  for (int i = 0; i < 3; ++i)
    if (p->bits[i] >= 0) fmax = std::max(fmax, 1u << p->bits[i]);
  int rc = p->scratch(std::min(fmax, 1u << kMaxHistBits), grid_size);
  if (rc) {
    delete p;
    return rc;
  }
  *out = p;
  return FI_OK;
}

extern "C" void fi_gpu_radix_partitioner_free(fi_gpu_radix_partitioner *p) {
  if (!p) return;
  p->hist_buf.release();
  p->tile_state.release();
  p->counter.release();
  p->status.release();
  p->tmp_rel.release();
  p->tmp_cursors.release();
  delete p;
}

extern "C" int fi_gpu_radix_partitioner_status(fi_gpu_radix_partitioner *p) {
  if (!p) return set_error(FI_ERR_INVALID_ARGUMENT, "null handle");
  return read_and_clear_status(p->status);
}

template <typename K>
static int prefix_sum_impl(fi_gpu_radix_partitioner *p, fi_radix_pass pass,
                           const K *keys, uint64_t len,
                           fi_partition_offsets *o, cudaStream_t stream) {
  if (!p || !o) return set_error(FI_ERR_INVALID_ARGUMENT, "null argument");
  uint32_t bits, ignore;
  int rc = p->pass_bits(pass, &bits, &ignore);
  if (rc) return rc;
  if (o->radix_bits != bits)
    return set_error(FI_ERR_INVALID_ARGUMENT,
                     "PartitionedRelation has mismatching radix bits");
  if (o->tuple_bytes != 2 * sizeof(K))
    return set_error(FI_ERR_INVALID_ARGUMENT, "PartitionOffsets has a different tuple type");
  if (p->hist == FI_HISTOGRAM_CHUNKED) {
    if (o->chunks != p->grid)
      return set_error(FI_ERR_INVALID_ARGUMENT,
                       "PartitionedRelation has mismatching number of chunks");
  } else {
    if (o->chunks != 1)
      return set_error(FI_ERR_INVALID_ARGUMENT,
                       "PartitionedRelation has mismatching number of chunks");
    if (!o->local_offsets || o->max_chunks < p->grid)
      return set_error(FI_ERR_INVALID_ARGUMENT,
                       "Contiguous offsets need local offsets for grid-size chunks");
  }
  if ((len + p->grid - 1) / p->grid >= 0xffffffffull)
    return set_error(FI_ERR_INTEGER_OVERFLOW,
                     "Relation is too large and causes an integer overflow. Try "
                     "using more chunks by setting a higher CUDA grid size");
  if (bits > kMaxHistBits)
    return set_error(FI_ERR_UNSUPPORTED,
                     "prefix sums support at most %u radix bits per pass",
                     kMaxHistBits);
  if (len > 0 && !keys)
    return set_error(FI_ERR_INVALID_ARGUMENT, "null key column");
  o->data_len = len;
  o->has_data_len = 1;
  const uint32_t F = 1u << bits;
  rc = p->scratch(F, p->grid);
  if (rc) return rc;
  const uint32_t pad = padding_len(2 * sizeof(K));
  cudaError_t e;
  if (p->hist == FI_HISTOGRAM_CHUNKED)
    e = launch_chunked_prefix_sum<K>(keys, len, p->grid, bits, ignore, pad,
                                     o->offsets, p->hs(), device_sm_count(),
                                     stream);
  else
    e = launch_contiguous_prefix_sum<K>(keys, nullptr, len, p->grid, bits,
                                        ignore, pad, nullptr, nullptr,
                                        o->offsets, o->local_offsets, 0,
                                        p->hs(), device_sm_count(), stream);
  if (e != cudaSuccess) return cuda_error(e, "prefix sum launch");
  return FI_OK;
}

extern "C" int fi_gpu_prefix_sum_int32(fi_gpu_radix_partitioner *p,
                                       fi_radix_pass pass,
                                       const int32_t *partition_attr,
                                       uint64_t len,
                                       fi_partition_offsets *offsets,
                                       fi_stream_t stream) {
  return prefix_sum_impl<int32_t>(p, pass, partition_attr, len, offsets,
                                  (cudaStream_t)stream);
}
extern "C" int fi_gpu_prefix_sum_int64(fi_gpu_radix_partitioner *p,
                                       fi_radix_pass pass,
                                       const int64_t *partition_attr,
                                       uint64_t len,
                                       fi_partition_offsets *offsets,
                                       fi_stream_t stream) {
  return prefix_sum_impl<int64_t>(p, pass, partition_attr, len, offsets,
                                  (cudaStream_t)stream);
}

template <typename K>
static int copy_with_payload_impl(fi_gpu_radix_partitioner *p,
                                  fi_radix_pass pass, const K *src_key,
                                  const K *src_pay, uint64_t len, K *dst_key,
                                  K *dst_pay, uint64_t dst_len,
                                  fi_partition_offsets *o,
                                  cudaStream_t stream) {
  if (!p || !o) return set_error(FI_ERR_INVALID_ARGUMENT, "null argument");
  uint32_t bits, ignore;
  int rc = p->pass_bits(pass, &bits, &ignore);
  if (rc) return rc;
  if (o->radix_bits != bits)
    return set_error(FI_ERR_INVALID_ARGUMENT,
                     "PartitionOffsets has mismatching radix bits");
  if (p->hist == FI_HISTOGRAM_CHUNKED)
    return set_error(FI_ERR_INVALID_ARGUMENT,
                     "Unsupported histogram algorithm, try using Contiguous instead");
  if (o->chunks != 1)
    return set_error(FI_ERR_INVALID_ARGUMENT,
                     "PartitionOffsets has mismatching number of chunks");
  if (!o->local_offsets || o->max_chunks < p->grid)
    return set_error(FI_ERR_INVALID_ARGUMENT,
                     "Contiguous offsets need local offsets for grid-size chunks");
  if (len >= 0xffffffffull)
    return set_error(FI_ERR_INTEGER_OVERFLOW,
                     "Relation is too large and causes an integer overflow.");
  if (dst_len != len)
    return set_error(FI_ERR_INVALID_ARGUMENT,
                     "Destination columns must have the source length");
  if (bits > kMaxHistBits)
    return set_error(FI_ERR_UNSUPPORTED,
                     "prefix sums support at most %u radix bits per pass",
                     kMaxHistBits);
  o->data_len = len;
  o->has_data_len = 1;
  const uint32_t F = 1u << bits;
  rc = p->scratch(F, p->grid);
  if (rc) return rc;
  cudaError_t e = launch_contiguous_prefix_sum<K>(
      src_key, src_pay, len, p->grid, bits, ignore, padding_len(2 * sizeof(K)),
      dst_key, dst_pay, o->offsets, o->local_offsets, 0, p->hs(),
      device_sm_count(), stream);
  if (e != cudaSuccess) return cuda_error(e, "prefix sum launch");
  return FI_OK;
}

extern "C" int fi_gpu_prefix_sum_and_copy_with_payload_int32(
    fi_gpu_radix_partitioner *p, fi_radix_pass pass, const int32_t *src_key,
    const int32_t *src_pay, uint64_t len, int32_t *dst_key, int32_t *dst_pay,
    uint64_t dst_len, fi_partition_offsets *offsets, fi_stream_t stream) {
  return copy_with_payload_impl<int32_t>(p, pass, src_key, src_pay, len,
                                         dst_key, dst_pay, dst_len, offsets,
                                         (cudaStream_t)stream);
}
extern "C" int fi_gpu_prefix_sum_and_copy_with_payload_int64(
    fi_gpu_radix_partitioner *p, fi_radix_pass pass, const int64_t *src_key,
    const int64_t *src_pay, uint64_t len, int64_t *dst_key, int64_t *dst_pay,
    uint64_t dst_len, fi_partition_offsets *offsets, fi_stream_t stream) {
  return copy_with_payload_impl<int64_t>(p, pass, src_key, src_pay, len,
                                         dst_key, dst_pay, dst_len, offsets,
                                         (cudaStream_t)stream);
}

template <typename K>
static int transform_impl(fi_gpu_radix_partitioner *p, fi_radix_pass pass,
                          uint32_t partition_id,
                          const fi_partitioned_relation *src, K *dst_key,
                          K *dst_pay, uint64_t dst_len,
                          fi_partition_offsets *o, cudaStream_t stream) {
  if (!p || !o || !src) return set_error(FI_ERR_INVALID_ARGUMENT, "null argument");
  uint32_t bits, ignore;
  int rc = p->pass_bits(pass, &bits, &ignore);
  if (rc) return rc;
  if (partition_id >= (1u << src->radix_bits))
    return set_error(FI_ERR_INVALID_ARGUMENT, "Invalid partition ID");
  if (o->radix_bits != bits)
    return set_error(FI_ERR_INVALID_ARGUMENT,
                     "PartitionedRelation has mismatching radix bits");
  if (p->hist == FI_HISTOGRAM_CHUNKED)
    return set_error(FI_ERR_INVALID_ARGUMENT,
                     "Unsupported histogram algorithm, try using Contiguous instead");
  if (o->chunks != 1)
    return set_error(FI_ERR_INVALID_ARGUMENT,
                     "PartitionedRelation has mismatching number of chunks");
  if (!o->local_offsets || o->max_chunks < p->grid)
    return set_error(FI_ERR_INVALID_ARGUMENT,
                     "Contiguous offsets need local offsets for grid-size chunks");
  if (src->tuple_bytes != 2 * sizeof(K) || o->tuple_bytes != 2 * sizeof(K))
    return set_error(FI_ERR_INVALID_ARGUMENT, "mismatching tuple types");
  if (rel_padded_len(src) >= 0xffffffffull)
    return set_error(FI_ERR_INTEGER_OVERFLOW,
                     "Relation is too large and causes an integer overflow.");
  if (src->chunks > kMaxTransformChunks)
    return set_error(FI_ERR_UNSUPPORTED,
                     "at most %u source chunks are supported", kMaxTransformChunks);
  if (bits > kMaxHistBits)
    return set_error(FI_ERR_UNSUPPORTED,
                     "prefix sums support at most %u radix bits per pass",
                     kMaxHistBits);
  o->data_len = dst_len;
  o->has_data_len = 1;
  const uint32_t F = 1u << bits;
  rc = p->scratch(F, p->grid);
  if (rc) return rc;
  cudaError_t e = launch_prefix_sum_and_transform<K>(
      partition_id, src->relation, src->offsets, src->chunks, src->radix_bits,
      rel_padded_len(src), padding_len(src->tuple_bytes), dst_len, p->grid,
      bits, ignore, padding_len(2 * sizeof(K)), dst_key, dst_pay, o->offsets,
      o->local_offsets, p->hs(), device_sm_count(), stream);
  if (e != cudaSuccess) return cuda_error(e, "transform launch");
  return FI_OK;
}

extern "C" int fi_gpu_prefix_sum_and_transform_int32(
    fi_gpu_radix_partitioner *p, fi_radix_pass pass, uint32_t partition_id,
    const fi_partitioned_relation *src, int32_t *dst_key, int32_t *dst_pay,
    uint64_t dst_len, fi_partition_offsets *offsets, fi_stream_t stream) {
  return transform_impl<int32_t>(p, pass, partition_id, src, dst_key, dst_pay,
                                 dst_len, offsets, (cudaStream_t)stream);
}
extern "C" int fi_gpu_prefix_sum_and_transform_int64(
    fi_gpu_radix_partitioner *p, fi_radix_pass pass, uint32_t partition_id,
    const fi_partitioned_relation *src, int64_t *dst_key, int64_t *dst_pay,
    uint64_t dst_len, fi_partition_offsets *offsets, fi_stream_t stream) {
  return transform_impl<int64_t>(p, pass, partition_id, src, dst_key, dst_pay,
                                 dst_len, offsets, (cudaStream_t)stream);
}

// Whether a pass of `bits` uses the hierarchical two-level scatter: above
// kSingleLevelBits for the write-combining algorithms, and above the
// single-level limit for all (NC keeps one level while its per-partition
// counters fit shared memory).
static bool two_level(const fi_gpu_radix_partitioner *p, uint32_t bits) {
  return bits > kMaxTileBits ||
         (bits > kSingleLevelBits && p->algo != FI_PARTITION_NC);
}

template <typename K>
static int preallocate_impl(fi_gpu_radix_partitioner *p, fi_radix_pass pass) {
  if (!p) return set_error(FI_ERR_INVALID_ARGUMENT, "null handle");
  uint32_t bits, ignore;
  int rc = p->pass_bits(pass, &bits, &ignore);
  if (rc) return rc;
  if (two_level(p, bits)) {
    const uint32_t hi = hierarchical_hi_bits(bits);
    rc = p->tmp_cursors.reserve(((size_t)p->grid << hi) * sizeof(uint64_t), false);
    if (rc) return rc;
  }
  return p->scratch(1u << std::min(bits, kMaxHistBits), p->grid);
}

extern "C" int fi_gpu_preallocate_partition_state_int32(
    fi_gpu_radix_partitioner *p, fi_radix_pass pass) {
  return preallocate_impl<int32_t>(p, pass);
}
extern "C" int fi_gpu_preallocate_partition_state_int64(
    fi_gpu_radix_partitioner *p, fi_radix_pass pass) {
  return preallocate_impl<int64_t>(p, pass);
}

template <typename K>
static int partition_impl(fi_gpu_radix_partitioner *p, fi_radix_pass pass,
                          const K *keys, const K *pays, uint64_t len,
                          fi_partition_offsets *o, fi_partitioned_relation *r,
                          cudaStream_t stream) {
  if (!p || !o || !r) return set_error(FI_ERR_INVALID_ARGUMENT, "null argument");
  uint32_t bits, ignore;
  int rc = p->pass_bits(pass, &bits, &ignore);
  if (rc) return rc;
  if (!o->has_data_len)
    return set_error(FI_ERR_INVALID_ARGUMENT, "PartitionOffsets has no length");
  if (r->len != o->data_len)
    return set_error(FI_ERR_INVALID_ARGUMENT,
                     "PartitionOffsets and PartitionedRelation have mismatching lengths");
  if (len != o->data_len)
    return set_error(FI_ERR_INVALID_ARGUMENT,
                     "Partition attribute and PartitionOffsets have mismatching lengths");
  if (r->radix_bits != bits)
    return set_error(FI_ERR_INVALID_ARGUMENT,
                     "PartitionedRelation has mismatching radix bits");
  if ((len + p->grid - 1) / p->grid >= 0xffffffffull)
    return set_error(FI_ERR_INTEGER_OVERFLOW,
                     "Relation is too large and causes an integer overflow. Try "
                     "using more chunks by setting a higher CUDA grid size");
  if (o->chunks != r->chunks)
    return set_error(FI_ERR_INVALID_ARGUMENT,
                     "PartitionOffsets and PartitionedRelation have mismatching chunks");
  if (o->radix_bits != bits)
    return set_error(FI_ERR_INVALID_ARGUMENT,
                     "PartitionOffsets has mismatching radix bits");
  if (r->tuple_bytes != 2 * sizeof(K) || o->tuple_bytes != 2 * sizeof(K))
    return set_error(FI_ERR_INVALID_ARGUMENT, "mismatching tuple types");
  if (r->relation_len < rel_padded_len(r))
    return set_error(FI_ERR_INVALID_ARGUMENT,
                     "PartitionedRelation memory is smaller than its padded length");
  const bool contiguous = o->local_offsets != nullptr && o->chunks == 1 &&
                          p->hist == FI_HISTOGRAM_CONTIGUOUS;
  if (!contiguous && o->chunks != p->grid)
    return set_error(FI_ERR_INVALID_ARGUMENT,
                     "PartitionOffsets has mismatching number of chunks");
  if (contiguous && rel_padded_len(r) >= 0xffffffffull)
    return set_error(FI_ERR_INTEGER_OVERFLOW,
                     "Contiguous relations must hold fewer than 2^32 tuples");
  if (len > 0 && (!keys || !pays || !r->relation))
    return set_error(FI_ERR_INVALID_ARGUMENT, "null data pointer");

  // the cursors are read from the PartitionOffsets' memory, which the swap
  // below hands over to the relation (gpu_radix_partition.rs:1113-1121)
  const uint64_t *cursors = contiguous ? o->local_offsets : o->offsets;
  std::swap(r->offsets, o->offsets);
  o->has_data_len = 0;
  if (len == 0) return FI_OK;

  const uint32_t chunks = p->grid;
  const uint32_t F = 1u << bits;
  rc = p->scratch(std::min(F, 1u << kMaxHistBits), chunks);
  if (rc) return rc;
  cudaError_t e;
  if (two_level(p, bits)) {
    const uint32_t hi = hierarchical_hi_bits(bits);
    rc = p->tmp_cursors.reserve(((size_t)chunks << hi) * sizeof(uint64_t), false);
    if (rc) return rc;
    rc = p->tmp_rel.reserve((size_t)len * 2 * sizeof(K), false);
    if (rc) return rc;
    e = launch_partition_hierarchical<K>(
        keys, pays, len, chunks, bits, ignore, cursors, contiguous,
        rel_padded_len(r), r->relation, r->relation_len, p->tmp_rel.ptr,
        (uint64_t *)p->tmp_cursors.ptr, p->hs(), device_sm_count(), stream);
  } else {
    e = launch_partition<K>(keys, pays, len, chunks, bits, ignore, cursors,
                            r->relation, r->relation_len,
                            p->algo == FI_PARTITION_NC ? kScatterNC
                                                       : kScatterAuto,
                            (int *)p->status.ptr, stream);
  }
  if (e != cudaSuccess) return cuda_error(e, "partition launch");
  return FI_OK;
}

extern "C" int fi_gpu_partition_int32(fi_gpu_radix_partitioner *p,
                                      fi_radix_pass pass,
                                      const int32_t *partition_attr,
                                      const int32_t *payload_attr, uint64_t len,
                                      fi_partition_offsets *offsets,
                                      fi_partitioned_relation *rel,
                                      fi_stream_t stream) {
  return partition_impl<int32_t>(p, pass, partition_attr, payload_attr, len,
                                 offsets, rel, (cudaStream_t)stream);
}
extern "C" int fi_gpu_partition_int64(fi_gpu_radix_partitioner *p,
                                      fi_radix_pass pass,
                                      const int64_t *partition_attr,
                                      const int64_t *payload_attr, uint64_t len,
                                      fi_partition_offsets *offsets,
                                      fi_partitioned_relation *rel,
                                      fi_stream_t stream) {
  return partition_impl<int64_t>(p, pass, partition_attr, payload_attr, len,
                                 offsets, rel, (cudaStream_t)stream);
}

// ---------------------------------------------------------------------------
// CudaRadixJoin
// ---------------------------------------------------------------------------
struct fi_cuda_radix_join {
  fi_radix_pass pass;
  int32_t bits[3];
  fi_hashing_scheme scheme;
  uint32_t grid, block;
  DevBuf item_start, item_part, counters, tile_state, status;

  JoinScratch js() {
    return JoinScratch{(uint32_t *)item_start.ptr, (uint32_t *)item_part.ptr,
                       (uint64_t *)tile_state.ptr, (uint32_t *)counters.ptr,
                       (int *)status.ptr};
  }
};

extern "C" int fi_cuda_radix_join_new(fi_radix_pass radix_pass,
                                      fi_radix_bits radix_bits,
                                      fi_hashing_scheme hashing_scheme,
                                      uint32_t grid_size, uint32_t block_size,
                                      fi_cuda_radix_join **out) {
  if (!out) return set_error(FI_ERR_INVALID_ARGUMENT, "null output handle");
  *out = nullptr;
  if ((int)radix_pass < 0 || (int)radix_pass > 2 ||
      radix_bits.pass_bits[radix_pass] < 0)
    return set_error(FI_ERR_INVALID_ARGUMENT,
                     "The requested partitioning pass is not specified");
  if (grid_size == 0 || block_size == 0 || block_size > 1024 ||
      block_size % 32 != 0)
    return set_error(FI_ERR_INVALID_ARGUMENT,
                     "block size must be a multiple of 32 up to 1024");
  if ((int)hashing_scheme < 0 || (int)hashing_scheme > 2)
    return set_error(FI_ERR_INVALID_ARGUMENT, "unknown hashing scheme");
  auto *j = new fi_cuda_radix_join();
  j->pass = radix_pass;
  for (int i = 0; i < 3; ++i) j->bits[i] = radix_bits.pass_bits[i];
  j->scheme = hashing_scheme;
  j->grid = grid_size;
  j->block = block_size;
  *out = j;
  return FI_OK;
}

extern "C" void fi_cuda_radix_join_free(fi_cuda_radix_join *j) {
  if (!j) return;
  j->item_start.release();
  j->item_part.release();
  j->counters.release();
  j->tile_state.release();
  j->status.release();
  delete j;
}

extern "C" int fi_cuda_radix_join_status(fi_cuda_radix_join *j) {
  if (!j) return set_error(FI_ERR_INVALID_ARGUMENT, "null handle");
  return read_and_clear_status(j->status);
}

template <typename K>
static int radix_join_impl(fi_cuda_radix_join *j,
                           const fi_partitioned_relation *b,
                           const fi_partitioned_relation *pr,
                           int64_t *result_set, uint64_t result_len,
                           uint32_t *tasks, uint64_t task_len,
                           uint64_t *match_count, cudaStream_t stream) {
  if (!j || !b || !pr) return set_error(FI_ERR_INVALID_ARGUMENT, "null argument");
  if (b->chunks != 1)
    return set_error(FI_ERR_INVALID_ARGUMENT,
                     "Chunked build relations are not supported, use a "
                     "contiguous relation instead");
  if (pr->chunks != 1)
    return set_error(FI_ERR_INVALID_ARGUMENT,
                     "Chunked probe relations are not supported, use a "
                     "contiguous relation instead");
  if ((uint64_t)j->grid + 1 != task_len)
    return set_error(FI_ERR_INVALID_ARGUMENT,
                     "Task assignement array must have length: grid size + 1");
  if (result_len < (uint64_t)j->grid * j->block)
    return set_error(FI_ERR_INVALID_ARGUMENT,
                     "Result set size is too small, must be at least grid * block size");
  if (j->scheme == FI_HASHING_LINEAR_PROBING)
    return set_error(FI_ERR_UNSUPPORTED,
                     "LinearProbing is not implemented for the radix join");
  if (b->tuple_bytes != 2 * sizeof(K) || pr->tuple_bytes != 2 * sizeof(K))
    return set_error(FI_ERR_INVALID_ARGUMENT, "mismatching tuple types");
  const uint32_t bits = (uint32_t)j->bits[j->pass];
  uint32_t ignore = bits;
  for (int i = 0; i < (int)j->pass; ++i) ignore += j->bits[i] > 0 ? j->bits[i] : 0;
  if (b->radix_bits != bits || pr->radix_bits != bits)
    return set_error(FI_ERR_INVALID_ARGUMENT,
                     "PartitionedRelation has mismatching radix bits");
  const uint32_t F = 1u << bits;
  int rc = j->item_start.reserve((size_t)(F + 1) * sizeof(uint32_t), false);
  if (rc) return rc;
  rc = j->item_part.reserve(
      (size_t)join_items_capacity(F, rel_padded_len(pr)) * sizeof(uint32_t), false);
  if (rc) return rc;
  rc = j->counters.reserve(4 * sizeof(uint32_t), true);
  if (rc) return rc;
  rc = j->tile_state.reserve(((size_t)F / 1024 + 2) * sizeof(uint64_t), true);
  if (rc) return rc;
  rc = j->status.reserve(4 * sizeof(int), true);
  if (rc) return rc;
  const uint64_t b_len = rel_padded_len(b), p_len = rel_padded_len(pr);
  if (p_len >= 0xffffffffull)
    return set_error(FI_ERR_INTEGER_OVERFLOW,
                     "Relation is too large and causes an integer overflow.");
  cudaError_t e = launch_assign_tasks<K>(pr->offsets, (uint32_t)p_len,
                                         padding_len(pr->tuple_bytes), bits,
                                         j->grid, tasks, stream);
  if (e != cudaSuccess) return cuda_error(e, "task assignment launch");
  e = launch_radix_join<K>(b->relation, b->offsets, b_len,
                           padding_len(b->tuple_bytes), pr->relation,
                           pr->offsets, p_len, padding_len(pr->tuple_bytes), F,
                           ignore, j->scheme == FI_HASHING_PERFECT ? 0 : 2,
                           j->grid, j->block, result_set, match_count, j->js(),
                           device_sm_count(), stream);
  if (e != cudaSuccess) return cuda_error(e, "join launch");
  return FI_OK;
}

extern "C" int fi_cuda_radix_join_int32(fi_cuda_radix_join *j,
                                        const fi_partitioned_relation *build_rel,
                                        const fi_partitioned_relation *probe_rel,
                                        int64_t *result_set, uint64_t result_len,
                                        uint32_t *task_assignments,
                                        uint64_t task_len, uint64_t *match_count,
                                        fi_stream_t stream) {
  return radix_join_impl<int32_t>(j, build_rel, probe_rel, result_set,
                                  result_len, task_assignments, task_len,
                                  match_count, (cudaStream_t)stream);
}
extern "C" int fi_cuda_radix_join_int64(fi_cuda_radix_join *j,
                                        const fi_partitioned_relation *build_rel,
                                        const fi_partitioned_relation *probe_rel,
                                        int64_t *result_set, uint64_t result_len,
                                        uint32_t *task_assignments,
                                        uint64_t task_len, uint64_t *match_count,
                                        fi_stream_t stream) {
  return radix_join_impl<int64_t>(j, build_rel, probe_rel, result_set,
                                  result_len, task_assignments, task_len,
                                  match_count, (cudaStream_t)stream);
}

// ---------------------------------------------------------------------------
// CudaHashJoin (no partitioning)
// ---------------------------------------------------------------------------
struct fi_cuda_hash_join {
  fi_hashing_scheme scheme;
  bool selective;
  void *ht;
  uint64_t mem_len, size;
  uint32_t bg, bb, pg, pb;
  // region-ordered probing and building: on by default, slices of
  // probe_slice / build_slice tuples; both share the scratch buffers
  bool grouping = true;
  uint64_t probe_slice = 1ull << 27;
  bool build_grouping = true;
  uint64_t build_slice = 1ull << 27;
  DevBuf group_tuples, group_counts;
};

// Probe (build) sides of at least one tuple per 128-byte table line, on
// tables larger than a region, are grouped by table region before probing
// (inserting).
static bool use_grouping(const fi_cuda_hash_join *h, bool enabled, uint64_t len,
                         uint32_t entry_bytes, uint32_t *region_bits) {
  if (!enabled) return false;
  *region_bits = ht_region_bits(h->size, entry_bytes);
  const uint64_t slots = 1ull << (63 - __builtin_clzll(h->size));
  return *region_bits > 0 && len * 128 >= slots * entry_bytes;
}

extern "C" int fi_cuda_hash_join_set_probe_grouping(fi_cuda_hash_join *hj,
                                                    int enable,
                                                    uint64_t slice_tuples) {
  if (!hj) return set_error(FI_ERR_INVALID_ARGUMENT, "null handle");
  if (enable && slice_tuples == 0)
    return set_error(FI_ERR_INVALID_ARGUMENT, "slice_tuples must be at least 1");
  if (slice_tuples >= 0xffffffffull)
    return set_error(FI_ERR_INVALID_ARGUMENT, "slice_tuples must be below 2^32");
  hj->grouping = enable != 0;
  if (enable) hj->probe_slice = slice_tuples;
  return FI_OK;
}

// The grouping scratch starts with the device status word of its scatter.
extern "C" int fi_cuda_hash_join_status(fi_cuda_hash_join *hj) {
  if (!hj) return set_error(FI_ERR_INVALID_ARGUMENT, "null handle");
  return read_and_clear_status(hj->group_counts);
}

extern "C" int fi_cuda_hash_join_set_build_grouping(fi_cuda_hash_join *hj,
                                                    int enable,
                                                    uint64_t slice_tuples) {
  if (!hj) return set_error(FI_ERR_INVALID_ARGUMENT, "null handle");
  if (enable && slice_tuples == 0)
    return set_error(FI_ERR_INVALID_ARGUMENT, "slice_tuples must be at least 1");
  if (slice_tuples >= 0xffffffffull)
    return set_error(FI_ERR_INVALID_ARGUMENT, "slice_tuples must be below 2^32");
  hj->build_grouping = enable != 0;
  if (enable) hj->build_slice = slice_tuples;
  return FI_OK;
}

extern "C" int fi_hash_table_init_int32(void *ht_mem, uint64_t mem_len,
                                        fi_stream_t stream) {
  cudaError_t e = launch_ht_init<int32_t>(ht_mem, mem_len, (cudaStream_t)stream);
  return e == cudaSuccess ? FI_OK : cuda_error(e, "hash table init");
}
extern "C" int fi_hash_table_init_int64(void *ht_mem, uint64_t mem_len,
                                        fi_stream_t stream) {
  cudaError_t e = launch_ht_init<int64_t>(ht_mem, mem_len, (cudaStream_t)stream);
  return e == cudaSuccess ? FI_OK : cuda_error(e, "hash table init");
}

extern "C" int fi_cuda_hash_join_new(fi_hashing_scheme hashing_scheme,
                                     int is_selective, void *ht_mem,
                                     uint64_t ht_mem_len, uint64_t ht_size,
                                     uint32_t build_grid, uint32_t build_block,
                                     uint32_t probe_grid, uint32_t probe_block,
                                     fi_cuda_hash_join **out) {
  if (!out) return set_error(FI_ERR_INVALID_ARGUMENT, "null output handle");
  *out = nullptr;
  if (!ht_mem) return set_error(FI_ERR_INVALID_ARGUMENT, "Hash table not set");
  if (ht_mem_len < ht_size || ht_size == 0)
    return set_error(FI_ERR_INVALID_ARGUMENT,
                     "Provided memory must be larger than hash table size");
  if (!build_grid || !build_block || !probe_grid || !probe_block)
    return set_error(FI_ERR_INVALID_ARGUMENT, "grid and block must be non-zero");
  auto *h = new fi_cuda_hash_join();
  h->scheme = hashing_scheme;
  h->selective = is_selective != 0;
  h->ht = ht_mem;
  h->mem_len = ht_mem_len;
  h->size = ht_size;
  h->bg = build_grid;
  h->bb = build_block;
  h->pg = probe_grid;
  h->pb = probe_block;
  *out = h;
  return FI_OK;
}

extern "C" void fi_cuda_hash_join_free(fi_cuda_hash_join *hj) {
  if (!hj) return;
  hj->group_tuples.release();
  hj->group_counts.release();
  delete hj;
}

template <typename K>
static int hj_build_impl(fi_cuda_hash_join *h, const K *key, const K *pay,
                         uint64_t len, cudaStream_t stream) {
  if (!h) return set_error(FI_ERR_INVALID_ARGUMENT, "null handle");
  if (len > h->mem_len)
    return set_error(FI_ERR_INVALID_ARGUMENT,
                     "Hash table is too small for the build data");
  if (h->scheme == FI_HASHING_BUCKET_CHAINING ||
      (h->scheme == FI_HASHING_LINEAR_PROBING && h->selective))
    return set_error(FI_ERR_UNSUPPORTED, "hashing scheme not implemented");
  uint32_t region_bits = 0;
  if (len > 0 && use_grouping(h, h->build_grouping, len, 2 * sizeof(K), &region_bits)) {
    const uint64_t slice = std::min(len, h->build_slice);
    int rc = h->group_tuples.reserve(slice * 2 * sizeof(K), false);
    if (!rc) rc = h->group_counts.reserve(ht_region_scratch_bytes(region_bits), true);
    if (rc) return rc;
    cudaError_t e = launch_ht_build_grouped<K>(
        h->scheme == FI_HASHING_LINEAR_PROBING ? 1 : 0, h->selective, h->ht,
        h->size, key, pay, len, h->bg, h->bb, region_bits, h->group_tuples.ptr,
        (uint32_t *)h->group_counts.ptr, slice, (uint32_t)device_sm_count(), stream);
    return e == cudaSuccess ? FI_OK : cuda_error(e, "hash table build");
  }
  cudaError_t e = launch_ht_build<K>(
      h->scheme == FI_HASHING_LINEAR_PROBING ? 1 : 0, h->selective, h->ht,
      h->size, key, pay, len, h->bg, h->bb, stream);
  return e == cudaSuccess ? FI_OK : cuda_error(e, "hash table build");
}

template <typename K>
static int hj_probe_impl(fi_cuda_hash_join *h, const K *key, const K *pay,
                         uint64_t len, uint64_t *result, uint64_t result_len,
                         cudaStream_t stream) {
  if (!h) return set_error(FI_ERR_INVALID_ARGUMENT, "null handle");
  if (result_len < (uint64_t)h->pg * h->pb)
    return set_error(FI_ERR_INVALID_ARGUMENT,
                     "Result set size is too small, must be at least grid * block size");
  if (h->scheme == FI_HASHING_BUCKET_CHAINING)
    return set_error(FI_ERR_UNSUPPORTED, "hashing scheme not implemented");
  uint32_t region_bits = 0;
  if (len > 0 && use_grouping(h, h->grouping, len, 2 * sizeof(K), &region_bits)) {
    const uint64_t slice = std::min(len, h->probe_slice);
    int rc = h->group_tuples.reserve(slice * 2 * sizeof(K), false);
    if (!rc) rc = h->group_counts.reserve(ht_region_scratch_bytes(region_bits), true);
    if (rc) return rc;
    cudaError_t e = launch_ht_probe_grouped<K>(
        h->scheme == FI_HASHING_LINEAR_PROBING ? 1 : 0, h->ht, h->size, key, pay,
        len, result, h->pg, h->pb, region_bits, h->group_tuples.ptr,
        (uint32_t *)h->group_counts.ptr, slice, (uint32_t)device_sm_count(), stream);
    return e == cudaSuccess ? FI_OK : cuda_error(e, "hash table probe");
  }
  cudaError_t e = launch_ht_probe_sum<K>(
      h->scheme == FI_HASHING_LINEAR_PROBING ? 1 : 0, h->ht, h->size, key, pay,
      len, result, h->pg, h->pb, stream);
  return e == cudaSuccess ? FI_OK : cuda_error(e, "hash table probe");
}

extern "C" int fi_cuda_hash_join_build_int32(fi_cuda_hash_join *hj,
                                             const int32_t *key,
                                             const int32_t *pay, uint64_t len,
                                             fi_stream_t stream) {
  return hj_build_impl<int32_t>(hj, key, pay, len, (cudaStream_t)stream);
}
extern "C" int fi_cuda_hash_join_build_int64(fi_cuda_hash_join *hj,
                                             const int64_t *key,
                                             const int64_t *pay, uint64_t len,
                                             fi_stream_t stream) {
  return hj_build_impl<int64_t>(hj, key, pay, len, (cudaStream_t)stream);
}
extern "C" int fi_cuda_hash_join_probe_sum_int32(
    fi_cuda_hash_join *hj, const int32_t *key, const int32_t *pay,
    uint64_t len, uint64_t *result_set, uint64_t result_len,
    fi_stream_t stream) {
  return hj_probe_impl<int32_t>(hj, key, pay, len, result_set, result_len,
                                (cudaStream_t)stream);
}
extern "C" int fi_cuda_hash_join_probe_sum_int64(
    fi_cuda_hash_join *hj, const int64_t *key, const int64_t *pay,
    uint64_t len, uint64_t *result_set, uint64_t result_len,
    fi_stream_t stream) {
  return hj_probe_impl<int64_t>(hj, key, pay, len, result_set, result_len,
                                (cudaStream_t)stream);
}

// ---------------------------------------------------------------------------
// generator
// ---------------------------------------------------------------------------
#define FI_GEN_RC(expr)                                                        \
  do {                                                                         \
    cudaError_t e_ = (expr);                                                   \
    return e_ == cudaSuccess ? FI_OK : cuda_error(e_, "generator launch");     \
  } while (0)

extern "C" int fi_datagen_primary_keys_int32(int32_t *keys, uint64_t n,
                                             uint64_t seed, int32_t base,
                                             fi_stream_t stream) {
  FI_GEN_RC(launch_gen_primary_keys<int32_t>(keys, n, seed, base, (cudaStream_t)stream));
}
extern "C" int fi_datagen_primary_keys_int64(int64_t *keys, uint64_t n,
                                             uint64_t seed, int64_t base,
                                             fi_stream_t stream) {
  FI_GEN_RC(launch_gen_primary_keys<int64_t>(keys, n, seed, base, (cudaStream_t)stream));
}
extern "C" int fi_datagen_uniform_foreign_keys_int32(int32_t *keys, uint64_t n,
                                                     uint64_t pk_n, uint64_t seed,
                                                     int32_t base,
                                                     fi_stream_t stream) {
  FI_GEN_RC(launch_gen_uniform_fk<int32_t>(keys, n, pk_n, seed, base, (cudaStream_t)stream));
}
extern "C" int fi_datagen_uniform_foreign_keys_int64(int64_t *keys, uint64_t n,
                                                     uint64_t pk_n, uint64_t seed,
                                                     int64_t base,
                                                     fi_stream_t stream) {
  FI_GEN_RC(launch_gen_uniform_fk<int64_t>(keys, n, pk_n, seed, base, (cudaStream_t)stream));
}
extern "C" int fi_datagen_zipf_foreign_keys_int32(int32_t *keys, uint64_t n,
                                                  uint64_t pk_n, double s,
                                                  uint64_t seed, uint64_t pk_seed,
                                                  int32_t base,
                                                  fi_stream_t stream) {
  FI_GEN_RC(launch_gen_zipf_fk<int32_t>(keys, n, pk_n, s, seed, pk_seed, base,
                                        (cudaStream_t)stream));
}
extern "C" int fi_datagen_zipf_foreign_keys_int64(int64_t *keys, uint64_t n,
                                                  uint64_t pk_n, double s,
                                                  uint64_t seed, uint64_t pk_seed,
                                                  int64_t base,
                                                  fi_stream_t stream) {
  FI_GEN_RC(launch_gen_zipf_fk<int64_t>(keys, n, pk_n, s, seed, pk_seed, base,
                                        (cudaStream_t)stream));
}
extern "C" int fi_datagen_uniform_u64_keys(int64_t *keys, uint64_t n,
                                           uint64_t seed, fi_stream_t stream) {
  FI_GEN_RC(launch_gen_uniform_u64(keys, n, seed, (cudaStream_t)stream));
}
extern "C" int fi_datagen_null_keys_int32(int32_t *keys, uint64_t n,
                                          uint32_t selectivity, uint64_t seed,
                                          int32_t base, fi_stream_t stream) {
  if (selectivity > 100)
    return set_error(FI_ERR_INVALID_ARGUMENT, "selectivity is a percentage");
  FI_GEN_RC(launch_null_keys<int32_t>(keys, n, selectivity, seed, base,
                                      (cudaStream_t)stream));
}
extern "C" int fi_datagen_null_keys_int64(int64_t *keys, uint64_t n,
                                          uint32_t selectivity, uint64_t seed,
                                          int64_t base, fi_stream_t stream) {
  if (selectivity > 100)
    return set_error(FI_ERR_INVALID_ARGUMENT, "selectivity is a percentage");
  FI_GEN_RC(launch_null_keys<int64_t>(keys, n, selectivity, seed, base,
                                      (cudaStream_t)stream));
}

// Data set shapes (datagen/src/popular.rs:22-105 and the data sets of
// radix-join/src/main.rs:657-760).
extern "C" int fi_dataset_shape(fi_dataset d, uint32_t tuple_bytes,
                                uint64_t *build_len, uint64_t *probe_len) {
  if (!build_len || !probe_len) return set_error(FI_ERR_INVALID_ARGUMENT, "null output");
  if (tuple_bytes != 8 && tuple_bytes != 16)
    return set_error(FI_ERR_INVALID_ARGUMENT, "tuple_bytes must be 8 or 16");
  switch (d) {
    case FI_DATASET_BLANAS:
      *build_len = 16ull << 20;
      *probe_len = 256ull << 20;
      return FI_OK;
    case FI_DATASET_BLANAS4MB:
      *build_len = 512ull << 10;
      *probe_len = 256ull << 20;
      return FI_OK;
    case FI_DATASET_KIM:
      *build_len = 128000000ull;
      *probe_len = 128000000ull;
      return FI_OK;
    case FI_DATASET_TEST:
      *build_len = 1000;
      *probe_len = 1000;
      return FI_OK;
    case FI_DATASET_LUTZ2GV32G:
      *build_len = (2ull << 30) / tuple_bytes;
      *probe_len = (32ull << 30) / tuple_bytes;
      return FI_OK;
    case FI_DATASET_LUTZ32GV32G:
      *build_len = (32ull << 30) / tuple_bytes;
      *probe_len = (32ull << 30) / tuple_bytes;
      return FI_OK;
  }
  return set_error(FI_ERR_INVALID_ARGUMENT, "unknown data set %d", (int)d);
}
