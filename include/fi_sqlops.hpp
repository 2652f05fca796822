// fi_sqlops.hpp -- C++17 host API over the C ABI of fi_sqlops.h.
//
// Mirrors the reference's Rust host API of the radix-partition / hash-join
// path (sql-ops/src/partition/gpu_radix_partition.rs,
// sql-ops/src/partition/partitioned_relation.rs,
// sql-ops/src/join/cuda_radix_join.rs, sql-ops/src/join/no_partitioning_join.rs):
// the same type names, argument meaning and error kinds, with RAII device
// memory and a CUDA stream in place of rustacuda's `Stream`.  Every call
// forwards to one C entry point; a failed status becomes fi_sqlops::Error
// carrying the reference's ErrorKind (sql-ops/src/error.rs:20-29) and the
// library's message.
//
// Link with fast-interconnects_b200/libfi_sqlops.so and the CUDA runtime.
#ifndef FI_SQLOPS_HPP
#define FI_SQLOPS_HPP

#include <cuda_runtime_api.h>

#include <cstdint>
#include <stdexcept>
#include <string>
#include <type_traits>
#include <utility>
#include <vector>

#include "fi_sqlops.h"

namespace fi_sqlops {

// ErrorKind (sql-ops/src/error.rs:20-29), plus the kinds a bounded device
// wait, a capacity check and a device allocation report.
enum class ErrorKind {
  InvalidArgument,
  IntegerOverflow,
  CudaError,
  RuntimeError,
  Timeout,
  Unsupported,
  Capacity,
  OutOfMemory
};

class Error : public std::runtime_error {
 public:
  Error(ErrorKind kind, int code, const std::string &msg)
      : std::runtime_error(msg), kind_(kind), code_(code) {}
  ErrorKind kind() const { return kind_; }
  int code() const { return code_; }

 private:
  ErrorKind kind_;
  int code_;
};

inline ErrorKind kind_of(int rc) {
  switch (rc) {
    case FI_ERR_INVALID_ARGUMENT: return ErrorKind::InvalidArgument;
    case FI_ERR_INTEGER_OVERFLOW: return ErrorKind::IntegerOverflow;
    case FI_ERR_CUDA: return ErrorKind::CudaError;
    case FI_ERR_TIMEOUT: return ErrorKind::Timeout;
    case FI_ERR_UNSUPPORTED: return ErrorKind::Unsupported;
    case FI_ERR_CAPACITY: return ErrorKind::Capacity;
    case FI_ERR_OUT_OF_MEMORY: return ErrorKind::OutOfMemory;
    default: return ErrorKind::RuntimeError;
  }
}

inline void check(int rc) {
  if (rc != FI_OK) throw Error(kind_of(rc), rc, fi_last_error());
}

inline void check_cuda(cudaError_t e, const char *what) {
  if (e != cudaSuccess)
    throw Error(ErrorKind::CudaError, FI_ERR_CUDA,
                std::string(what) + ": " + cudaGetErrorString(e));
}

// ---- vocabulary (sql-ops/src/partition.rs:35-134) -------------------------
enum class GpuHistogramAlgorithm { Chunked = FI_HISTOGRAM_CHUNKED, Contiguous = FI_HISTOGRAM_CONTIGUOUS };
enum class GpuRadixPartitionAlgorithm {
  NC = FI_PARTITION_NC,
  LASWWC = FI_PARTITION_LASWWC,
  SSWWCv2 = FI_PARTITION_SSWWC_V2,
  SSWWCv2G = FI_PARTITION_SSWWC_V2G,
  HSSWWCv4 = FI_PARTITION_HSSWWC_V4
};
enum class RadixPass { First = FI_PASS_FIRST, Second = FI_PASS_SECOND, Third = FI_PASS_THIRD };
enum class HashingScheme {
  Perfect = FI_HASHING_PERFECT,
  LinearProbing = FI_HASHING_LINEAR_PROBING,
  BucketChaining = FI_HASHING_BUCKET_CHAINING
};

// RadixBits (partition.rs:64-110): bits per pass; a pass given as -1 is
// absent, like `None`.
class RadixBits {
 public:
  explicit RadixBits(int first, int second = -1, int third = -1) {
    raw_.pass_bits[0] = first;
    raw_.pass_bits[1] = second;
    raw_.pass_bits[2] = third;
  }
  // pass_radix_bits: the pass's bits, -1 when the pass is not specified
  int pass_radix_bits(RadixPass pass) const { return raw_.pass_bits[(int)pass]; }
  // pass_ignore_bits: the bits of the earlier passes
  int pass_ignore_bits(RadixPass pass) const {
    int s = 0;
    for (int i = 0; i < (int)pass; ++i) s += raw_.pass_bits[i] > 0 ? raw_.pass_bits[i] : 0;
    return s;
  }
  const fi_radix_bits &raw() const { return raw_; }

 private:
  fi_radix_bits raw_{};
};

// Owned device memory (the reference's `Mem<T>` allocated by `alloc_fn`).
template <typename T>
class DeviceBuffer {
 public:
  DeviceBuffer() = default;
  explicit DeviceBuffer(size_t n) : n_(n) {
    if (n) check_cuda(cudaMalloc(reinterpret_cast<void **>(&p_), n * sizeof(T)), "cudaMalloc");
  }
  DeviceBuffer(const DeviceBuffer &) = delete;
  DeviceBuffer &operator=(const DeviceBuffer &) = delete;
  DeviceBuffer(DeviceBuffer &&o) noexcept : p_(o.p_), n_(o.n_) { o.p_ = nullptr; o.n_ = 0; }
  DeviceBuffer &operator=(DeviceBuffer &&o) noexcept {
    std::swap(p_, o.p_);
    std::swap(n_, o.n_);
    return *this;
  }
  ~DeviceBuffer() {
    if (p_) cudaFree(p_);
  }
  T *data() { return p_; }
  const T *data() const { return p_; }
  size_t len() const { return n_; }
  void swap(DeviceBuffer &o) noexcept {
    std::swap(p_, o.p_);
    std::swap(n_, o.n_);
  }

 private:
  T *p_ = nullptr;
  size_t n_ = 0;
};

template <typename K>
constexpr uint32_t tuple_bytes() {
  static_assert(std::is_same<K, int32_t>::value || std::is_same<K, int64_t>::value,
                "keys are int32_t or int64_t (gpu_radix_partition.rs:1245-1246)");
  return 2 * sizeof(K);
}

// Tuple<K, V> with V = K (sql-ops/src/partition.rs:144-147).
template <typename K>
struct Tuple {
  K key;
  K value;
};

// PartitionOffsets<Tuple<K, K>> (partitioned_relation.rs:62-201): the
// offsets (and, for Contiguous, the per-chunk cursors) in device memory.
template <typename K>
class PartitionOffsets {
 public:
  PartitionOffsets(GpuHistogramAlgorithm histogram_type, uint32_t max_chunks,
                   uint32_t radix_bits) {
    const uint32_t chunks = histogram_type == GpuHistogramAlgorithm::Chunked ? max_chunks : 1;
    offsets_ = DeviceBuffer<uint64_t>((size_t)chunks << radix_bits);
    if (histogram_type == GpuHistogramAlgorithm::Contiguous)
      local_ = DeviceBuffer<uint64_t>((size_t)max_chunks << radix_bits);
    check(fi_partition_offsets_init(&raw_, (fi_histogram_algorithm)histogram_type,
                                    max_chunks, radix_bits, tuple_bytes<K>(),
                                    offsets_.data(), local_.data()));
  }
  uint32_t num_chunks() const { return raw_.chunks; }
  uint32_t radix_bits() const { return raw_.radix_bits; }
  uint32_t padding_len() const { return fi_padding_len(tuple_bytes<K>()); }
  // len(): the data length a prefix sum set, or none (-1 here)
  int64_t len() const { return raw_.has_data_len ? (int64_t)raw_.data_len : -1; }
  fi_partition_offsets *raw() { return &raw_; }
  // the device buffer behind raw().offsets (partition swaps it out)
  DeviceBuffer<uint64_t> &offsets_buffer() { return offsets_; }

 private:
  fi_partition_offsets raw_{};
  DeviceBuffer<uint64_t> offsets_, local_;
};

// PartitionedRelation<Tuple<K, K>> (partitioned_relation.rs:323-497).
template <typename K>
class PartitionedRelation {
 public:
  PartitionedRelation(uint64_t len, GpuHistogramAlgorithm histogram_type,
                      uint32_t radix_bits, uint32_t max_chunks) {
    const auto h = (fi_histogram_algorithm)histogram_type;
    const uint64_t alloc = fi_partitioned_relation_alloc_len(
        len, h, radix_bits, max_chunks, tuple_bytes<K>());
    const uint32_t chunks = histogram_type == GpuHistogramAlgorithm::Chunked ? max_chunks : 1;
    relation_ = DeviceBuffer<Tuple<K>>(alloc);
    offsets_ = DeviceBuffer<uint64_t>((size_t)chunks << radix_bits);
    check(fi_partitioned_relation_init(&raw_, len, h, radix_bits, max_chunks,
                                       tuple_bytes<K>(), relation_.data(), alloc,
                                       offsets_.data()));
  }
  uint64_t len() const { return raw_.len; }
  uint64_t padded_len() const {
    return raw_.len + ((uint64_t)raw_.chunks << raw_.radix_bits) * padding_len();
  }
  uint32_t num_chunks() const { return raw_.chunks; }
  uint32_t radix_bits() const { return raw_.radix_bits; }
  uint32_t padding_len() const { return fi_padding_len(tuple_bytes<K>()); }
  uint32_t fanout() const { return 1u << raw_.radix_bits; }
  // partition_len(partition_id) summed over the chunks (:409-437); reads the
  // offsets back to the host (synchronising the device)
  uint64_t partition_len(uint32_t partition_id) const {
    std::vector<uint64_t> host(((size_t)raw_.chunks << raw_.radix_bits));
    check_cuda(cudaMemcpy(host.data(), raw_.offsets, host.size() * 8, cudaMemcpyDeviceToHost),
               "offset copy");
    uint64_t n = 0;
    check(fi_partition_len(&raw_, host.data(), partition_id, &n));
    return n;
  }
  void resize(uint64_t len) { check(fi_partitioned_relation_resize(&raw_, len)); }
  const Tuple<K> *relation() const { return static_cast<const Tuple<K> *>(raw_.relation); }
  const uint64_t *offsets() const { return raw_.offsets; }
  fi_partitioned_relation *raw() { return &raw_; }
  const fi_partitioned_relation *raw() const { return &raw_; }
  // partition() swaps the offsets pointers of this relation and the
  // PartitionOffsets (gpu_radix_partition.rs:1117-1121), also when it fails
  // after its argument checks; the owning device buffers follow the pointers.
  void adopt_offsets(PartitionOffsets<K> &o) {
    if (raw_.offsets == o.offsets_buffer().data() && raw_.offsets != offsets_.data())
      offsets_.swap(o.offsets_buffer());
  }

 private:
  fi_partitioned_relation raw_{};
  DeviceBuffer<Tuple<K>> relation_;
  DeviceBuffer<uint64_t> offsets_;
};

namespace detail {
template <typename K>
struct Ops;
template <>
struct Ops<int32_t> {
  static constexpr auto prefix_sum = fi_gpu_prefix_sum_int32;
  static constexpr auto copy_with_payload = fi_gpu_prefix_sum_and_copy_with_payload_int32;
  static constexpr auto transform = fi_gpu_prefix_sum_and_transform_int32;
  static constexpr auto preallocate = fi_gpu_preallocate_partition_state_int32;
  static constexpr auto partition = fi_gpu_partition_int32;
  static constexpr auto join = fi_cuda_radix_join_int32;
  static constexpr auto ht_build = fi_cuda_hash_join_build_int32;
  static constexpr auto ht_probe_sum = fi_cuda_hash_join_probe_sum_int32;
};
template <>
struct Ops<int64_t> {
  static constexpr auto prefix_sum = fi_gpu_prefix_sum_int64;
  static constexpr auto copy_with_payload = fi_gpu_prefix_sum_and_copy_with_payload_int64;
  static constexpr auto transform = fi_gpu_prefix_sum_and_transform_int64;
  static constexpr auto preallocate = fi_gpu_preallocate_partition_state_int64;
  static constexpr auto partition = fi_gpu_partition_int64;
  static constexpr auto join = fi_cuda_radix_join_int64;
  static constexpr auto ht_build = fi_cuda_hash_join_build_int64;
  static constexpr auto ht_probe_sum = fi_cuda_hash_join_probe_sum_int64;
};
inline fi_stream_t st(cudaStream_t s) { return reinterpret_cast<fi_stream_t>(s); }
}  // namespace detail

// GpuRadixPartitioner (gpu_radix_partition.rs:314-555).  Not thread-safe
// for concurrent callers, like the reference.
class GpuRadixPartitioner {
 public:
  GpuRadixPartitioner(GpuHistogramAlgorithm prefix_sum_algorithm,
                      GpuRadixPartitionAlgorithm partition_algorithm,
                      const RadixBits &radix_bits, uint32_t grid_size,
                      uint32_t block_size, uint64_t dmem_buffer_bytes = 8 << 10) {
    check(fi_gpu_radix_partitioner_new((fi_histogram_algorithm)prefix_sum_algorithm,
                                       (fi_partition_algorithm)partition_algorithm,
                                       radix_bits.raw(), grid_size, block_size,
                                       dmem_buffer_bytes, &p_));
  }
  GpuRadixPartitioner(const GpuRadixPartitioner &) = delete;
  GpuRadixPartitioner &operator=(const GpuRadixPartitioner &) = delete;
  ~GpuRadixPartitioner() { fi_gpu_radix_partitioner_free(p_); }

  template <typename K>
  void prefix_sum(RadixPass pass, const K *partition_attr, uint64_t len,
                  PartitionOffsets<K> &offsets, cudaStream_t stream) {
    check(detail::Ops<K>::prefix_sum(p_, (fi_radix_pass)pass, partition_attr, len,
                                     offsets.raw(), detail::st(stream)));
  }
  template <typename K>
  void prefix_sum_and_copy_with_payload(RadixPass pass, const K *src_key,
                                        const K *src_pay, uint64_t len, K *dst_key,
                                        K *dst_pay, uint64_t dst_len,
                                        PartitionOffsets<K> &offsets,
                                        cudaStream_t stream) {
    check(detail::Ops<K>::copy_with_payload(p_, (fi_radix_pass)pass, src_key, src_pay,
                                            len, dst_key, dst_pay, dst_len,
                                            offsets.raw(), detail::st(stream)));
  }
  template <typename K>
  void prefix_sum_and_transform(RadixPass pass, uint32_t partition_id,
                                const PartitionedRelation<K> &src, K *dst_key,
                                K *dst_pay, uint64_t dst_len,
                                PartitionOffsets<K> &offsets, cudaStream_t stream) {
    check(detail::Ops<K>::transform(p_, (fi_radix_pass)pass, partition_id, src.raw(),
                                    dst_key, dst_pay, dst_len, offsets.raw(),
                                    detail::st(stream)));
  }
  template <typename K>
  void preallocate_partition_state(RadixPass pass) {
    check(detail::Ops<K>::preallocate(p_, (fi_radix_pass)pass));
  }
  // partition: scatters (key, payload) into `rel` and swaps the offsets into
  // it; `offsets` is left "uninitialized but reusable" (:532-535)
  template <typename K>
  void partition(RadixPass pass, const K *partition_attr, const K *payload_attr,
                 uint64_t len, PartitionOffsets<K> &offsets,
                 PartitionedRelation<K> &rel, cudaStream_t stream) {
    const int rc = detail::Ops<K>::partition(p_, (fi_radix_pass)pass, partition_attr,
                                             payload_attr, len, offsets.raw(), rel.raw(),
                                             detail::st(stream));
    rel.adopt_offsets(offsets);
    check(rc);
  }
  // a device-side error (bounded wait that gave up, capacity) of earlier calls
  void status() { check(fi_gpu_radix_partitioner_status(p_)); }

 private:
  fi_gpu_radix_partitioner *p_ = nullptr;
};

// CudaRadixJoin (cuda_radix_join.rs:127-276).
class CudaRadixJoin {
 public:
  CudaRadixJoin(RadixPass radix_pass, const RadixBits &radix_bits,
                HashingScheme hashing_scheme, uint32_t grid_size, uint32_t block_size) {
    check(fi_cuda_radix_join_new((fi_radix_pass)radix_pass, radix_bits.raw(),
                                 (fi_hashing_scheme)hashing_scheme, grid_size,
                                 block_size, &j_));
  }
  CudaRadixJoin(const CudaRadixJoin &) = delete;
  CudaRadixJoin &operator=(const CudaRadixJoin &) = delete;
  ~CudaRadixJoin() { fi_cuda_radix_join_free(j_); }

  // SELECT SUM(s.value) FROM build JOIN probe ON key; result_set (grid*block
  // i64, zeroed by the caller) is accumulated with +=, task_assignments gets
  // grid+1 entries; match_count (optional, device) adds the matches
  template <typename K>
  void join(const PartitionedRelation<K> &build_rel, const PartitionedRelation<K> &probe_rel,
            int64_t *result_set, uint64_t result_len, uint32_t *task_assignments,
            uint64_t task_len, cudaStream_t stream, uint64_t *match_count = nullptr) {
    check(detail::Ops<K>::join(j_, build_rel.raw(), probe_rel.raw(), result_set,
                               result_len, task_assignments, task_len, match_count,
                               detail::st(stream)));
  }
  void status() { check(fi_cuda_radix_join_status(j_)); }

 private:
  fi_cuda_radix_join *j_ = nullptr;
};

// HashTable (no_partitioning_join.rs:579-625): `size` entries of Tuple<K, K>
// in device memory, every key the null key.
template <typename K>
class HashTable {
 public:
  HashTable(uint64_t size, cudaStream_t stream) : mem_(size), size_(size) {
    const int rc = std::is_same<K, int32_t>::value
                       ? fi_hash_table_init_int32(mem_.data(), size, detail::st(stream))
                       : fi_hash_table_init_int64(mem_.data(), size, detail::st(stream));
    check(rc);
  }
  uint64_t size() const { return size_; }
  Tuple<K> *data() { return mem_.data(); }

 private:
  DeviceBuffer<Tuple<K>> mem_;
  uint64_t size_;
};

// CudaHashJoin (no_partitioning_join.rs:153-279): build, then probe_sum
// (SUM of the probe payloads of all matches, per thread, += into
// result_set[probe_grid * probe_block]).
template <typename K>
class CudaHashJoin {
 public:
  CudaHashJoin(HashingScheme scheme, bool is_selective, HashTable<K> &table,
               uint32_t build_grid, uint32_t build_block, uint32_t probe_grid,
               uint32_t probe_block) {
    check(fi_cuda_hash_join_new((fi_hashing_scheme)scheme, is_selective ? 1 : 0,
                                table.data(), table.size(), table.size(), build_grid,
                                build_block, probe_grid, probe_block, &hj_));
  }
  CudaHashJoin(const CudaHashJoin &) = delete;
  CudaHashJoin &operator=(const CudaHashJoin &) = delete;
  ~CudaHashJoin() { fi_cuda_hash_join_free(hj_); }
  void build(const K *key, const K *pay, uint64_t len, cudaStream_t stream) {
    check(detail::Ops<K>::ht_build(hj_, key, pay, len, detail::st(stream)));
  }
  void probe_sum(const K *key, const K *pay, uint64_t len, uint64_t *result_set,
                 uint64_t result_len, cudaStream_t stream) {
    check(detail::Ops<K>::ht_probe_sum(hj_, key, pay, len, result_set, result_len,
                                       detail::st(stream)));
  }
  // Region-ordered build and probe (no counterpart in the reference; on by
  // default): fi_cuda_hash_join_set_{build,probe}_grouping.
  void set_build_grouping(bool enable, uint64_t slice_tuples = 1ull << 27) {
    check(fi_cuda_hash_join_set_build_grouping(hj_, enable ? 1 : 0, slice_tuples));
  }
  void set_probe_grouping(bool enable, uint64_t slice_tuples = 1ull << 27) {
    check(fi_cuda_hash_join_set_probe_grouping(hj_, enable ? 1 : 0, slice_tuples));
  }
  // Throws on a device-side error of the grouped build or probe.
  void status() { check(fi_cuda_hash_join_status(hj_)); }

 private:
  fi_cuda_hash_join *hj_ = nullptr;
};

}  // namespace fi_sqlops

#endif  // FI_SQLOPS_HPP
