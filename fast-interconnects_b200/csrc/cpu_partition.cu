// Radix partitioning on the CPU: the first pass of the hybrid join, and the
// counterpart of the reference's CpuRadixPartitioner
// (sql-ops/src/partition/cpu_radix_partition.rs:25-560, kernels in
// sql-ops/cpputils/radix_partition.cpp).
//
// Same layout as the GPU Chunked partitioner: the input is cut into the
// canonical chunks (fi_input_chunk_size), chunk c owns the output region
// [c * (chunk_len + F * pad), ...), and partition p of chunk c starts at
//     offsets[c*F + p] = excl_c[p] + (chunk_len + pad*F) * c + (p+1) * pad
// (radix_partition.cu:40-96, cpu_chunked_prefix_sum in radix_partition.cpp),
// so CPU and GPU offsets are identical and a relation partitioned here can
// be finished by the GPU's second pass.  Every chunk is independent: a
// thread computes its chunk's histogram, offsets and scatter without
// waiting for any other (the caller runs one chunk per thread, as the
// reference's rayon scopes do).  Padding slots are never written.
//
// Scatter variants: NC stores each tuple at its partition cursor; SWWC
// (software write-combining, Schuh et al.) collects each partition's
// tuples in a 64-byte line-sized buffer and copies full lines out, so the
// scatter writes whole cache lines instead of touching F lines per few
// tuples.  Tuples keep their input order within a (chunk, partition).
#include <algorithm>
#include <cstdint>
#include <cstring>
#include <emmintrin.h>
#include <new>
#include <vector>

#include "../../include/fi_sqlops.h"
#include "api_internal.h"
#include "common.cuh"

namespace fi {
constexpr uint32_t kLineBytes = 64;  // write-combining line
namespace {

constexpr uint32_t kCpuMaxBits = 16;

template <typename K>
inline uint32_t cpu_partition_of(K key, uint64_t mask, uint32_t ignore) {
  return (uint32_t)(((uint64_t)(int64_t)key & mask) >> ignore);
}

struct ChunkRange {
  uint64_t begin, end, chunk_len;
};

template <typename K>
int chunk_range(uint64_t data_len, uint32_t chunk_id, uint32_t num_chunks,
                ChunkRange *r) {
  if (num_chunks == 0 || chunk_id >= num_chunks)
    return set_error(FI_ERR_INVALID_ARGUMENT, "chunk %u of %u", chunk_id, num_chunks);
  uint64_t clen = 0;
  int rc = fi_input_chunk_size(data_len, num_chunks, (uint32_t)sizeof(K), &clen);
  if (rc) return rc;
  r->chunk_len = clen;
  r->begin = std::min<uint64_t>(data_len, clen * chunk_id);
  r->end = chunk_id + 1 == num_chunks ? data_len
                                      : std::min<uint64_t>(data_len, r->begin + clen);
  return FI_OK;
}

}  // namespace
}  // namespace fi

struct fi_cpu_radix_partitioner {
  fi_cpu_partition_algorithm algorithm;
  uint32_t radix_bits;
  std::vector<uint64_t> cursors;   // F
  std::vector<uint32_t> fill;      // SWWC: tuples buffered per partition
  std::vector<uint32_t> lo;        // SWWC: first slot of a line that is ours
  unsigned char *lines = nullptr;  // SWWC: F line buffers, 64-byte aligned
  ~fi_cpu_radix_partitioner() { ::operator delete[](lines, std::align_val_t(fi::kLineBytes)); }
};

using namespace fi;

extern "C" int fi_cpu_radix_partitioner_new(fi_cpu_histogram_algorithm histogram,
                                            fi_cpu_partition_algorithm algorithm,
                                            uint32_t radix_bits,
                                            fi_cpu_radix_partitioner **out) {
  if (!out) return set_error(FI_ERR_INVALID_ARGUMENT, "null output handle");
  *out = nullptr;
  if (histogram != FI_CPU_HISTOGRAM_CHUNKED && histogram != FI_CPU_HISTOGRAM_CHUNKED_SIMD)
    return set_error(FI_ERR_INVALID_ARGUMENT, "unknown CPU histogram algorithm");
  if (algorithm != FI_CPU_PARTITION_NC && algorithm != FI_CPU_PARTITION_SWWC &&
      algorithm != FI_CPU_PARTITION_SWWC_SIMD)
    return set_error(FI_ERR_INVALID_ARGUMENT, "unknown CPU partition algorithm");
  if (radix_bits > kCpuMaxBits)
    return set_error(FI_ERR_INVALID_ARGUMENT, "at most %u radix bits", kCpuMaxBits);
  auto *p = new (std::nothrow) fi_cpu_radix_partitioner();
  if (!p) return set_error(FI_ERR_OUT_OF_MEMORY, "partitioner");
  p->algorithm = algorithm;
  p->radix_bits = radix_bits;
  const uint32_t F = 1u << radix_bits;
  p->cursors.resize(F);
  p->lo.resize(F);
  if (algorithm != FI_CPU_PARTITION_NC) {
    p->fill.resize(F);
    p->lines = static_cast<unsigned char *>(
        ::operator new[]((size_t)F * kLineBytes, std::align_val_t(kLineBytes), std::nothrow));
    if (!p->lines) {
      delete p;
      return set_error(FI_ERR_OUT_OF_MEMORY, "write-combining buffers");
    }
  }
  *out = p;
  return FI_OK;
}

extern "C" void fi_cpu_radix_partitioner_free(fi_cpu_radix_partitioner *p) { delete p; }

namespace fi {
namespace {

template <typename K>
int cpu_prefix_sum(fi_cpu_radix_partitioner *p, const K *keys, uint64_t data_len,
                   uint32_t chunk_id, uint32_t num_chunks, uint32_t ignore_bits,
                   uint64_t *offsets) {
  if (!p || (!keys && data_len) || !offsets)
    return set_error(FI_ERR_INVALID_ARGUMENT, "null argument");
  ChunkRange r;
  int rc = chunk_range<K>(data_len, chunk_id, num_chunks, &r);
  if (rc) return rc;
  const uint32_t F = 1u << p->radix_bits;
  const uint64_t mask = (uint64_t)(F - 1) << ignore_bits;
  const uint64_t pad = kPaddingBytes / sizeof(Tuple<K>);
  std::vector<uint64_t> hist(F, 0);
  for (uint64_t i = r.begin; i < r.end; ++i)
    ++hist[cpu_partition_of(keys[i], mask, ignore_bits)];
  uint64_t run = (r.chunk_len + pad * F) * chunk_id;
  for (uint32_t q = 0; q < F; ++q) {
    run += pad;
    offsets[q] = run;
    run += hist[q];
  }
  return FI_OK;
}

// SWWC with line-aligned flushes (relation base aligned to the tuple size).
// Each partition's buffer mirrors the 64-byte line of the relation that its
// next tuple lands in: the first line of a partition starts at the slot
// its first tuple takes (the slots before it belong to the previous
// partition or its padding and are not written), every later line is
// whole and aligned and goes out with non-temporal 16-byte stores (no
// read-for-ownership of the destination), the last one with plain stores.
// p->cursors holds the partition offsets on entry.
template <typename K>
int swwc_aligned(fi_cpu_radix_partitioner *p, const K *keys, const K *pays,
                 const ChunkRange &r, uint32_t F, uint64_t mask, uint32_t ignore_bits,
                 Tuple<K> *out, uint64_t out_len) {
  constexpr uint32_t T = sizeof(Tuple<K>), B = kLineBytes / T;
  Tuple<K> *lines = reinterpret_cast<Tuple<K> *>(p->lines);
  uint32_t *fill = p->fill.data(), *lo = p->lo.data();
  uint64_t *lb = p->cursors.data();  // index of the line's slot 0 (mod 2^64)
  const uintptr_t base = reinterpret_cast<uintptr_t>(out);
  for (uint32_t q = 0; q < F; ++q) {
    const uint32_t off = (uint32_t)(((base + lb[q] * T) % kLineBytes) / T);
    fill[q] = lo[q] = off;
    lb[q] -= off;
  }
  for (uint64_t i = r.begin; i < r.end; ++i) {
    const K k = keys[i];
    const uint32_t q = cpu_partition_of(k, mask, ignore_bits);
    Tuple<K> *line = lines + (size_t)q * B;
    line[fill[q]] = Tuple<K>{k, pays[i]};
    if (++fill[q] == B) {
      if (lb[q] + B > out_len)
        return set_error(FI_ERR_CAPACITY, "partition offsets point outside the relation");
      if (lo[q] == 0) {
        const __m128i *src = reinterpret_cast<const __m128i *>(line);
        __m128i *dst = reinterpret_cast<__m128i *>(out + lb[q]);
        _mm_stream_si128(dst + 0, _mm_load_si128(src + 0));
        _mm_stream_si128(dst + 1, _mm_load_si128(src + 1));
        _mm_stream_si128(dst + 2, _mm_load_si128(src + 2));
        _mm_stream_si128(dst + 3, _mm_load_si128(src + 3));
      } else {
        std::memcpy(out + (lb[q] + lo[q]), line + lo[q], (B - lo[q]) * T);
        lo[q] = 0;
      }
      lb[q] += B;
      fill[q] = 0;
    }
  }
  for (uint32_t q = 0; q < F; ++q)
    if (fill[q] > lo[q]) {
      if (lb[q] + fill[q] > out_len)
        return set_error(FI_ERR_CAPACITY, "partition offsets point outside the relation");
      std::memcpy(out + (lb[q] + lo[q]), lines + (size_t)q * B + lo[q],
                  (fill[q] - lo[q]) * T);
    }
  _mm_sfence();  // the streamed lines are visible before the caller reads them
  return FI_OK;
}

template <typename K>
int cpu_partition(fi_cpu_radix_partitioner *p, const K *keys, const K *pays,
                  uint64_t data_len, uint32_t chunk_id, uint32_t num_chunks,
                  uint32_t ignore_bits, const uint64_t *offsets, Tuple<K> *out,
                  uint64_t out_len) {
  if (!p || ((!keys || !pays) && data_len) || !offsets || !out)
    return set_error(FI_ERR_INVALID_ARGUMENT, "null argument");
  ChunkRange r;
  int rc = chunk_range<K>(data_len, chunk_id, num_chunks, &r);
  if (rc) return rc;
  const uint32_t F = 1u << p->radix_bits;
  const uint64_t mask = (uint64_t)(F - 1) << ignore_bits;
  uint64_t *cur = p->cursors.data();
  std::memcpy(cur, offsets, (size_t)F * sizeof(uint64_t));
  auto outside = [&]() {
    return set_error(FI_ERR_CAPACITY, "partition offsets point outside the relation");
  };
  if (p->algorithm == FI_CPU_PARTITION_NC) {
    for (uint64_t i = r.begin; i < r.end; ++i) {
      const K k = keys[i];
      const uint64_t d = cur[cpu_partition_of(k, mask, ignore_bits)]++;
      if (d >= out_len) return outside();
      out[d] = Tuple<K>{k, pays[i]};
    }
    return FI_OK;
  }
  constexpr uint32_t B = kLineBytes / sizeof(Tuple<K>);
  Tuple<K> *lines = reinterpret_cast<Tuple<K> *>(p->lines);
  uint32_t *fill = p->fill.data();
  if (reinterpret_cast<uintptr_t>(out) % sizeof(Tuple<K>) == 0)
    return swwc_aligned<K>(p, keys, pays, r, F, mask, ignore_bits, out, out_len);
  std::memset(fill, 0, (size_t)F * sizeof(uint32_t));
  for (uint64_t i = r.begin; i < r.end; ++i) {
    const K k = keys[i];
    const uint32_t q = cpu_partition_of(k, mask, ignore_bits);
    Tuple<K> *line = lines + (size_t)q * B;
    line[fill[q]] = Tuple<K>{k, pays[i]};
    if (++fill[q] == B) {  // a full line goes out in one piece
      if (cur[q] + B > out_len) return outside();
      std::memcpy(out + cur[q], line, kLineBytes);
      cur[q] += B;
      fill[q] = 0;
    }
  }
  for (uint32_t q = 0; q < F; ++q)
    if (fill[q]) {
      if (cur[q] + fill[q] > out_len) return outside();
      std::memcpy(out + cur[q], lines + (size_t)q * B, fill[q] * sizeof(Tuple<K>));
      cur[q] += fill[q];
    }
  return FI_OK;
}

}  // namespace
}  // namespace fi

extern "C" int fi_cpu_prefix_sum_int32(fi_cpu_radix_partitioner *p, const int32_t *keys,
                                       uint64_t data_len, uint32_t chunk_id,
                                       uint32_t num_chunks, uint32_t ignore_bits,
                                       uint64_t *chunk_offsets) {
  return cpu_prefix_sum<int32_t>(p, keys, data_len, chunk_id, num_chunks, ignore_bits,
                                 chunk_offsets);
}
extern "C" int fi_cpu_prefix_sum_int64(fi_cpu_radix_partitioner *p, const int64_t *keys,
                                       uint64_t data_len, uint32_t chunk_id,
                                       uint32_t num_chunks, uint32_t ignore_bits,
                                       uint64_t *chunk_offsets) {
  return cpu_prefix_sum<int64_t>(p, keys, data_len, chunk_id, num_chunks, ignore_bits,
                                 chunk_offsets);
}
extern "C" int fi_cpu_partition_int32(fi_cpu_radix_partitioner *p, const int32_t *keys,
                                      const int32_t *pays, uint64_t data_len,
                                      uint32_t chunk_id, uint32_t num_chunks,
                                      uint32_t ignore_bits, const uint64_t *chunk_offsets,
                                      void *relation, uint64_t relation_len) {
  return cpu_partition<int32_t>(p, keys, pays, data_len, chunk_id, num_chunks,
                                ignore_bits, chunk_offsets,
                                static_cast<Tuple<int32_t> *>(relation), relation_len);
}
extern "C" int fi_cpu_partition_int64(fi_cpu_radix_partitioner *p, const int64_t *keys,
                                      const int64_t *pays, uint64_t data_len,
                                      uint32_t chunk_id, uint32_t num_chunks,
                                      uint32_t ignore_bits, const uint64_t *chunk_offsets,
                                      void *relation, uint64_t relation_len) {
  return cpu_partition<int64_t>(p, keys, pays, data_len, chunk_id, num_chunks,
                                ignore_bits, chunk_offsets,
                                static_cast<Tuple<int64_t> *>(relation), relation_len);
}
