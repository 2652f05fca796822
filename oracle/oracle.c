/*
 * CPU oracle for the radix-partition / radix hash-join path.
 *
 * TEST INFRASTRUCTURE ONLY.  This file restates, in plain sequential C, the
 * algorithms of the reference's sql-ops operators so that tests can check the
 * CUDA kernels bit-exactly.  It is linked only by tests/, by the smoke check
 * and by bench.py's CPU-baseline leg; the product library never calls it.
 *
 * Every function names the reference file:line it follows (paths relative to
 * the reference project root).  The restatement is itself pinned against the
 * reference's own CPU code compiled from its sources (oracle/build_ref.sh ->
 * oracle/_ref/libref_cpu.so) in tests/test_oracle.py.
 *
 * Conventions shared with the reference:
 *   - Tuple<K,V> is {K key; V value;} (sql-ops/src/partition.rs:144-147).
 *   - fanout F = 1 << radix_bits; padding = PADDING_BYTES / sizeof(Tuple) with
 *     PADDING_BYTES = 128 (sql-ops/build.rs:58, partitioned_relation.rs:27-29).
 *   - key_to_partition(key) = (u64(key) & ((F-1) << ignore)) >> ignore,
 *     truncated to u32 (sql-ops/include/gpu_radix_partition.h:122-127).
 *   - The null key is all ones (sql-ops/include/gpu_common.h:113-123).
 */
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#include <math.h>

#define OR_ALIGN_BYTES 128u
#define OR_CHAINING_BUCKETS 2048u /* sql-ops/build.rs:72 */

/* sql-ops/src/partition/partition_input_chunk.rs:24-35 and the GPU
 * re-derivation sql-ops/cudautils/radix_partition.cu:46-57. */
uint64_t or_input_chunk_size(uint64_t data_len, uint32_t num_chunks,
                             uint32_t key_bytes) {
  uint64_t align_mask = ~((uint64_t)(OR_ALIGN_BYTES / key_bytes) - 1ull);
  return ((data_len + num_chunks - 1) / num_chunks) & align_mask;
}

static inline uint32_t key_to_partition(uint64_t key, uint64_t mask,
                                        uint32_t ignore) {
  return (uint32_t)((key & mask) >> ignore);
}

/* Multiply-shift hash, sql-ops/include/gpu_common.h:144-168. */
static inline uint32_t mult_shift_hash32(uint32_t v, uint32_t log2_buckets) {
  return (v * 2654435769u) >> (32u - log2_buckets);
}
static inline uint64_t mult_shift_hash64(uint64_t v, uint32_t log2_buckets) {
  return (v * 11400714819323198485ull) >> (64u - log2_buckets);
}

static uint32_t log2_floor_u64(uint64_t x) {
  uint32_t r = 0;
  while (x >>= 1) r++;
  return r;
}

/* ------------------------------------------------------------------------ */
/* Typed operators, generated for (int32 key, int32 value) and                */
/* (int64 key, int64 value).                                                  */
/* ------------------------------------------------------------------------ */
#define OR_DEFINE(K, SUF, HASHFN)                                              \
  typedef struct {                                                             \
    K key;                                                                     \
    K value;                                                                   \
  } or_tuple_##SUF;                                                            \
                                                                               \
  /* Chunked histogram + offsets, sql-ops/cudautils/radix_partition.cu:40-96   \
   * (GPU, any ignore_bits) == sql-ops/cpputils/radix_partition.cpp:228-267    \
   * (CPU, ignore 0).  offsets[c*F+i] = excl_c[i] +                            \
   * (chunk_len + pad*F)*c + (i+1)*pad. */                                     \
  void or_chunked_prefix_sum_##SUF(const K *keys, uint64_t len,                \
                                   uint32_t num_chunks, uint32_t radix_bits,   \
                                   uint32_t ignore_bits, uint32_t pad,         \
                                   uint64_t *offsets) {                        \
    const uint64_t F = 1ull << radix_bits;                                     \
    const uint64_t mask = (F - 1ull) << ignore_bits;                           \
    const uint64_t clen = or_input_chunk_size(len, num_chunks, sizeof(K));     \
    uint64_t *hist = (uint64_t *)malloc(F * sizeof(uint64_t));                 \
    for (uint32_t c = 0; c < num_chunks; ++c) {                                \
      uint64_t begin = clen * c;                                               \
      uint64_t end = (c + 1 == num_chunks) ? len : begin + clen;               \
      memset(hist, 0, F * sizeof(uint64_t));                                   \
      for (uint64_t i = begin; i < end; ++i)                                   \
        hist[key_to_partition((uint64_t)(int64_t)keys[i], mask,                \
                              ignore_bits)]++;                                 \
      uint64_t off = (clen + (uint64_t)pad * F) * c + pad;                     \
      for (uint64_t p = 0; p < F; ++p) {                                       \
        offsets[c * F + p] = off;                                              \
        off += hist[p] + pad;                                                  \
      }                                                                        \
    }                                                                          \
    free(hist);                                                                \
  }                                                                            \
                                                                               \
  /* Contiguous histogram, sql-ops/cudautils/radix_partition.cu:105-199:       \
   * per-block histograms laid out partition-major, one exclusive scan,        \
   * plus (p+1)*pad.  local_offsets[b*F+p] is block b's cursor for p;          \
   * offsets[p] equals local_offsets[0*F+p]. */                                \
  void or_contiguous_prefix_sum_##SUF(                                         \
      const K *keys, uint64_t len, uint32_t grid, uint32_t radix_bits,         \
      uint32_t ignore_bits, uint32_t pad, uint64_t *offsets,                   \
      uint64_t *local_offsets) {                                               \
    const uint64_t F = 1ull << radix_bits;                                     \
    const uint64_t mask = (F - 1ull) << ignore_bits;                           \
    const uint64_t clen = or_input_chunk_size(len, grid, sizeof(K));           \
    uint64_t *tmp = (uint64_t *)calloc(F * grid, sizeof(uint64_t));            \
    for (uint32_t b = 0; b < grid; ++b) {                                      \
      uint64_t begin = clen * b;                                               \
      uint64_t end = (b + 1 == grid) ? len : begin + clen;                     \
      for (uint64_t i = begin; i < end; ++i)                                   \
        tmp[(uint64_t)grid *                                                   \
                key_to_partition((uint64_t)(int64_t)keys[i], mask,             \
                                 ignore_bits) +                                \
            b]++;                                                              \
    }                                                                          \
    uint64_t run = 0;                                                          \
    for (uint64_t i = 0; i < F * grid; ++i) {                                  \
      uint64_t v = tmp[i];                                                     \
      tmp[i] = run;                                                            \
      run += v;                                                                \
    }                                                                          \
    for (uint32_t b = 0; b < grid; ++b)                                        \
      for (uint64_t p = 0; p < F; ++p)                                         \
        local_offsets[(uint64_t)b * F + p] =                                   \
            tmp[(uint64_t)grid * p + b] + (p + 1) * pad;                       \
    for (uint64_t p = 0; p < F; ++p) offsets[p] = local_offsets[p];            \
    free(tmp);                                                                 \
  }                                                                            \
                                                                               \
  /* Sequential non-caching scatter of every chunk, i.e. the CPU partitioner   \
   * sql-ops/cpputils/radix_partition.cpp:409-446 generalised to ignore_bits   \
   * like the GPU NC kernel sql-ops/cudautils/radix_partition.cu:472-525.      \
   * chunk_offsets[c*F+p] is the first slot of (chunk c, partition p); the     \
   * input chunks follow partition_input_chunk.rs:24-35.  Padding slots are    \
   * not written.  Within a partition the input order is kept. */              \
  void or_chunked_radix_partition_##SUF(                                       \
      const K *keys, const K *pays, uint64_t len,                              \
      const uint64_t *chunk_offsets, uint32_t num_chunks, uint32_t radix_bits, \
      uint32_t ignore_bits, or_tuple_##SUF *out) {                             \
    const uint64_t F = 1ull << radix_bits;                                     \
    const uint64_t mask = (F - 1ull) << ignore_bits;                           \
    const uint64_t clen = or_input_chunk_size(len, num_chunks, sizeof(K));     \
    uint64_t *cur = (uint64_t *)malloc(F * sizeof(uint64_t));                  \
    for (uint32_t c = 0; c < num_chunks; ++c) {                                \
      memcpy(cur, chunk_offsets + (uint64_t)c * F, F * sizeof(uint64_t));      \
      uint64_t begin = clen * c;                                               \
      uint64_t end = (c + 1 == num_chunks) ? len : begin + clen;               \
      for (uint64_t i = begin; i < end; ++i) {                                 \
        uint32_t p = key_to_partition((uint64_t)(int64_t)keys[i], mask,        \
                                      ignore_bits);                            \
        or_tuple_##SUF t;                                                      \
        t.key = keys[i];                                                       \
        t.value = pays[i];                                                     \
        out[cur[p]++] = t;                                                     \
      }                                                                        \
    }                                                                          \
    free(cur);                                                                 \
  }                                                                            \
                                                                               \
  /* Pass-2 prologue, sql-ops/cudautils/radix_partition.cu:323-467: gathers    \
   * partition `pid` of every source chunk (chunk order 0..C-1) into columns,  \
   * then computes the contiguous histogram of the gathered columns.  The      \
   * last source partition ends at src_padded_len (:354-357). */               \
  uint64_t or_prefix_sum_and_transform_##SUF(                                  \
      uint32_t pid, const or_tuple_##SUF *src, const uint64_t *src_offsets,    \
      uint32_t src_chunks, uint32_t src_radix_bits, uint64_t src_padded_len,   \
      uint32_t pad, uint32_t grid, uint32_t radix_bits, uint32_t ignore_bits,  \
      K *dst_key, K *dst_pay, uint64_t *offsets, uint64_t *local_offsets) {    \
    const uint64_t SF = 1ull << src_radix_bits;                                \
    uint64_t n = 0;                                                            \
    for (uint32_t c = 0; c < src_chunks; ++c) {                                \
      uint64_t begin = src_offsets[c * SF + pid];                              \
      uint64_t end = (c + 1 == src_chunks && pid + 1 == SF)                    \
                         ? src_padded_len                                      \
                         : src_offsets[c * SF + pid + 1] - pad;                \
      for (uint64_t i = begin; i < end; ++i) {                                 \
        dst_key[n] = src[i].key;                                               \
        dst_pay[n] = src[i].value;                                             \
        ++n;                                                                   \
      }                                                                        \
    }                                                                          \
    or_contiguous_prefix_sum_##SUF(dst_key, n, grid, radix_bits, ignore_bits,  \
                                   pad, offsets, local_offsets);               \
    return n;                                                                  \
  }                                                                            \
                                                                               \
  /* Greedy task assignment, sql-ops/cudautils/radix_join.cu:58-98. */         \
  void or_assign_tasks_##SUF(const uint64_t *probe_offsets, uint32_t probe_len,\
                             uint32_t probe_pad, uint32_t radix_bits,          \
                             uint32_t grid, uint32_t *tasks) {                 \
    const uint32_t F = 1u << radix_bits;                                       \
    const uint32_t probe_tuples = probe_len - probe_pad * F;                   \
    const uint32_t avg = (probe_tuples + grid - 1u) / grid;                    \
    tasks[0] = 0;                                                              \
    uint32_t task_id = 1, task_size = 0;                                       \
    for (uint32_t p = 0; p < F && task_id < grid; ++p) {                       \
      uint32_t upper = (p + 1 < F) ? (uint32_t)(probe_offsets[p + 1] -         \
                                                probe_pad)                     \
                                   : probe_len;                                \
      task_size += (uint32_t)(upper - probe_offsets[p]);                       \
      if (task_size >= avg) {                                                  \
        tasks[task_id++] = p + 1;                                              \
        task_size = 0;                                                         \
      }                                                                        \
    }                                                                          \
    for (uint32_t t = task_id; t <= grid; ++t) tasks[t] = F;                   \
  }                                                                            \
                                                                               \
  /* Per-partition bucket-chaining join-aggregate,                             \
   * sql-ops/cudautils/radix_join.cu:199-311: heads[2048] (tail = 0xFFFF),     \
   * links, keys, values; bucket = hash(key_to_partition(key, ~(2^ignore-1),   \
   * ignore)); probe walks the chain and adds s.value on key equality.         \
   * Partition p of a contiguous relation spans [off[p], off[p+1]-pad), the    \
   * last one ends at rel_len.  Returns the wrapping i64 sum; *count gets the  \
   * number of matches (the reference reports the sum only). */               \
  int64_t or_radix_join_chaining_##SUF(                                        \
      const or_tuple_##SUF *build, const uint64_t *build_off,                  \
      uint64_t build_len, uint32_t build_pad, const or_tuple_##SUF *probe,     \
      const uint64_t *probe_off, uint64_t probe_len, uint32_t probe_pad,       \
      uint32_t radix_bits, uint32_t ignore_bits, uint64_t *count) {            \
    const uint32_t F = 1u << radix_bits;                                       \
    const uint64_t mask = ~(uint64_t)((1ull << ignore_bits) - 1ull);           \
    const uint32_t log2_buckets = log2_floor_u64(OR_CHAINING_BUCKETS);         \
    uint64_t sum = 0, cnt = 0;                                                 \
    uint64_t cap = 0;                                                          \
    uint32_t *links = NULL;                                                    \
    uint32_t heads[OR_CHAINING_BUCKETS];                                       \
    for (uint32_t p = 0; p < F; ++p) {                                         \
      uint64_t bb = build_off[p];                                              \
      uint64_t be = (p + 1 < F) ? build_off[p + 1] - build_pad : build_len;    \
      uint64_t pb = probe_off[p];                                              \
      uint64_t pe = (p + 1 < F) ? probe_off[p + 1] - probe_pad : probe_len;    \
      uint64_t bn = be - bb;                                                   \
      if (bn > cap) {                                                          \
        cap = bn;                                                              \
        links = (uint32_t *)realloc(links, cap * sizeof(uint32_t));            \
      }                                                                        \
      for (uint32_t b = 0; b < OR_CHAINING_BUCKETS; ++b) heads[b] = UINT32_MAX;\
      for (uint64_t i = 0; i < bn; ++i) {                                      \
        uint64_t idx = key_to_partition((uint64_t)(int64_t)build[bb + i].key,  \
                                        mask, ignore_bits);                    \
        uint32_t bucket = (uint32_t)HASHFN(idx, log2_buckets);                 \
        links[i] = heads[bucket];                                              \
        heads[bucket] = (uint32_t)i;                                           \
      }                                                                        \
      for (uint64_t j = pb; j < pe; ++j) {                                     \
        K key = probe[j].key;                                                  \
        uint64_t idx =                                                         \
            key_to_partition((uint64_t)(int64_t)key, mask, ignore_bits);       \
        uint32_t bucket = (uint32_t)HASHFN(idx, log2_buckets);                 \
        for (uint32_t e = heads[bucket]; e != UINT32_MAX; e = links[e]) {      \
          if (build[bb + e].key == key) {                                      \
            sum += (uint64_t)(int64_t)probe[j].value;                          \
            cnt += 1;                                                          \
          }                                                                    \
        }                                                                      \
      }                                                                        \
    }                                                                          \
    free(links);                                                               \
    if (count) *count = cnt;                                                   \
    return (int64_t)sum;                                                       \
  }                                                                            \
                                                                               \
  /* Per-partition perfect-hash join-aggregate,                                \
   * sql-ops/cudautils/radix_join.cu:103-194: ht[key >> ignore] holds the last \
   * build tuple written to that slot; a probe tuple matches when the slot's   \
   * key equals its key.  ht_entries bounds the index as on the GPU. */        \
  int64_t or_radix_join_perfect_##SUF(                                         \
      const or_tuple_##SUF *build, const uint64_t *build_off,                  \
      uint64_t build_len, uint32_t build_pad, const or_tuple_##SUF *probe,     \
      const uint64_t *probe_off, uint64_t probe_len, uint32_t probe_pad,       \
      uint32_t radix_bits, uint32_t ignore_bits, uint64_t ht_entries,          \
      uint64_t *count) {                                                       \
    const uint32_t F = 1u << radix_bits;                                       \
    const uint64_t mask = ~(uint64_t)((1ull << ignore_bits) - 1ull);           \
    or_tuple_##SUF *ht =                                                       \
        (or_tuple_##SUF *)malloc(ht_entries * sizeof(or_tuple_##SUF));         \
    uint64_t sum = 0, cnt = 0;                                                 \
    for (uint32_t p = 0; p < F; ++p) {                                         \
      uint64_t bb = build_off[p];                                              \
      uint64_t be = (p + 1 < F) ? build_off[p + 1] - build_pad : build_len;    \
      uint64_t pb = probe_off[p];                                              \
      uint64_t pe = (p + 1 < F) ? probe_off[p + 1] - probe_pad : probe_len;    \
      for (uint64_t e = 0; e < ht_entries; ++e) {                              \
        ht[e].key = (K)-1;                                                     \
        ht[e].value = 0;                                                       \
      }                                                                        \
      for (uint64_t i = bb; i < be; ++i) {                                     \
        uint64_t idx = key_to_partition((uint64_t)(int64_t)build[i].key, mask, \
                                        ignore_bits);                          \
        if (idx < ht_entries) ht[idx] = build[i];                              \
      }                                                                        \
      for (uint64_t j = pb; j < pe; ++j) {                                     \
        uint64_t idx = key_to_partition((uint64_t)(int64_t)probe[j].key, mask, \
                                        ignore_bits);                          \
        if (idx < ht_entries && ht[idx].key == probe[j].key) {                 \
          sum += (uint64_t)(int64_t)probe[j].value;                            \
          cnt += 1;                                                            \
        }                                                                      \
      }                                                                        \
    }                                                                          \
    free(ht);                                                                  \
    if (count) *count = cnt;                                                   \
    return (int64_t)sum;                                                       \
  }                                                                            \
                                                                               \
  /* No-partitioning linear-probing build,                                     \
   * sql-ops/cpputils/no_partitioning_join.cpp:27-86: slot = hash(key) mod     \
   * 2^log2(entries), probe forward until a null key.  A one-slot table       \
   * (log2 = 0) hashes to slot 0: the reference shifts by the full word width \
   * there, which is undefined. */                                            \
  void or_ht_build_linearprobing_##SUF(or_tuple_##SUF *ht, uint64_t entries,   \
                                       const K *keys, const K *pays,           \
                                       uint64_t len) {                         \
    uint32_t lg = log2_floor_u64(entries);                                     \
    uint64_t n = 1ull << lg, m = n - 1;                                        \
    for (uint64_t t = 0; t < len; ++t) {                                       \
      uint64_t idx = lg ? (uint64_t)HASHFN((uint64_t)(int64_t)keys[t], lg) : 0;\
      for (uint64_t i = 0; i < n; ++i, idx = (idx + 1) & m) {                  \
        if (ht[idx].key == (K)-1) {                                            \
          ht[idx].key = keys[t];                                               \
          ht[idx].value = pays[t];                                             \
          break;                                                               \
        }                                                                      \
      }                                                                        \
    }                                                                          \
  }                                                                            \
                                                                               \
  /* No-partitioning linear-probing probe-aggregate,                           \
   * sql-ops/cpputils/no_partitioning_join.cpp:88-140 (every matching slot     \
   * adds the probe payload; stops at a null key). */                          \
  uint64_t or_ht_probe_aggregate_linearprobing_##SUF(                          \
      const or_tuple_##SUF *ht, uint64_t entries, const K *keys,               \
      const K *pays, uint64_t len) {                                           \
    uint32_t lg = log2_floor_u64(entries);                                     \
    uint64_t n = 1ull << lg, m = n - 1, sum = 0;                               \
    for (uint64_t t = 0; t < len; ++t) {                                       \
      uint64_t idx = lg ? (uint64_t)HASHFN((uint64_t)(int64_t)keys[t], lg) : 0;\
      for (uint64_t i = 0; i < n; ++i, idx = (idx + 1) & m) {                  \
        if (ht[idx].key == keys[t])                                            \
          sum += (uint64_t)(int64_t)pays[t];                                   \
        else if (ht[idx].key == (K)-1)                                         \
          break;                                                               \
      }                                                                        \
    }                                                                          \
    return sum;                                                                \
  }                                                                            \
                                                                               \
  /* No-partitioning perfect build/probe,                                      \
   * sql-ops/cpputils/no_partitioning_join.cpp:165-273 (the selective build    \
   * skips null keys).  Keys outside [0, entries) are skipped, as the GPU      \
   * library does; the reference indexes the table with them unchecked. */    \
  void or_ht_build_perfect_##SUF(or_tuple_##SUF *ht, uint64_t entries,       \
                                 const K *keys, const K *pays, uint64_t len,   \
                                 int selective) {                              \
    for (uint64_t t = 0; t < len; ++t) {                                       \
      if (selective && keys[t] == (K)-1) continue;                             \
      const uint64_t s = (uint64_t)(int64_t)keys[t];                           \
      if (s >= entries) continue; /* the reference indexes out of bounds */    \
      ht[s].key = keys[t];                                                     \
      ht[s].value = pays[t];                                                   \
    }                                                                          \
  }                                                                            \
  uint64_t or_ht_probe_aggregate_perfect_##SUF(const or_tuple_##SUF *ht,       \
                                               uint64_t entries,               \
                                               const K *keys, const K *pays,   \
                                               uint64_t len) {                 \
    uint64_t sum = 0;                                                          \
    for (uint64_t t = 0; t < len; ++t) {                                       \
      const uint64_t s = (uint64_t)(int64_t)keys[t];                           \
      if (s < entries && ht[s].key == keys[t])                                 \
        sum += (uint64_t)(int64_t)pays[t];                                     \
    }                                                                          \
    return sum;                                                                \
  }

OR_DEFINE(int32_t, i32, mult_shift_hash32)
OR_DEFINE(int64_t, i64, mult_shift_hash64)

/* Block-wide and device-wide exclusive scans over u64,
 * sql-ops/include/prefix_scan.h:55-122 and :213-347 (sequential meaning). */
void or_exclusive_prefix_sum_u64(const uint64_t *in, uint64_t *out,
                                 uint64_t len, uint64_t init) {
  uint64_t run = init;
  for (uint64_t i = 0; i < len; ++i) {
    uint64_t v = in[i];
    out[i] = run;
    run += v;
  }
}
