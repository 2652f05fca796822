/*
 * fi_sqlops.h -- C ABI of the B200 (sm_100a) radix-partition and hash-join
 * operators.
 *
 * This is the drop-in boundary for the reference's `sql-ops` crate: every
 * entry point below replaces the body of one Rust API call of the reference
 * (cited per declaration, paths relative to the reference project root) and
 * keeps that call's argument meaning, memory layout and error behaviour.  A
 * Rust binding is a plain `extern "C"` block over these declarations.
 *
 * Conventions
 *  - Every function returns `int` status: FI_OK (0) or a negative FI_ERR_*
 *    code (the reference's ErrorKind, sql-ops/src/error.rs:20-29).  No entry
 *    point aborts the process; fi_last_error() returns a thread-local message.
 *  - Pointers are device pointers (or any memory the GPU can address, such as
 *    pinned or managed memory) unless a parameter says "host".
 *  - Work is enqueued on the caller's CUDA stream (`cudaStream_t` passed as
 *    fi_stream_t); functions return before the GPU has finished, exactly as
 *    the reference's launches do.  A CUDA context must be current.
 *  - Handles are not thread-safe for concurrent callers (like
 *    GpuRadixPartitioner, gpu_radix_partition.rs:396-399).
 *  - Tuples are `{K key; K value;}` with K = int32_t or int64_t
 *    (Tuple<K,V>, sql-ops/src/partition.rs:144-147); padding in front of
 *    every partition is PADDING_BYTES = 128 bytes (sql-ops/build.rs:58).
 *  - Device-side waits are bounded.  A wait that gives up records
 *    FI_ERR_TIMEOUT in the handle; fi_*_status() reports it.
 */
#ifndef FI_SQLOPS_H
#define FI_SQLOPS_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* cudaStream_t without including the CUDA headers. */
typedef struct CUstream_st *fi_stream_t;

/* ---- status codes: sql-ops/src/error.rs:20-29 ------------------------- */
#define FI_OK 0
#define FI_ERR_INVALID_ARGUMENT (-1) /* ErrorKind::InvalidArgument */
#define FI_ERR_INTEGER_OVERFLOW (-2) /* ErrorKind::IntegerOverflow */
#define FI_ERR_CUDA (-3)             /* ErrorKind::CudaError */
#define FI_ERR_RUNTIME (-4)          /* ErrorKind::RuntimeError */
#define FI_ERR_TIMEOUT (-5)          /* a bounded device wait gave up */
#define FI_ERR_UNSUPPORTED (-6)      /* `unimplemented!()` in the reference */
#define FI_ERR_CAPACITY (-7)         /* hash-table / shared-memory capacity */
#define FI_ERR_OUT_OF_MEMORY (-8)    /* device allocation failed */

/* Message of the last failed call on this thread ("" if none). */
const char *fi_last_error(void);

/* Version string of the library. */
const char *fi_version(void);

/* ---- vocabulary: sql-ops/src/partition.rs:35-134 ----------------------- */
/* HistogramAlgorithmType / GpuHistogramAlgorithm
 * (partition.rs:35-46, gpu_radix_partition.rs:192-222) */
typedef enum {
  FI_HISTOGRAM_CHUNKED = 0,
  FI_HISTOGRAM_CONTIGUOUS = 1
} fi_histogram_algorithm;

/* GpuRadixPartitionAlgorithm (gpu_radix_partition.rs:233-293).  All five
 * produce the same partitions; on B200 they select between the per-tuple
 * scatter (NC) and the shared-memory tile write-combining scatter (the
 * others), which becomes the hierarchical two-level scatter for fanouts
 * above 2^11 (NC: above 2^14). */
typedef enum {
  FI_PARTITION_NC = 0,
  FI_PARTITION_LASWWC = 1,
  FI_PARTITION_SSWWC_V2 = 2,
  FI_PARTITION_SSWWC_V2G = 3,
  FI_PARTITION_HSSWWC_V4 = 4
} fi_partition_algorithm;

/* RadixPass (partition.rs:56-60) */
typedef enum { FI_PASS_FIRST = 0, FI_PASS_SECOND = 1, FI_PASS_THIRD = 2 } fi_radix_pass;

/* HashingScheme (sql-ops/src/join/hashing_scheme.rs:18-43) */
typedef enum {
  FI_HASHING_PERFECT = 0,
  FI_HASHING_LINEAR_PROBING = 1,
  FI_HASHING_BUCKET_CHAINING = 2
} fi_hashing_scheme;

/* RadixBits (partition.rs:64-110): bits per pass; a negative value means the
 * pass is absent (`None`). */
typedef struct {
  int32_t pass_bits[3];
} fi_radix_bits;

/* PartitionOffsets<Tuple<K,K>> (partitioned_relation.rs:62-201).
 * Chunk-major `offsets` (C0.P0 .. C0.PF-1, C1.P0, ...): chunks = max_chunks
 * for Chunked, 1 for Contiguous.  `local_offsets` ([max_chunks * fanout],
 * Contiguous only, NULL otherwise) is the per-chunk cursor array that the
 * Contiguous prefix sum hands to `partition`.  `data_len` is set by the
 * prefix-sum calls.  Memory is owned by the caller. */
typedef struct {
  uint64_t *offsets;
  uint64_t *local_offsets;
  uint32_t chunks;
  uint32_t max_chunks;
  uint32_t radix_bits;
  uint32_t histogram_type; /* fi_histogram_algorithm */
  uint64_t data_len;
  uint32_t has_data_len;
  uint32_t tuple_bytes; /* 8 (int32 tuples) or 16 (int64 tuples) */
} fi_partition_offsets;

/* PartitionedRelation<Tuple<K,K>> (partitioned_relation.rs:323-497).
 * `relation` holds len + chunks*fanout*padding tuples (relation_len is the
 * allocated number of tuples, >= that); partition (c,p) spans
 * [offsets[c*F+p], offsets[c*F+p+1] - padding), the last one ends at
 * len + chunks*fanout*padding (index rule :510-537).  Memory is owned by the
 * caller; `partition` swaps the offsets pointer with the PartitionOffsets'
 * one (gpu_radix_partition.rs:1117-1121). */
typedef struct {
  void *relation;
  uint64_t relation_len;
  uint64_t *offsets;
  uint64_t len;
  uint32_t chunks;
  uint32_t radix_bits;
  uint32_t tuple_bytes;
  uint32_t reserved;
} fi_partitioned_relation;

/* ---- host-side helpers (no GPU needed) --------------------------------- */

/* input_chunk_size (sql-ops/src/partition/partition_input_chunk.rs:24-35):
 * ceil(len/chunks) rounded down to ALIGN_BYTES/key_bytes.  Returns
 * FI_ERR_INTEGER_OVERFLOW when the chunk length is >= 2^32-1. */
int fi_input_chunk_size(uint64_t data_len, uint32_t num_chunks,
                        uint32_t key_bytes, uint64_t *chunk_len);

/* Number of padding tuples per partition: PADDING_BYTES / tuple_bytes
 * (partitioned_relation.rs:27-29). */
uint32_t fi_padding_len(uint32_t tuple_bytes);

/* PartitionOffsets::new (partitioned_relation.rs:74-103) on caller memory:
 * fills the descriptor; `offsets` must hold chunks*fanout entries and, for
 * Contiguous, `local_offsets` max_chunks*fanout entries. */
int fi_partition_offsets_init(fi_partition_offsets *o,
                              fi_histogram_algorithm histogram_type,
                              uint32_t max_chunks, uint32_t radix_bits,
                              uint32_t tuple_bytes, uint64_t *offsets,
                              uint64_t *local_offsets);

/* PartitionedRelation::new (partitioned_relation.rs:335-362) on caller
 * memory; `relation` must hold fi_partitioned_relation_alloc_len() tuples. */
int fi_partitioned_relation_init(fi_partitioned_relation *r, uint64_t len,
                                 fi_histogram_algorithm histogram_type,
                                 uint32_t radix_bits, uint32_t max_chunks,
                                 uint32_t tuple_bytes, void *relation,
                                 uint64_t relation_len, uint64_t *offsets);

/* len + chunks*fanout*padding: tuples to allocate for a PartitionedRelation
 * (partitioned_relation.rs:347-352). */
uint64_t fi_partitioned_relation_alloc_len(uint64_t len,
                                           fi_histogram_algorithm histogram_type,
                                           uint32_t radix_bits,
                                           uint32_t max_chunks,
                                           uint32_t tuple_bytes);

/* PartitionedRelation::partition_len (partitioned_relation.rs:409-437);
 * `host_offsets` are the relation's offsets as host-readable memory. */
int fi_partition_len(const fi_partitioned_relation *r,
                     const uint64_t *host_offsets, uint32_t partition_id,
                     uint64_t *len);

/* PartitionedRelation::resize (partitioned_relation.rs:383-395). */
int fi_partitioned_relation_resize(fi_partitioned_relation *r,
                                   uint64_t new_len);

/* ---- GpuRadixPartitioner (gpu_radix_partition.rs:314-555) -------------- */
typedef struct fi_gpu_radix_partitioner fi_gpu_radix_partitioner;

/* GpuRadixPartitioner::new (gpu_radix_partition.rs:329-383).  grid_size is
 * the number of chunks of the Chunked layout; block_size and
 * dmem_buffer_bytes are tuning hints. */
int fi_gpu_radix_partitioner_new(fi_histogram_algorithm prefix_sum_algorithm,
                                 fi_partition_algorithm partition_algorithm,
                                 fi_radix_bits radix_bits, uint32_t grid_size,
                                 uint32_t block_size,
                                 uint64_t dmem_buffer_bytes,
                                 fi_gpu_radix_partitioner **out);
void fi_gpu_radix_partitioner_free(fi_gpu_radix_partitioner *p);

/* Synchronises the device and reports (and clears) a device-side error the
 * partitioner's kernels recorded (FI_ERR_TIMEOUT, FI_ERR_CAPACITY). */
int fi_gpu_radix_partitioner_status(fi_gpu_radix_partitioner *p);

/* GpuRadixPartitioner::prefix_sum (gpu_radix_partition.rs:400-408, impl
 * :561-696): histogram + exclusive prefix sum + padding -> offsets (Chunked)
 * or offsets + local_offsets (Contiguous). */
int fi_gpu_prefix_sum_int32(fi_gpu_radix_partitioner *p, fi_radix_pass pass,
                            const int32_t *partition_attr, uint64_t len,
                            fi_partition_offsets *offsets, fi_stream_t stream);
int fi_gpu_prefix_sum_int64(fi_gpu_radix_partitioner *p, fi_radix_pass pass,
                            const int64_t *partition_attr, uint64_t len,
                            fi_partition_offsets *offsets, fi_stream_t stream);

/* GpuRadixPartitioner::prefix_sum_and_copy_with_payload
 * (gpu_radix_partition.rs:431-451, impl :698-824): Contiguous prefix sum
 * that also copies both columns to dst (dst_len must equal len). */
int fi_gpu_prefix_sum_and_copy_with_payload_int32(
    fi_gpu_radix_partitioner *p, fi_radix_pass pass, const int32_t *src_key,
    const int32_t *src_pay, uint64_t len, int32_t *dst_key, int32_t *dst_pay,
    uint64_t dst_len, fi_partition_offsets *offsets, fi_stream_t stream);
int fi_gpu_prefix_sum_and_copy_with_payload_int64(
    fi_gpu_radix_partitioner *p, fi_radix_pass pass, const int64_t *src_key,
    const int64_t *src_pay, uint64_t len, int64_t *dst_key, int64_t *dst_pay,
    uint64_t dst_len, fi_partition_offsets *offsets, fi_stream_t stream);

/* GpuRadixPartitioner::prefix_sum_and_transform
 * (gpu_radix_partition.rs:480-500, impl :826-957): gathers partition
 * `partition_id` of every chunk of `src` (whose offsets must be device
 * readable) into the columns dst_key/dst_pay (dst_len = that partition's
 * length) and computes their Contiguous prefix sum. */
int fi_gpu_prefix_sum_and_transform_int32(
    fi_gpu_radix_partitioner *p, fi_radix_pass pass, uint32_t partition_id,
    const fi_partitioned_relation *src, int32_t *dst_key, int32_t *dst_pay,
    uint64_t dst_len, fi_partition_offsets *offsets, fi_stream_t stream);
int fi_gpu_prefix_sum_and_transform_int64(
    fi_gpu_radix_partitioner *p, fi_radix_pass pass, uint32_t partition_id,
    const fi_partitioned_relation *src, int64_t *dst_key, int64_t *dst_pay,
    uint64_t dst_len, fi_partition_offsets *offsets, fi_stream_t stream);

/* GpuRadixPartitioner::preallocate_partition_state
 * (gpu_radix_partition.rs:511-526): allocates the internal device state of
 * `partition` ahead of time. */
int fi_gpu_preallocate_partition_state_int32(fi_gpu_radix_partitioner *p,
                                             fi_radix_pass pass);
int fi_gpu_preallocate_partition_state_int64(fi_gpu_radix_partitioner *p,
                                             fi_radix_pass pass);

/* GpuRadixPartitioner::partition (gpu_radix_partition.rs:536-554, impl
 * :1022-1239): scatters (key, payload) into `rel`; swaps the offsets into
 * the relation (the PartitionOffsets becomes "uninitialised but reusable"). */
int fi_gpu_partition_int32(fi_gpu_radix_partitioner *p, fi_radix_pass pass,
                           const int32_t *partition_attr,
                           const int32_t *payload_attr, uint64_t len,
                           fi_partition_offsets *offsets,
                           fi_partitioned_relation *rel, fi_stream_t stream);
int fi_gpu_partition_int64(fi_gpu_radix_partitioner *p, fi_radix_pass pass,
                           const int64_t *partition_attr,
                           const int64_t *payload_attr, uint64_t len,
                           fi_partition_offsets *offsets,
                           fi_partitioned_relation *rel, fi_stream_t stream);

/* Chunked prefix sum that allocates no device memory.  No counterpart in
 * the reference.  For callers that cannot call cudaMalloc (an engine that
 * owns all device memory through its own pool, a host that forbids
 * allocation on its threads, code that must not stall a stream on an
 * allocation): same offsets as fi_gpu_prefix_sum_int64 on a Chunked
 * partitioner with grid = num_chunks, pass bits = radix_bits and
 * ignore_bits, but the scratch counters live in a fixed 2 MiB array inside
 * the library (held on every GPU that loads it until exit).  Limit:
 * num_chunks * 2^radix_bits <= 524288 counters (more fail with
 * FI_ERR_INVALID_ARGUMENT) and radix_bits <= 18 (more fail with
 * FI_ERR_UNSUPPORTED, as for every prefix sum of the library).  The caller
 * passes the keys and the offsets buffer (num_chunks * 2^radix_bits u64).
 * All calls share the array: calls that overlap on the GPU race; serialise
 * them.  The first call on a device looks the array's address up
 * (cudaGetSymbolAddress), so make it before capturing the stream into a
 * graph; later calls outside a capture look it up again, so a
 * cudaDeviceReset between calls is harmless. */
int fi_gpu_chunked_prefix_sum_noalloc_int64(const int64_t *partition_attr,
                                            uint64_t len, uint32_t num_chunks,
                                            uint32_t radix_bits,
                                            uint32_t ignore_bits,
                                            uint64_t *offsets,
                                            fi_stream_t stream);

/* ---- prefix scans of u64 arrays (the reference's scan test exports,
 *      sql-ops/include/prefix_scan.h:55-122,213-384) -------------------- */

/* GpuPrefixSum::state_len (sql-ops/src/prefix_scan/gpu_prefix_scan.rs:
 * 40-51): entries of 32 bytes of scan state for a grid x block launch. */
uint64_t fi_gpu_prefix_sum_state_len(uint32_t grid_size, uint32_t block_size);
/* host_block_exclusive_prefix_sum_uint64: each of grid_size blocks scans its
 * size/grid_size items in place; thread t of a block owns ceil(items /
 * block_size) consecutive items and adds (t+1) * padding to each. */
int fi_block_exclusive_prefix_sum_uint64(uint64_t *data, uint64_t size,
                                         uint64_t padding, uint32_t grid_size,
                                         uint32_t block_size, fi_stream_t stream);
/* host_device_exclusive_prefix_sum_initialize_uint64 and
 * host_device_exclusive_prefix_sum_uint64: a scan of the whole array over
 * the grid, with state (fi_gpu_prefix_sum_state_len entries of 32 bytes)
 * initialised before every scan; thread g of the grid owns ceil(size /
 * threads) consecutive items and adds (g+1) * padding.  A look-back that
 * waits too long records FI_ERR_TIMEOUT in *status (may be null). */
int fi_device_exclusive_prefix_sum_initialize_uint64(void *state,
                                                     uint32_t grid_size,
                                                     uint32_t block_size,
                                                     fi_stream_t stream);
int fi_device_exclusive_prefix_sum_uint64(uint64_t *data, uint64_t size,
                                          uint64_t padding, void *state,
                                          uint32_t grid_size, uint32_t block_size,
                                          int *status, fi_stream_t stream);

/* ---- CpuRadixPartitioner (sql-ops/src/partition/cpu_radix_partition.rs:
 *      25-560; kernels in sql-ops/cpputils/radix_partition.cpp) --------- */

typedef enum {
  FI_CPU_HISTOGRAM_CHUNKED = 0,
  FI_CPU_HISTOGRAM_CHUNKED_SIMD = 1 /* same result as Chunked */
} fi_cpu_histogram_algorithm;
typedef enum {
  FI_CPU_PARTITION_NC = 0,   /* one store per tuple at its partition cursor */
  FI_CPU_PARTITION_SWWC = 1, /* software write-combining: 64-byte line buffers */
  FI_CPU_PARTITION_SWWC_SIMD = 2 /* same as SWWC */
} fi_cpu_partition_algorithm;

typedef struct fi_cpu_radix_partitioner fi_cpu_radix_partitioner;

/* A partitioner owns the per-thread state of one chunk at a time (its
 * write-combining buffers): use one per thread, as the reference does.
 * radix_bits <= 16.  Host only. */
int fi_cpu_radix_partitioner_new(fi_cpu_histogram_algorithm histogram,
                                 fi_cpu_partition_algorithm algorithm,
                                 uint32_t radix_bits,
                                 fi_cpu_radix_partitioner **out);
void fi_cpu_radix_partitioner_free(fi_cpu_radix_partitioner *p);
/* CpuRadixPartitioner::prefix_sum for chunk chunk_id of num_chunks (the
 * canonical chunking of fi_input_chunk_size over data_len keys):
 * chunk_offsets[0..F) receive the chunk's Chunked offsets, identical to
 * fi_gpu_prefix_sum with Chunked at the same chunk count, i.e.
 * offsets[c*F + p] of the whole relation. */
int fi_cpu_prefix_sum_int32(fi_cpu_radix_partitioner *p, const int32_t *keys,
                            uint64_t data_len, uint32_t chunk_id,
                            uint32_t num_chunks, uint32_t ignore_bits,
                            uint64_t *chunk_offsets);
int fi_cpu_prefix_sum_int64(fi_cpu_radix_partitioner *p, const int64_t *keys,
                            uint64_t data_len, uint32_t chunk_id,
                            uint32_t num_chunks, uint32_t ignore_bits,
                            uint64_t *chunk_offsets);
/* CpuRadixPartitioner::partition for the same chunk: writes its tuples
 * (AoS) into the relation (relation_len tuples, padded Chunked layout)
 * from chunk_offsets, in input order within each partition; padding is not
 * written.  Offsets that lead outside the relation are FI_ERR_CAPACITY. */
int fi_cpu_partition_int32(fi_cpu_radix_partitioner *p, const int32_t *keys,
                           const int32_t *pays, uint64_t data_len,
                           uint32_t chunk_id, uint32_t num_chunks,
                           uint32_t ignore_bits, const uint64_t *chunk_offsets,
                           void *relation, uint64_t relation_len);
int fi_cpu_partition_int64(fi_cpu_radix_partitioner *p, const int64_t *keys,
                           const int64_t *pays, uint64_t data_len,
                           uint32_t chunk_id, uint32_t num_chunks,
                           uint32_t ignore_bits, const uint64_t *chunk_offsets,
                           void *relation, uint64_t relation_len);

/* ---- CudaRadixJoin (sql-ops/src/join/cuda_radix_join.rs:116-164) ------ */
typedef struct fi_cuda_radix_join fi_cuda_radix_join;

/* CudaRadixJoin::new (cuda_radix_join.rs:127-142). */
int fi_cuda_radix_join_new(fi_radix_pass radix_pass, fi_radix_bits radix_bits,
                           fi_hashing_scheme hashing_scheme, uint32_t grid_size,
                           uint32_t block_size, fi_cuda_radix_join **out);
void fi_cuda_radix_join_free(fi_cuda_radix_join *j);
int fi_cuda_radix_join_status(fi_cuda_radix_join *j);

/* CudaRadixJoin::join (cuda_radix_join.rs:144-163, impl :172-276):
 * SELECT SUM(s.value) FROM build r JOIN probe s ON r.key = s.key, per
 * partition of two Contiguous relations.  result_set[grid*block] receives
 * per-thread i64 sums with `+=` (the caller zeroes it); task_assignments
 * ([grid+1]) receives the reference's greedy partition ranges
 * (radix_join.cu:58-98).  match_count (optional, may be NULL) is a device
 * u64 that receives `+=` the number of matches. */
int fi_cuda_radix_join_int32(fi_cuda_radix_join *j,
                             const fi_partitioned_relation *build_rel,
                             const fi_partitioned_relation *probe_rel,
                             int64_t *result_set, uint64_t result_len,
                             uint32_t *task_assignments, uint64_t task_len,
                             uint64_t *match_count, fi_stream_t stream);
int fi_cuda_radix_join_int64(fi_cuda_radix_join *j,
                             const fi_partitioned_relation *build_rel,
                             const fi_partitioned_relation *probe_rel,
                             int64_t *result_set, uint64_t result_len,
                             uint32_t *task_assignments, uint64_t task_len,
                             uint64_t *match_count, fi_stream_t stream);

/* ---- CudaHashJoin: no-partitioning join
 *      (sql-ops/src/join/no_partitioning_join.rs:153-304) -------------- */
typedef struct fi_cuda_hash_join fi_cuda_hash_join;

/* HashTable::new_on_gpu (no_partitioning_join.rs:579-625): sets every key of
 * `mem_len` entries to the null key. */
int fi_hash_table_init_int32(void *ht_mem, uint64_t mem_len, fi_stream_t stream);
int fi_hash_table_init_int64(void *ht_mem, uint64_t mem_len, fi_stream_t stream);

/* CudaHashJoinBuilder::build (no_partitioning_join.rs:688-735).  ht_mem holds
 * ht_mem_len entries; ht_size is the table size used for hashing. */
int fi_cuda_hash_join_new(fi_hashing_scheme hashing_scheme, int is_selective,
                          void *ht_mem, uint64_t ht_mem_len, uint64_t ht_size,
                          uint32_t build_grid, uint32_t build_block,
                          uint32_t probe_grid, uint32_t probe_block,
                          fi_cuda_hash_join **out);
void fi_cuda_hash_join_free(fi_cuda_hash_join *hj);

/* CudaHashJoin::build (no_partitioning_join.rs:250-258, impl :333-386). */
int fi_cuda_hash_join_build_int32(fi_cuda_hash_join *hj, const int32_t *key,
                                  const int32_t *pay, uint64_t len,
                                  fi_stream_t stream);
int fi_cuda_hash_join_build_int64(fi_cuda_hash_join *hj, const int64_t *key,
                                  const int64_t *pay, uint64_t len,
                                  fi_stream_t stream);

/* CudaHashJoin::probe_sum (no_partitioning_join.rs:266-279, impl :388-433):
 * result_set[probe_grid*probe_block] receives per-thread u64 sums (`+=`). */
int fi_cuda_hash_join_probe_sum_int32(fi_cuda_hash_join *hj,
                                      const int32_t *key, const int32_t *pay,
                                      uint64_t len, uint64_t *result_set,
                                      uint64_t result_len, fi_stream_t stream);
int fi_cuda_hash_join_probe_sum_int64(fi_cuda_hash_join *hj,
                                      const int64_t *key, const int64_t *pay,
                                      uint64_t len, uint64_t *result_set,
                                      uint64_t result_len, fi_stream_t stream);

/* Probe-side grouping of CudaHashJoin::probe_sum; no counterpart in the
 * reference.  A probe side of at least one probe per 128-byte table line on
 * a table larger than 8 MB is grouped, slice by slice, by the table region of each
 * probe's first slot before it is probed, so the active region stays in L2
 * (the sum is the same).  A slice whose largest region would hold more than
 * a quarter of its probes (heavy skew, whose probes already share a few
 * table lines) is probed in input order; the device decides per slice, with
 * no host round trip.  On by default with slices of 2^27 tuples; each slice
 * takes slice * tuple_bytes bytes of scratch that the handle keeps, so
 * builds and probes of one handle whose work overlaps on the GPU (different
 * streams) race on it: order them, as the table itself requires.  The
 * grouped probe runs with the library's own launch shape (every SM full of
 * warps) and adds each of its threads' sums into result_set[thread modulo
 * probe_grid * probe_block], so the entries' total is the join's sum, as
 * with the caller's grid.  enable = 0 probes in input order with no scratch,
 * on the probe grid. */
int fi_cuda_hash_join_set_probe_grouping(fi_cuda_hash_join *hj, int enable,
                                         uint64_t slice_tuples);

/* Build-side grouping of CudaHashJoin::build; no counterpart in the
 * reference.  The same grouping for the build: a build side of at least one
 * tuple per 128-byte table line on a table larger than 8 MB is grouped, slice
 * by slice, by the table region of each tuple's first slot before it is
 * inserted, so the lines being written stay in L2.  The probe sums are the
 * same; with linear probing the slots that equal keys occupy may differ from
 * an ungrouped build, as they may between any two concurrent builds.  The
 * grouped inserts run with the library's own launch shape (blocks take
 * tiles of the grouped slice in order), not the handle's build grid.  On by
 * default with slices of 2^27 tuples, sharing the probe's scratch (the larger
 * of the two slices is kept).  enable = 0 inserts in input order with no
 * scratch, on the build grid. */
int fi_cuda_hash_join_set_build_grouping(fi_cuda_hash_join *hj, int enable,
                                         uint64_t slice_tuples);

/* Device-side errors of the grouped build and probe; no counterpart in the
 * reference, whose kernels have no bounded waits.  Synchronises the device,
 * then returns FI_ERR_TIMEOUT if a bounded wait of a grouping scatter gave
 * up since the last call (and clears it), else FI_OK. */
int fi_cuda_hash_join_status(fi_cuda_hash_join *hj);

/* ---- CpuHashJoin: no-partitioning join on the host
 *      (sql-ops/src/join/no_partitioning_join.rs:281-304, impl :440-560;
 *      kernels sql-ops/cpputils/no_partitioning_join.cpp:27-273) -------- */
typedef struct fi_cpu_hash_join fi_cpu_hash_join;

/* HashTable::new_on_cpu (no_partitioning_join.rs:568-581): sets every key of
 * `entries` host entries of {key, value} to the null key. */
int fi_cpu_hash_table_init_int32(void *table, uint64_t entries);
int fi_cpu_hash_table_init_int64(void *table, uint64_t entries);

/* CpuHashJoinBuilder::build (no_partitioning_join.rs:765-772).  The table
 * holds mem_len host entries; size (1..mem_len) is the size used for
 * hashing.  The handle does not own the table.  Schemes: PERFECT,
 * LINEAR_PROBING. */
int fi_cpu_hash_join_new(fi_hashing_scheme hashing_scheme, int is_selective,
                         void *hash_table, uint64_t mem_len, uint64_t size,
                         fi_cpu_hash_join **out);
void fi_cpu_hash_join_free(fi_cpu_hash_join *hj);

/* CpuHashJoin::build (no_partitioning_join.rs:286-288, impl :446-505).
 * Several threads may build disjoint slices into one table at once.
 * InvalidArgument when len exceeds mem_len; Unsupported for a selective
 * linear-probing build (unimplemented in the reference). */
int fi_cpu_hash_join_build_int32(fi_cpu_hash_join *hj, const int32_t *key,
                                 const int32_t *pay, uint64_t len);
int fi_cpu_hash_join_build_int64(fi_cpu_hash_join *hj, const int64_t *key,
                                 const int64_t *pay, uint64_t len);

/* CpuHashJoin::probe_sum (no_partitioning_join.rs:296-303, impl :507-553):
 * adds (wrapping) the payloads of all matches to *join_result; threads may
 * probe disjoint slices into one result. */
int fi_cpu_hash_join_probe_sum_int32(fi_cpu_hash_join *hj, const int32_t *key,
                                     const int32_t *pay, uint64_t len,
                                     uint64_t *join_result);
int fi_cpu_hash_join_probe_sum_int64(fi_cpu_hash_join *hj, const int64_t *key,
                                     const int64_t *pay, uint64_t len,
                                     uint64_t *join_result);

/* ---- Radix exchange between GPUs (no reference counterpart: the exchange
 *      step of a distributed radix join; exchange.cu) --------------------- */
#define FI_EXCHANGE_MAX_RANKS 64
#define FI_IPC_HANDLE_BYTES 64

/* One destination rank's receive columns as seen from the sending rank: a
 * local device pointer for its own share, a peer pointer (opened with
 * fi_ipc_open_handle) for the others.  The sender writes its tuples for
 * this rank into slots [base, base + count) of both columns; cap is the
 * columns' length, checked by every store. */
typedef struct {
  void *key;
  void *pay;
  uint64_t base;
  uint64_t cap;
} fi_exchange_dest;

/* counts[d] (device u64[2^exchange_bits]) = number of keys whose bits
 * [shift, shift + exchange_bits) equal d (key_to_partition of
 * sql-ops/include/gpu_radix_partition.h:122-127 with ignore_bits = shift).
 * exchange_bits <= 6; shift + exchange_bits <= the key's bit width. */
int fi_exchange_histogram_int32(const int32_t *keys, uint64_t len, uint32_t shift,
                                uint32_t exchange_bits, uint64_t *counts,
                                fi_stream_t stream);
int fi_exchange_histogram_int64(const int64_t *keys, uint64_t len, uint32_t shift,
                                uint32_t exchange_bits, uint64_t *counts,
                                fi_stream_t stream);

/* Partition + send in one kernel: every tuple goes to destination d =
 * its key bits [shift, shift + exchange_bits) and is stored into
 * dests[d] (host array of 2^exchange_bits entries) at a slot in
 * [base, base + counts[d]); the order within the region is unspecified.
 * cursors: device u64[2^exchange_bits] workspace.  A store beyond cap is
 * skipped and FI_ERR_CAPACITY recorded in the device word *status (may be
 * null).  No kernel waits on another rank; the caller orders the ranks'
 * steps (synchronize, then a process-group barrier, before the receivers
 * read). */
int fi_exchange_scatter_int32(const int32_t *keys, const int32_t *pays, uint64_t len,
                              uint32_t shift, uint32_t exchange_bits,
                              const fi_exchange_dest *dests, uint64_t *cursors,
                              int *status, fi_stream_t stream);
int fi_exchange_scatter_int64(const int64_t *keys, const int64_t *pays, uint64_t len,
                              uint32_t shift, uint32_t exchange_bits,
                              const fi_exchange_dest *dests, uint64_t *cursors,
                              int *status, fi_stream_t stream);

/* CUDA IPC for the receive columns.  fi_ipc_get_handle: the handle
 * (FI_IPC_HANDLE_BYTES) of the whole allocation holding dev_ptr (e.g. a
 * block of a caching allocator) and dev_ptr's offset in it.
 * fi_ipc_open_handle (another process, another GPU): the allocation's base
 * as a peer pointer (peer access enabled lazily); add the offset.  An
 * allocation is opened once per process: callers share one mapping among
 * equal handles.  fi_ipc_close_handle takes the opened base. */
int fi_ipc_get_handle(const void *dev_ptr, void *handle, uint64_t *offset);
int fi_ipc_open_handle(const void *handle, void **base);
int fi_ipc_close_handle(void *base);

/* ---- gpu_radix_join execution method
 *      (radix-join/src/execution_methods/gpu_radix_join.rs:90-565) ------ */

/* Result of a whole join: wrapping i64 sum of the matched probe payloads
 * (what gpu_radix_join returns) and the number of matches. */
typedef struct {
  int64_t sum;
  uint64_t count;
} fi_join_result;

typedef struct fi_radix_join_engine fi_radix_join_engine;

/* Allocates device workspace for joins of up to max_build x max_probe
 * tuples of `tuple_bytes`-byte tuples with `radix_bits` (one or two passes)
 * and `hashing_scheme` (PERFECT or BUCKET_CHAINING). */
int fi_radix_join_engine_new(uint64_t max_build_len, uint64_t max_probe_len,
                             uint32_t tuple_bytes, fi_radix_bits radix_bits,
                             fi_hashing_scheme hashing_scheme,
                             fi_radix_join_engine **out);
void fi_radix_join_engine_free(fi_radix_join_engine *e);

/* Device bytes the engine holds. */
uint64_t fi_radix_join_engine_workspace_bytes(const fi_radix_join_engine *e);

/* Execution plan of the following runs (no reference counterpart; the
 * reference fixes bits, scheme and launch shape per call site).  The
 * engine's buffers were sized for the radix bits given at creation; a plan
 * may use fewer bits per pass, one pass instead of two, and tuples no
 * larger than the creation's tuple_bytes.  join_block: threads per join CTA
 * (256: four CTAs per SM, 512: two, 1024: one), or 0: for BucketChaining the
 * most CTAs per SM whose shared-memory table holds an average partition with
 * 1/8 headroom, for Perfect 512 (a table of ~14.5K int64 keys).  scatter: 0 = tile scatter fed by TMA bulk
 * copies where the columns allow it, 1 = fed by register loads.  Setting a
 * plan drops a resident build side. */
typedef struct {
  fi_radix_bits radix_bits;
  fi_hashing_scheme hashing_scheme;
  uint32_t join_block;
  uint32_t scatter;
} fi_join_plan;
int fi_radix_join_engine_set_plan(fi_radix_join_engine *e,
                                  const fi_join_plan *plan);

/* Build once, probe many (no reference counterpart; the reference
 * re-partitions both relations on every gpu_radix_join call).  build
 * partitions the build relation and keeps it resident in the engine until
 * the next build or plan; every probe partitions a probe relation, or one
 * slice of a larger one, and joins it against the resident build side,
 * writing {sum, count} of that probe to the device `result`.  The sums and
 * counts of the slices of one probe relation add up (wrapping) to the
 * result of one run over the whole relation.  Device pointers; asynchronous
 * on `stream`; build and probe must be ordered on the GPU by the caller. */
int fi_radix_join_engine_build_int32(fi_radix_join_engine *e,
                                     const int32_t *build_key,
                                     const int32_t *build_pay,
                                     uint64_t build_len, fi_stream_t stream);
int fi_radix_join_engine_build_int64(fi_radix_join_engine *e,
                                     const int64_t *build_key,
                                     const int64_t *build_pay,
                                     uint64_t build_len, fi_stream_t stream);
int fi_radix_join_engine_probe_int32(fi_radix_join_engine *e,
                                     const int32_t *probe_key,
                                     const int32_t *probe_pay,
                                     uint64_t probe_len,
                                     fi_join_result *result,
                                     fi_stream_t stream);
int fi_radix_join_engine_probe_int64(fi_radix_join_engine *e,
                                     const int64_t *probe_key,
                                     const int64_t *probe_pay,
                                     uint64_t probe_len,
                                     fi_join_result *result,
                                     fi_stream_t stream);

/* Hybrid join (cpu_partitioned_radix_join.rs:118-769): host columns in,
 * (sum, count) out.  The first pass runs on the CPU (threads host threads,
 * one canonical chunk each, 0 = all hardware threads, at most the engine's
 * chunk count) into the engine's pinned host buffers; the partitioned
 * relations and their Chunked offsets are copied to the device, and the
 * GPU runs the second pass and the join.  The CPU partitions S while the GPU
 * copies and partitions R.  Needs a two-pass plan.  Synchronous. */
int fi_radix_join_engine_run_hybrid_int32(fi_radix_join_engine *e,
                                          const int32_t *build_key,
                                          const int32_t *build_pay,
                                          uint64_t build_len,
                                          const int32_t *probe_key,
                                          const int32_t *probe_pay,
                                          uint64_t probe_len, uint32_t threads,
                                          fi_join_result *result,
                                          fi_stream_t stream);
int fi_radix_join_engine_run_hybrid_int64(fi_radix_join_engine *e,
                                          const int64_t *build_key,
                                          const int64_t *build_pay,
                                          uint64_t build_len,
                                          const int64_t *probe_key,
                                          const int64_t *probe_pay,
                                          uint64_t probe_len, uint32_t threads,
                                          fi_join_result *result,
                                          fi_stream_t stream);

/* Out-of-core join (no reference counterpart; the nearest reference pieces
 * are the chunked multi-stream copy of numa-gpu/src/runtime/cuda.rs:891-985
 * and the cache-and-spill staging of gpu_triton_join.rs:391-470).  The four
 * columns stay in host memory (pinned for overlap).  The first radix pass
 * streams them over the host link once, in blocks of `block_tuples` tuples
 * (0 = 2^26; rounded up to a multiple of 2^16), with two device staging
 * slots so that the copy of block j+1 overlaps the partitioning of block j.
 * The partitioned relations, the second pass and the join stay in HBM.  A
 * relation may span at most SM-count blocks.  The engine's plan must have
 * two passes.  Same result as fi_radix_join_engine_run_*; `result` is host
 * memory.  Synchronous. */
int fi_radix_join_engine_run_streamed_int32(
    fi_radix_join_engine *e, const int32_t *build_key, const int32_t *build_pay,
    uint64_t build_len, const int32_t *probe_key, const int32_t *probe_pay,
    uint64_t probe_len, uint64_t block_tuples, fi_join_result *result,
    fi_stream_t stream);
int fi_radix_join_engine_run_streamed_int64(
    fi_radix_join_engine *e, const int64_t *build_key, const int64_t *build_pay,
    uint64_t build_len, const int64_t *probe_key, const int64_t *probe_pay,
    uint64_t probe_len, uint64_t block_tuples, fi_join_result *result,
    fi_stream_t stream);

/* gpu_radix_join over device-resident columns: prefix sum, partition (one
 * or two passes) and per-partition join, all enqueued on `stream`.
 * `result` is a device fi_join_result that receives the result (it is
 * overwritten).  Asynchronous. */
int fi_radix_join_engine_run_int32(fi_radix_join_engine *e,
                                   const int32_t *build_key,
                                   const int32_t *build_pay, uint64_t build_len,
                                   const int32_t *probe_key,
                                   const int32_t *probe_pay, uint64_t probe_len,
                                   fi_join_result *result, fi_stream_t stream);
int fi_radix_join_engine_run_int64(fi_radix_join_engine *e,
                                   const int64_t *build_key,
                                   const int64_t *build_pay, uint64_t build_len,
                                   const int64_t *probe_key,
                                   const int64_t *probe_pay, uint64_t probe_len,
                                   fi_join_result *result, fi_stream_t stream);

/* Same join from host memory (ideally pinned): copies the four columns to
 * the device inside the call, runs the join and copies the result back into
 * the host `result`.  Synchronous.  With two radix passes the columns are
 * streamed as by fi_radix_join_engine_run_streamed_* (blocks of 2^26 tuples,
 * or len / SM count when larger), so the first pass overlaps the copy; with
 * one pass they are copied whole first. */
int fi_radix_join_engine_run_host_int32(fi_radix_join_engine *e,
                                        const int32_t *build_key,
                                        const int32_t *build_pay,
                                        uint64_t build_len,
                                        const int32_t *probe_key,
                                        const int32_t *probe_pay,
                                        uint64_t probe_len,
                                        fi_join_result *result,
                                        fi_stream_t stream);
int fi_radix_join_engine_run_host_int64(fi_radix_join_engine *e,
                                        const int64_t *build_key,
                                        const int64_t *build_pay,
                                        uint64_t build_len,
                                        const int64_t *probe_key,
                                        const int64_t *probe_pay,
                                        uint64_t probe_len,
                                        fi_join_result *result,
                                        fi_stream_t stream);

/* Synchronises and reports (and clears) a device-side error of the engine. */
int fi_radix_join_engine_status(fi_radix_join_engine *e);
/* The same without a device-wide synchronisation: enqueues on `stream` a
 * copy of the engine's device error word (0 or an FI_ERR_* code) into the
 * host int `host_status` (pinned, valid once the stream reaches it) and
 * clears the word.  For callers that overlap engines with other work. */
int fi_radix_join_engine_status_async(fi_radix_join_engine *e, int *host_status,
                                      fi_stream_t stream);

/* ---- batched small joins (no reference counterpart; the reference runs
 *      one join per gpu_radix_join call) ---------------------------------- */

/* A batch runs many small joins of one tuple type at once: one radix pass
 * per job, all jobs' histograms, scans, scatters and per-partition joins as
 * four kernels over the whole batch, replayed as one CUDA graph (the join
 * kernel takes (job, partition) items from a device work queue).  A batch
 * handle owns a partition arena of max_tuples tuples (build + probe of all
 * jobs) and holds at most max_jobs (<= 1024) jobs. */
typedef struct fi_join_batch fi_join_batch;
typedef struct {
  const void *build_key, *build_pay, *probe_key, *probe_pay; /* device */
  uint64_t build_len, probe_len;
  int32_t radix_bits; /* <= 12; -1 = chosen from build_len */
} fi_batch_job;
int fi_join_batch_new(uint32_t tuple_bytes, uint32_t max_jobs,
                      uint64_t max_tuples, fi_join_batch **out);
void fi_join_batch_free(fi_join_batch *b);
uint64_t fi_join_batch_device_bytes(const fi_join_batch *b);
/* Runs the jobs; results[i] (host) gets job i's {sum, count}.  Synchronous.
 * Jobs beyond the batch's capacity fail with FI_ERR_CAPACITY. */
int fi_join_batch_run(fi_join_batch *b, const fi_batch_job *jobs,
                      uint32_t n_jobs, fi_join_result *results);

/* Phase timing (no reference counterpart; the reference times its phases
 * with CUDA events in gpu_radix_join.rs:255-276,281-356,415-532).  When
 * `events` (cudaEvent_t[n_events], n_events >= FI_ENGINE_PHASE_EVENTS) is
 * set, every run records events[i] on its stream after phase i:
 *   0 start, then per relation r in {build, probe}: 1+4r pass-1 histogram,
 *   2+4r pass-1 scatter, 3+4r pass-2 plan + histogram + cursors,
 *   4+4r pass-2 scatter; 9 join; 10 result.
 * Pass NULL to stop recording. */
#define FI_ENGINE_PHASE_EVENTS 11
int fi_radix_join_engine_set_events(fi_radix_join_engine *e, void **events,
                                    uint32_t n_events);

/* Number of kernels the last run launched. */
uint32_t fi_radix_join_engine_last_launches(const fi_radix_join_engine *e);

/* ---- seeded relation generator (datagen/src/relation.rs counterpart) -- */

/* keys[i] = base + perm(i), a seeded permutation of base..base+n-1. */
int fi_datagen_primary_keys_int32(int32_t *keys, uint64_t n, uint64_t seed,
                                  int32_t base, fi_stream_t stream);
int fi_datagen_primary_keys_int64(int64_t *keys, uint64_t n, uint64_t seed,
                                  int64_t base, fi_stream_t stream);
/* Uniform foreign keys over base..base+pk_n-1. */
int fi_datagen_uniform_foreign_keys_int32(int32_t *keys, uint64_t n,
                                          uint64_t pk_n, uint64_t seed,
                                          int32_t base, fi_stream_t stream);
int fi_datagen_uniform_foreign_keys_int64(int64_t *keys, uint64_t n,
                                          uint64_t pk_n, uint64_t seed,
                                          int64_t base, fi_stream_t stream);
/* Zipf(s) ranks over pk_n primary keys generated with pk_seed, mapped to
 * their keys (s = 0: uniform ranks). */
int fi_datagen_zipf_foreign_keys_int32(int32_t *keys, uint64_t n,
                                       uint64_t pk_n, double s, uint64_t seed,
                                       uint64_t pk_seed, int32_t base,
                                       fi_stream_t stream);
int fi_datagen_zipf_foreign_keys_int64(int64_t *keys, uint64_t n,
                                       uint64_t pk_n, double s, uint64_t seed,
                                       uint64_t pk_seed, int64_t base,
                                       fi_stream_t stream);
/* Uniform 64-bit keys. */
int fi_datagen_uniform_u64_keys(int64_t *keys, uint64_t n, uint64_t seed,
                                fi_stream_t stream);
/* Join selectivity (datagen/src/relation.rs:85-151, the `selectivity`
 * argument of the reference's primary-key generators): every key k of the
 * column stays when a seeded uniform draw from 0..100, a function of
 * (seed, k - base), is at most `selectivity` percent, and becomes the null
 * key (all ones) otherwise.  Applied to primary keys base..base+n-1, a
 * foreign key f then matches iff f's draw kept it.  selectivity >= 100
 * keeps every key. */
int fi_datagen_null_keys_int32(int32_t *keys, uint64_t n, uint32_t selectivity,
                               uint64_t seed, int32_t base, fi_stream_t stream);
int fi_datagen_null_keys_int64(int64_t *keys, uint64_t n, uint32_t selectivity,
                               uint64_t seed, int64_t base, fi_stream_t stream);

/* ---- data sets and relation files (datagen/src/popular.rs,
 *      radix-join/src/main.rs:657-760, data-store/src/join_data.rs) ----- */

/* The reference's named data sets: primary-key relation R (build) and
 * uniform foreign-key relation S (probe).  Blanas (SIGMOD 2011):
 * 16 x 2^20 and 256 x 2^20 tuples, 8-byte keys in the paper; Blanas4MB:
 * 512 x 2^10 and 256 x 2^20; Kim (PVLDB 2009): 128e6 and 128e6 tuples,
 * 4-byte keys in the paper; Test: 1000 and 1000; Lutz2Gv32G and
 * Lutz32Gv32G: 2 GiB and 32 GiB, 32 GiB and 32 GiB of tuples of
 * tuple_bytes each. */
typedef enum {
  FI_DATASET_BLANAS = 0,
  FI_DATASET_BLANAS4MB = 1,
  FI_DATASET_KIM = 2,
  FI_DATASET_TEST = 3,
  FI_DATASET_LUTZ2GV32G = 4,
  FI_DATASET_LUTZ32GV32G = 5
} fi_dataset;
int fi_dataset_shape(fi_dataset d, uint32_t tuple_bytes, uint64_t *build_len,
                     uint64_t *probe_len);

/* Relation files of the reference's file-backed join data
 * (data-store/src/join_data.rs:173-260, build_with_files): one header line,
 * then one tuple per line, key and payload as decimal integers separated by
 * one space; a file whose name ends in "gz" is gzip-compressed.  Like the
 * reference, loading takes two passes: fi_relation_file_len counts the
 * tuples, fi_relation_file_read_* parses them into caller-owned host columns
 * of exactly that length.  A malformed line (other than two fields, not a
 * decimal integer, out of the key type's range) is an InvalidArgument error
 * naming the file and line; empty lines are skipped.  Host only. */
int fi_relation_file_len(const char *path, uint64_t *len);
int fi_relation_file_read_int32(const char *path, int32_t *keys, int32_t *pays,
                                uint64_t len);
int fi_relation_file_read_int64(const char *path, int64_t *keys, int64_t *pays,
                                uint64_t len);

/* ---- autotuner and join server (no reference counterpart; the nearest
 *      reference pieces are the radix-bits heuristic of
 *      scripts/benchmark_gpu_radix_join.py:92 and the two reused
 *      StreamStates of gpu_radix_join.rs:51-68,321-396) ------------------ */

/* What the autotuner chooses per (tuple type, |R|, |S|, skew). */
typedef struct {
  uint32_t batched;       /* 1: run in a batch of small joins */
  fi_radix_bits radix_bits;
  fi_hashing_scheme hashing_scheme;
  uint32_t join_block;    /* threads per join CTA */
  uint32_t scatter;       /* 0 TMA-fed tile scatter, 1 register-fed */
} fi_tuned_plan;

/* The plan for one join.  skew: 0 uniform probe keys, 1 skewed (Zipf).
 * Joins below small_tuples (0 = 4M) tuples in total are batched.  Others
 * use the nearest entry of the table loaded by fi_autotune_load (by tuple
 * type, log2 |R|, log2 (|S|/|R|) and skew) or, without one, a model: about
 * 4K build tuples per final partition, one pass up to 11 bits and two
 * balanced passes above, bucket chaining, 256-thread join CTAs, TMA-fed
 * scatters.  A table entry may name the perfect scheme, which is valid
 * only for dense unique build keys. */
int fi_autotune_plan(uint32_t tuple_bytes, uint64_t build_len,
                     uint64_t probe_len, uint32_t skew, uint64_t small_tuples,
                     fi_tuned_plan *out);
/* Loads a measured table (text lines "tuple_bytes log2_build log2_ratio
 * skew bits1 bits2 scheme join_block scatter", '#' comments), replacing
 * the previous one; NULL clears it. */
int fi_autotune_load(const char *path);

typedef struct fi_join_server fi_join_server;

typedef struct {
  uint64_t hbm_budget_bytes; /* device memory the server may hold (0: 150e9):
                                the workers' engines, the batch arenas and a
                                slab for the relations it holds (the rest,
                                capped by the device's free memory) */
  uint32_t workers;          /* concurrent large joins (0: 2, or 1 when two
                                engines would take over half the budget) */
  uint64_t small_tuples;     /* joins below this (|R|+|S|) are batched (0: 4M) */
  uint32_t max_batch_jobs;   /* jobs per batch (0: 256) */
  uint64_t batch_tuples;     /* partition arena of one batch (0: 2^25) */
  uint32_t batch_wait_us;    /* longest wait for a fuller batch (0: 200) */
  uint64_t max_build;        /* largest build relation (0: 2^28 tuples) */
  uint64_t probe_slice;      /* probe tuples per engine probe (0: 2^28) */
} fi_join_server_config;

/* Where a request's relations come from. */
typedef enum {
  FI_SOURCE_DEVICE = 0,    /* device columns owned by the caller, ready when
                              submitted and valid until the response */
  FI_SOURCE_HOST = 1,      /* host columns: the server reserves device memory
                              and copies them in */
  FI_SOURCE_SYNTHETIC = 2  /* the server generates them: R keys a permutation
                              of 1..|R| (seed), S keys foreign keys of R,
                              uniform or Zipf(zipf_s) (seed + 1), payload =
                              key */
} fi_join_source;

typedef struct {
  uint32_t tuple_bytes; /* 8: (int32, int32); 16: (int64, int64) */
  uint32_t source;      /* fi_join_source */
  uint64_t build_len, probe_len;
  const void *build_key, *build_pay, *probe_key, *probe_pay;
  uint64_t seed;  /* FI_SOURCE_SYNTHETIC */
  double zipf_s;  /* FI_SOURCE_SYNTHETIC; > 0 is also the autotuner's skew hint */
} fi_join_request;

typedef struct {
  int32_t status;         /* FI_OK or the error of this request */
  uint32_t batched;       /* 1: ran in a batch */
  fi_join_result result;
  uint32_t batch_jobs;    /* jobs in its batch */
  uint32_t reserved;
  double queue_us;        /* submit -> admitted (memory reserved) */
  double latency_us;      /* submit -> result in host memory */
} fi_join_response;

typedef struct {
  uint64_t submitted, completed, batches, batched_jobs, engine_runs;
  uint64_t reserved_bytes, peak_reserved_bytes, fixed_bytes;
  uint64_t arena_bytes;   /* device slab for the relations the server holds */
  double engine_busy_us;  /* device time of the large joins (events) */
  double batch_busy_us;   /* device time of the batches (events) */
  double enqueue_us;      /* host time the scheduler spent issuing work */
  uint64_t workers;       /* engines running large joins (the config's, or
                             the automatic choice for workers = 0) */
} fi_join_server_stats;

/* Starts a server on the current device: allocates the workers' engines and
 * the batch runners (fixed_bytes of the budget) and a scheduler thread. */
int fi_join_server_new(const fi_join_server_config *cfg, fi_join_server **out);
/* Finishes the queued requests and releases everything. */
void fi_join_server_free(fi_join_server *s);
/* Queues one join and returns its ticket at once.  The scheduler admits it
 * when its memory fits the budget, runs it (batched, or on a worker's
 * engine, overlapping with other requests) and keeps the response until it
 * is collected. */
int fi_join_server_submit(fi_join_server *s, const fi_join_request *req,
                          uint64_t *ticket);
/* Blocks until the ticket's join is done; the response is handed over. */
int fi_join_server_wait(fi_join_server *s, uint64_t ticket,
                        fi_join_response *resp);
/* Non-blocking: *done = 1 and the response handed over when finished. */
int fi_join_server_poll(fi_join_server *s, uint64_t ticket, int *done,
                        fi_join_response *resp);
int fi_join_server_stats_get(fi_join_server *s, fi_join_server_stats *out);

#ifdef __cplusplus
}
#endif

#endif /* FI_SQLOPS_H */
