// Host-side launchers of the sm_100a kernels (internal C++ interface between
// the kernels and the C ABI in api.cu).  All launchers enqueue work on
// `stream` and return the cudaError_t of the launch.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

namespace fi {

// Device scratch a histogram launch needs.  All arrays are owned by the
// caller (a partitioner handle, an engine or the allocation-free entry
// points) and must be zero on entry; the kernels leave them zero again.
struct HistScratch {
  uint32_t *hist;        // [chunks * fanout] per-chunk histograms
  uint64_t *tile_state;  // [fanout / kScanTile + 1] look-back state
  uint32_t *tile_counter;// [1] dynamic tile ids of the look-back scan
  int *status;           // [1] device error word (0 = ok)
};

constexpr uint32_t kScanTile = 32;  // partitions per look-back tile

// Number of CTAs that share one chunk in the histogram kernels.
uint32_t hist_splits(uint32_t chunks, uint32_t sm_count);

// Chunked prefix sum (reference radix_partition.cu:40-96 semantics):
// offsets[c*F+p] = excl_c[p] + (chunk_len + pad*F)*c + (p+1)*pad.
template <typename K>
cudaError_t launch_chunked_prefix_sum(const K *keys, uint64_t len,
                                      uint32_t chunks, uint32_t radix_bits,
                                      uint32_t ignore_bits, uint32_t pad,
                                      uint64_t *offsets, HistScratch s,
                                      uint32_t sm_count, cudaStream_t stream);

// Contiguous prefix sum (radix_partition.cu:105-199 semantics) over the
// canonical chunks of `grid` blocks: offsets[p] and local_offsets[b*F+p],
// both shifted by `base` slots (0 for the reference's semantics; the
// streamed pass 1 places each block of the input at its own base).
// When dst_key/dst_pay are given the columns are also copied
// (prefix_sum_and_copy_with_payload, radix_partition.cu:207-315).
template <typename K>
cudaError_t launch_contiguous_prefix_sum(const K *keys, const K *pays,
                                         uint64_t len, uint32_t grid,
                                         uint32_t radix_bits,
                                         uint32_t ignore_bits, uint32_t pad,
                                         K *dst_key, K *dst_pay,
                                         uint64_t *offsets,
                                         uint64_t *local_offsets,
                                         uint64_t base, HistScratch s,
                                         uint32_t sm_count,
                                         cudaStream_t stream);

// prefix_sum_and_transform (radix_partition.cu:323-467 semantics).
template <typename K>
cudaError_t launch_prefix_sum_and_transform(
    uint32_t partition_id, const void *src_relation, const uint64_t *src_offsets,
    uint32_t src_chunks, uint32_t src_radix_bits, uint64_t src_padded_len,
    uint32_t src_pad, uint64_t dst_len, uint32_t grid, uint32_t radix_bits,
    uint32_t ignore_bits, uint32_t pad, K *dst_key, K *dst_pay,
    uint64_t *offsets, uint64_t *local_offsets, HistScratch s,
    uint32_t sm_count, cudaStream_t stream);

// Scatter variants: the shared-memory tile write-combining scatter, fed by
// TMA bulk copies where the columns allow it (kScatterAuto) or by register
// loads (kScatterRegisters), or the per-tuple atomic scatter (kScatterNC).
constexpr int kScatterAuto = 0;
constexpr int kScatterNC = 1;
constexpr int kScatterRegisters = 2;

// Scatter of columns into a partitioned relation.  cursors[c*F+p] is the
// first slot of (chunk c, partition p); the input is split into `chunks`
// canonical chunks.
template <typename K>
cudaError_t launch_partition(const K *keys, const K *pays, uint64_t len,
                             uint32_t chunks, uint32_t radix_bits,
                             uint32_t ignore_bits, const uint64_t *cursors,
                             void *out, uint64_t out_len, int variant,
                             int *status, cudaStream_t stream);

// Hierarchical (two-level) scatter for large fanouts: level 1 scatters by the
// high half of the pass bits into `tmp` (same chunking), level 2 scatters
// every (chunk, high bucket) by the low half into `out`.  tmp_cursors holds
// chunks * 2^hi_bits u64; tmp holds len tuples.  The level-1 layout comes
// from the final cursors (Chunked offsets, or Contiguous per-block cursors
// when `contiguous`; padded_len is the relation's padded length).
template <typename K>
cudaError_t launch_partition_hierarchical(
    const K *keys, const K *pays, uint64_t len, uint32_t chunks,
    uint32_t radix_bits, uint32_t ignore_bits, const uint64_t *cursors,
    bool contiguous, uint64_t padded_len, void *out, uint64_t out_len,
    void *tmp, uint64_t *tmp_cursors, HistScratch s, uint32_t sm_count,
    cudaStream_t stream);
uint32_t hierarchical_hi_bits(uint32_t radix_bits);


// ---- radix join ---------------------------------------------------------
struct JoinScratch {
  uint32_t *item_start;   // [fanout + 1]
  uint32_t *item_part;    // [join_items_capacity(fanout, probe_len)]
  uint64_t *tile_state;   // [fanout / 1024 + 2] look-back state of the plan
  uint32_t *tile_counter; // [1]
  int *status;
};

// Reference greedy task assignment (radix_join.cu:58-98).
template <typename K>
cudaError_t launch_assign_tasks(const uint64_t *probe_offsets,
                                uint32_t probe_len, uint32_t probe_pad,
                                uint32_t radix_bits, uint32_t grid,
                                uint32_t *tasks, cudaStream_t stream);

// Shared-memory per-partition join over all partitions.  scheme: 0 perfect,
// 2 bucket chaining.  The build/probe relations are Contiguous (one chunk):
// partition p spans [off[p], off[p+1]-pad), the last ends at len.
template <typename K>
cudaError_t launch_radix_join(const void *build, const uint64_t *build_off,
                              uint64_t build_len, uint32_t build_pad,
                              const void *probe, const uint64_t *probe_off,
                              uint64_t probe_len, uint32_t probe_pad,
                              uint32_t fanout, uint32_t ignore_bits, int scheme,
                              uint32_t grid, uint32_t block,
                              int64_t *result_set, uint64_t *match_count,
                              JoinScratch s, uint32_t sm_count,
                              cudaStream_t stream);
uint32_t join_items_capacity(uint32_t fanout, uint64_t probe_len);
// CTAs of `block` threads the join runs per SM (4, 2 or 1).
uint32_t join_ctas_per_sm(uint32_t block);
// Bucket-chaining join shape for `build_tuples` over `fanout` partitions:
// the block (256, 512 or 1024 threads) with the most CTAs per SM whose
// shared-memory table still holds an average partition with 1/8 headroom.
template <typename K>
uint32_t join_auto_block(uint64_t build_tuples, uint32_t fanout);

// ---- no-partitioning join ------------------------------------------------
template <typename K>
cudaError_t launch_ht_init(void *ht, uint64_t entries, cudaStream_t stream);
template <typename K>
cudaError_t launch_ht_build(int scheme, bool selective, void *ht,
                            uint64_t ht_size, const K *key, const K *pay,
                            uint64_t len, uint32_t grid, uint32_t block,
                            cudaStream_t stream);
template <typename K>
cudaError_t launch_ht_probe_sum(int scheme, const void *ht, uint64_t ht_size,
                                const K *key, const K *pay, uint64_t len,
                                uint64_t *result, uint32_t grid, uint32_t block,
                                cudaStream_t stream);

// Region-ordered probe (hash_join.cu): the probe side grouped by the table
// region of its first slot, slice by slice (tuples: slice * 2*sizeof(K)
// bytes of scratch, region_scratch: ht_region_scratch_bytes), then probed in
// that order so the active table region stays in L2.
// The scratch starts with a device status word (FI_ERR_TIMEOUT when a bounded
// wait of the grouping scatter gave up; word 1 is the in-order build's tile
// counter, word 2 the probe's "slice left in input order" flag), padded to
// kRegionStatusWords u32;
// grouping runs one chunk per SM, for at most kMaxRegionChunks SMs.
constexpr uint32_t kRegionStatusWords = 64;
constexpr uint32_t kMaxRegionChunks = 256;
uint32_t ht_region_bits(uint64_t size, uint32_t entry_bytes);
size_t ht_region_scratch_bytes(uint32_t region_bits);
template <typename K>
cudaError_t launch_ht_probe_grouped(int scheme, const void *ht, uint64_t ht_size,
                                    const K *key, const K *pay, uint64_t len,
                                    uint64_t *result, uint32_t grid, uint32_t block,
                                    uint32_t region_bits, void *tuples,
                                    uint32_t *region_scratch, uint64_t slice,
                                    uint32_t sm_count, cudaStream_t stream);
// Region-ordered build: the build side grouped the same way, slice by slice,
// then inserted in that order so the lines being written stay in L2.
template <typename K>
cudaError_t launch_ht_build_grouped(int scheme, bool selective, void *ht,
                                    uint64_t ht_size, const K *key, const K *pay,
                                    uint64_t len, uint32_t grid, uint32_t block,
                                    uint32_t region_bits, void *tuples,
                                    uint32_t *region_scratch, uint64_t slice,
                                    uint32_t sm_count, cudaStream_t stream);

// ---- generator -------------------------------------------------------------
template <typename K>
cudaError_t launch_gen_primary_keys(K *keys, uint64_t n, uint64_t seed, K base,
                                    cudaStream_t stream);
template <typename K>
cudaError_t launch_gen_uniform_fk(K *keys, uint64_t n, uint64_t pk_n,
                                  uint64_t seed, K base, cudaStream_t stream);
template <typename K>
cudaError_t launch_gen_zipf_fk(K *keys, uint64_t n, uint64_t pk_n, double s,
                               uint64_t seed, uint64_t pk_seed, K base,
                               cudaStream_t stream);
template <typename K>
cudaError_t launch_null_keys(K *keys, uint64_t n, uint32_t selectivity,
                             uint64_t seed, K base, cudaStream_t stream);
cudaError_t launch_gen_uniform_u64(int64_t *keys, uint64_t n, uint64_t seed,
                                   cudaStream_t stream);

int device_sm_count();
int device_max_smem_optin();

}  // namespace fi
