// Radix-partition scatter kernels (sm_100a).
//
// Replaces the reference's scatter variants NC, LASWWC, SSWWCv2, SSWWCv2G and
// HSSWWCv4 (sql-ops/cudautils/radix_partition.cu:472-1477).  Every variant
// writes tuple (key, payload) of chunk c with partition p into the slots
// [cursors[c*F+p], ...) of the partitioned relation, so the per-(chunk,
// partition) tuple multisets equal the reference's; padding is never written.
//
// B200 design of the write-combining scatter ("tile scatter",
// tile_scatter.cuh):
//  * One CTA owns one chunk (the Chunked layout's unit) and walks it in tiles.
//    The next tile's keys and payloads are brought into a shared-memory
//    stage by TMA bulk copies (tma_scatter.cuh) while the current tile is
//    processed, so HBM reads stay in flight across the block barriers and
//    the CTA can run 1024 threads.  Columns that are not 16-byte aligned, or
//    fanouts whose stages do not fit shared memory, use the same algorithm
//    with a register double buffer (tile_scatter.cuh).
//  * Each tile is counting-sorted by partition in shared memory (shared
//    atomic ranks + a block scan of the tile histogram) into a staging
//    buffer, then written out in partition runs: consecutive threads write
//    consecutive tuples of a run, so a warp store covers a few contiguous
//    128-byte segments instead of 32 scattered ones.  Partially written
//    lines are completed by the next tiles while they sit in the 126 MB L2,
//    which therefore acts as the write-combining buffer that the reference
//    keeps in shared memory and flushes under warp locks.
//  * No device-side waits: the only synchronisation is __syncthreads.
//  * Every store is bounds-checked against the relation's length.
#include "common.cuh"
#include "kernels.h"
#include "tile_scatter.cuh"
#include "tma_scatter.cuh"

namespace fi {

// One CTA per canonical chunk of column input.
template <typename K, typename S>
__global__ void __launch_bounds__(S::kThreads, S::kMinBlocks)
    tile_scatter_kernel(const K *__restrict__ keys, const K *__restrict__ pays,
                        uint64_t len, uint64_t clen, uint32_t chunks,
                        uint32_t radix_bits, uint32_t ignore_bits,
                        const uint64_t *__restrict__ cursors,
                        Tuple<K> *__restrict__ out, uint64_t out_len,
                        int *status) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const uint32_t F = 1u << radix_bits;
  const uint64_t mask = static_cast<uint64_t>(F - 1u) << ignore_bits;
  Tuple<K> *staged = reinterpret_cast<Tuple<K> *>(smem_raw);
  uint32_t *toff = reinterpret_cast<uint32_t *>(staged + S::kTile);
  uint32_t *cur = toff + F + 1;
  uint32_t *scan_tmp = cur + F;

  const uint32_t c = blockIdx.x;
  const uint64_t cb = clen * c, ce = (c + 1 == chunks) ? len : cb + clen;
  const uint64_t base = cursors[(uint64_t)c * F];
  for (uint32_t p = threadIdx.x; p < F; p += blockDim.x) {
    cur[p] = (uint32_t)(cursors[(uint64_t)c * F + p] - base);
    toff[p] = 0;
  }
  if (threadIdx.x == 0) toff[F] = 0;
  __syncthreads();
  ColumnSource<K> src{keys, pays};
  tile_scatter_range<K, S>(src, cb, ce, F, mask, ignore_bits, cur, toff,
                           scan_tmp, staged, out, base, out_len, status);
}

// Same as tile_scatter_kernel with TMA-fed input stages (tma_scatter.cuh).
// Shared memory: bars | stages | toff | cur | scan_tmp.
template <typename K>
__global__ void __launch_bounds__(TmaShape<K>::kThreads, 1)
    tma_tile_scatter_kernel(const K *__restrict__ keys,
                            const K *__restrict__ pays, uint64_t len,
                            uint64_t clen, uint32_t chunks, uint32_t radix_bits,
                            uint32_t ignore_bits,
                            const uint64_t *__restrict__ cursors,
                            Tuple<K> *__restrict__ out, uint64_t out_len,
                            int *status) {
  using S = TmaShape<K>;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const uint32_t F = 1u << radix_bits;
  const uint64_t mask = static_cast<uint64_t>(F - 1u) << ignore_bits;
  uint64_t *bars = reinterpret_cast<uint64_t *>(smem_raw);
  unsigned char *stages = smem_raw + 64;
  uint32_t *toff =
      reinterpret_cast<uint32_t *>(stages + S::kStages * tma_stage_bytes<K>());
  uint32_t *cur = toff + F + 1;
  uint32_t *scan_tmp = cur + F;

  const uint32_t c = blockIdx.x;
  const uint64_t cb = clen * c, ce = (c + 1 == chunks) ? len : cb + clen;
  const uint64_t base = cursors[(uint64_t)c * F];
  for (uint32_t p = threadIdx.x; p < F; p += blockDim.x)
    cur[p] = (uint32_t)(cursors[(uint64_t)c * F + p] - base);
  for (uint32_t p = threadIdx.x; p <= F; p += blockDim.x) toff[p] = 0;
  if (threadIdx.x == 0) {
    for (uint32_t s = 0; s < S::kStages; ++s) mbar_init(&bars[s], 1);
    mbar_fence_init();
  }
  __syncthreads();
  TmaColumnSource<K> src{keys, pays};
  tma_tile_scatter_range<K>(src, cb, ce, F, mask, ignore_bits, cur, toff,
                            scan_tmp, stages, bars, out, base, out_len,
                            status);
}

// Non-caching scatter: one shared-memory atomic per tuple and a direct
// store (the reference's NC, radix_partition.cu:472-525).
template <typename K>
__global__ void __launch_bounds__(1024)
    nc_scatter_kernel(const K *__restrict__ keys, const K *__restrict__ pays,
                      uint64_t len, uint64_t clen, uint32_t chunks,
                      uint32_t radix_bits, uint32_t ignore_bits,
                      const uint64_t *__restrict__ cursors,
                      Tuple<K> *__restrict__ out, uint64_t out_len,
                      int *status) {
  extern __shared__ uint32_t cur[];
  const uint32_t F = 1u << radix_bits;
  const uint64_t mask = static_cast<uint64_t>(F - 1u) << ignore_bits;
  const uint32_t c = blockIdx.x;
  const uint64_t cb = clen * c, ce = (c + 1 == chunks) ? len : cb + clen;
  const uint64_t base = cursors[(uint64_t)c * F];
  for (uint32_t p = threadIdx.x; p < F; p += blockDim.x)
    cur[p] = (uint32_t)(cursors[(uint64_t)c * F + p] - base);
  __syncthreads();
  for (uint64_t i = cb + threadIdx.x; i < ce; i += blockDim.x) {
    const K k = load_cs(keys + i), v = load_cs(pays + i);
    const uint32_t p = key_to_partition(k, mask, ignore_bits);
    const uint64_t dst = base + atomicAdd(&cur[p], 1u);
    if (dst < out_len)
      store_tuple(out + dst, Tuple<K>{k, v});
    else
      record_error(status, kDevErrCapacity);
  }
}

// Level 2 of the hierarchical scatter: CTA per (chunk, high bucket) region
// of the level-1 buffer; scatters it by the low bits into the final slots.
template <typename K, typename S>
__global__ void __launch_bounds__(S::kThreads, S::kMinBlocks)
    hierarchical_level2_kernel(const Tuple<K> *__restrict__ tmp,
                               const uint64_t *__restrict__ tmp_cursors,
                               uint64_t len, uint32_t chunks, uint32_t hi_bits,
                               uint32_t lo_bits, uint32_t ignore_bits,
                               const uint64_t *__restrict__ cursors,
                               Tuple<K> *__restrict__ out, uint64_t out_len,
                               int *status) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const uint32_t FH = 1u << hi_bits, FL = 1u << lo_bits, F = FH * FL;
  const uint64_t mask = static_cast<uint64_t>(FL - 1u) << ignore_bits;
  Tuple<K> *staged = reinterpret_cast<Tuple<K> *>(smem_raw);
  uint32_t *toff = reinterpret_cast<uint32_t *>(staged + S::kTile);
  uint32_t *cur = toff + FL + 1;
  uint32_t *scan_tmp = cur + FL;

  const uint32_t item = blockIdx.x;  // c * FH + h
  const uint32_t c = item / FH, h = item % FH;
  const uint64_t begin = tmp_cursors[item];
  const uint64_t end = (item + 1 < chunks * FH) ? tmp_cursors[item + 1] : len;
  if (begin >= end) return;
  const uint64_t *cp = cursors + (uint64_t)c * F + (uint64_t)h * FL;
  const uint64_t base = cp[0];
  for (uint32_t p = threadIdx.x; p < FL; p += blockDim.x) {
    cur[p] = (uint32_t)(cp[p] - base);
    toff[p] = 0;
  }
  if (threadIdx.x == 0) toff[FL] = 0;
  __syncthreads();
  TupleSource<K> src{tmp};
  tile_scatter_range<K, S>(src, begin, end, FL, mask, ignore_bits, cur, toff,
                           scan_tmp, staged, out, base, out_len, status);
}

uint32_t hierarchical_hi_bits(uint32_t radix_bits) { return (radix_bits + 1) / 2; }

// Tuples of final region (c, p) under the cursor layout: Chunked offsets
// (region (c, p) ends where (c, p+1) starts minus padding, a chunk's last
// region where the next chunk's first starts minus padding, the relation's
// last at its padded length), or Contiguous per-block cursors (block c's
// share of partition p ends where block c+1's share starts; the last
// block's where partition p+1 starts minus padding).
__device__ __forceinline__ uint64_t region_len(const uint64_t *cur, uint32_t c,
                                               uint32_t p, uint32_t chunks,
                                               uint32_t F, uint32_t pad,
                                               bool contiguous,
                                               uint64_t padded_len) {
  const uint64_t i = (uint64_t)c * F + p;
  uint64_t next;
  if (contiguous) {
    if (c + 1 < chunks)
      next = cur[i + F];
    else
      next = (p + 1 < F) ? cur[p + 1] - pad : padded_len;
  } else {
    next = (p + 1 < F || c + 1 < chunks) ? cur[i + 1] - pad : padded_len;
  }
  return next - cur[i];
}

// Level-1 layout of the hierarchical scatter from the final cursors, one CTA
// per chunk: high bucket h of chunk c (the final regions (c, h*FL) ..
// (c, h*FL + FL - 1)) starts at c * clen + the tuples of the chunk's buckets
// before it, so a chunk's buckets fill its input range of `tmp`.  Replaces a
// second histogram pass over the keys.
__global__ void hierarchical_layout_kernel(const uint64_t *__restrict__ cursors,
                                           uint32_t chunks, uint32_t radix_bits,
                                           uint32_t hi, uint32_t pad,
                                           bool contiguous, uint64_t padded_len,
                                           uint64_t clen,
                                           uint64_t *__restrict__ tmp_cursors) {
  __shared__ uint64_t scan[33];
  const uint32_t c = blockIdx.x, F = 1u << radix_bits, FH = 1u << hi;
  const uint32_t FL = F >> hi;
  uint64_t run = (uint64_t)c * clen;
  for (uint32_t h0 = 0; h0 < FH; h0 += blockDim.x) {
    const uint32_t h = h0 + threadIdx.x;
    uint64_t n = 0;
    if (h < FH)
      for (uint32_t l = 0; l < FL; ++l)
        n += region_len(cursors, c, h * FL + l, chunks, F, pad, contiguous,
                        padded_len);
    uint64_t total;
    const uint64_t ex = block_exclusive_scan_u64(n, scan, &total);
    if (h < FH) tmp_cursors[(uint64_t)c * FH + h] = run + ex;
    run += total;
  }
}

template <typename K, typename S>
static cudaError_t launch_tile_shape(const K *keys, const K *pays, uint64_t len,
                                     uint64_t clen, uint32_t chunks,
                                     uint32_t radix_bits, uint32_t ignore_bits,
                                     const uint64_t *cursors, void *out,
                                     uint64_t out_len, int *status,
                                     cudaStream_t stream) {
  const size_t sm = tile_scatter_smem<K, S>(1u << radix_bits);
  cudaError_t e = cudaFuncSetAttribute(
      (const void *)tile_scatter_kernel<K, S>,
      cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
  if (e != cudaSuccess) return e;
  tile_scatter_kernel<K, S><<<chunks, S::kThreads, sm, stream>>>(
      keys, pays, len, clen, chunks, radix_bits, ignore_bits, cursors,
      reinterpret_cast<Tuple<K> *>(out), out_len, status);
  return cudaGetLastError();
}

// The wide shape: longer partition runs per tile coalesce better than two
// narrower CTAs per SM (measured on B200: 4.6 vs 3.4 TB/s at 512 partitions).
template <typename K>
static cudaError_t launch_tile(const K *keys, const K *pays, uint64_t len,
                               uint32_t chunks, uint32_t radix_bits,
                               uint32_t ignore_bits, const uint64_t *cursors,
                               void *out, uint64_t out_len, int *status,
                               cudaStream_t stream, bool allow_tma = true) {
  constexpr uint64_t kAlignMask = ~((uint64_t)(kAlignBytes / sizeof(K)) - 1ull);
  const uint64_t clen = ((len + chunks - 1) / chunks) & kAlignMask;
  // TMA-fed stages when both columns are 16-byte aligned and the stages fit
  const size_t tma_sm = tma_scatter_smem<K>(1u << radix_bits);
  if (allow_tma && (reinterpret_cast<uintptr_t>(keys) % 16) == 0 &&
      (reinterpret_cast<uintptr_t>(pays) % 16) == 0 &&
      tma_sm <= (size_t)device_max_smem_optin()) {
    cudaError_t e = cudaFuncSetAttribute(
        (const void *)tma_tile_scatter_kernel<K>,
        cudaFuncAttributeMaxDynamicSharedMemorySize, (int)tma_sm);
    if (e != cudaSuccess) return e;
    tma_tile_scatter_kernel<K><<<chunks, TmaShape<K>::kThreads, tma_sm, stream>>>(
        keys, pays, len, clen, chunks, radix_bits, ignore_bits, cursors,
        reinterpret_cast<Tuple<K> *>(out), out_len, status);
    return cudaGetLastError();
  }
  return launch_tile_shape<K, TileWide<K>>(keys, pays, len, clen, chunks,
                                           radix_bits, ignore_bits, cursors,
                                           out, out_len, status, stream);
}

template <typename K>
cudaError_t launch_partition(const K *keys, const K *pays, uint64_t len,
                             uint32_t chunks, uint32_t radix_bits,
                             uint32_t ignore_bits, const uint64_t *cursors,
                             void *out, uint64_t out_len, int variant,
                             int *status, cudaStream_t stream) {
  const uint32_t F = 1u << radix_bits;
  if (variant == kScatterNC) {
    constexpr uint64_t kAlignMask =
        ~((uint64_t)(kAlignBytes / sizeof(K)) - 1ull);
    const uint64_t clen = ((len + chunks - 1) / chunks) & kAlignMask;
    const size_t sm = (size_t)F * sizeof(uint32_t);
    cudaError_t e = cudaFuncSetAttribute(
        (const void *)nc_scatter_kernel<K>,
        cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
    if (e != cudaSuccess) return e;
    nc_scatter_kernel<K><<<chunks, 1024, sm, stream>>>(
        keys, pays, len, clen, chunks, radix_bits, ignore_bits, cursors,
        reinterpret_cast<Tuple<K> *>(out), out_len, status);
    return cudaGetLastError();
  }
  return launch_tile<K>(keys, pays, len, chunks, radix_bits, ignore_bits,
                        cursors, out, out_len, status, stream,
                        variant != kScatterRegisters);
}

template <typename K>
cudaError_t launch_partition_hierarchical(
    const K *keys, const K *pays, uint64_t len, uint32_t chunks,
    uint32_t radix_bits, uint32_t ignore_bits, const uint64_t *cursors,
    bool contiguous, uint64_t padded_len, void *out, uint64_t out_len,
    void *tmp, uint64_t *tmp_cursors, HistScratch s, uint32_t sm_count,
    cudaStream_t stream) {
  using S = TileWide<K>;
  const uint32_t hi = hierarchical_hi_bits(radix_bits), lo = radix_bits - hi;
  // level-1 layout: same canonical chunks, partitions by the high bits, no
  // padding; bucket sizes are sums of the final regions' sizes
  constexpr uint64_t kAlignMask = ~((uint64_t)(kAlignBytes / sizeof(K)) - 1ull);
  const uint64_t clen = ((len + chunks - 1) / chunks) & kAlignMask;
  hierarchical_layout_kernel<<<chunks, 256, 0, stream>>>(
      cursors, chunks, radix_bits, hi, (uint32_t)(kPaddingBytes / sizeof(Tuple<K>)),
      contiguous, padded_len, clen, tmp_cursors);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return e;
  e = launch_tile<K>(keys, pays, len, chunks, hi, ignore_bits + lo,
                     tmp_cursors, tmp, len, s.status, stream);
  if (e != cudaSuccess) return e;
  const size_t sm = tile_scatter_smem<K, S>(1u << lo);
  e = cudaFuncSetAttribute((const void *)hierarchical_level2_kernel<K, S>,
                           cudaFuncAttributeMaxDynamicSharedMemorySize,
                           (int)sm);
  if (e != cudaSuccess) return e;
  hierarchical_level2_kernel<K, S><<<chunks << hi, S::kThreads, sm, stream>>>(
      reinterpret_cast<const Tuple<K> *>(tmp), tmp_cursors, len, chunks, hi,
      lo, ignore_bits, cursors, reinterpret_cast<Tuple<K> *>(out), out_len,
      s.status);
  return cudaGetLastError();
}

#define FI_INSTANTIATE_PARTITION(K)                                            \
  template cudaError_t launch_partition<K>(                                    \
      const K *, const K *, uint64_t, uint32_t, uint32_t, uint32_t,            \
      const uint64_t *, void *, uint64_t, int, int *, cudaStream_t);           \
  template cudaError_t launch_partition_hierarchical<K>(                       \
      const K *, const K *, uint64_t, uint32_t, uint32_t, uint32_t,            \
      const uint64_t *, bool, uint64_t, void *, uint64_t, void *, uint64_t *,  \
      HistScratch, uint32_t, cudaStream_t);

FI_INSTANTIATE_PARTITION(int32_t)
FI_INSTANTIATE_PARTITION(int64_t)

}  // namespace fi
