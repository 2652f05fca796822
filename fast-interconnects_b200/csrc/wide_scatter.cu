// High-fanout radix partitioning in one HBM round trip (sm_100a).
//
// Above 11 radix bits a tile of a few thousand tuples holds one or two
// tuples per partition, so the tile scatter's shared-memory sort no longer
// buys coalesced runs, and with one CTA per chunk the partially written
// lines of chunks x 2^bits partitions (148 x 2^14 x 128 B = 310 MB at 14 bits)
// overflow the 126 MB L2, which then writes half-filled lines back to HBM.
//
// The wide scatter keeps the open lines in L2 instead: all CTAs walk the
// input together, tile by tile in input order (tiles come from a global
// counter, so no CTA drifts ahead), and the input order is chunk order, so
// only the partitions of one or two chunks are being written at any time:
// 2^bits x 128 B of open lines (2 MB at 14 bits, 34 MB at 18 bits).  Every
// tuple claims its slot with an atomic add on its (chunk, partition) cursor,
// aggregated over the lanes of a warp that share one (match.any), and is
// stored straight to its slot; L2 completes the lines.  The cursors are the
// partition offsets made relative to each chunk's first slot, in u32, in the
// partitioner's histogram scratch (chunks x 2^bits u32, idle after the
// prefix sum), L2-resident for the chunks in flight.
//
// The chunked histogram of 17 and 18 bits works the same way: one reduction
// per tuple (aggregated per warp) into the chunk's histogram in global
// memory, which stays in L2 for the chunks in flight; the scan that turns it
// into offsets is the existing per-chunk scan.  It reads every key once,
// where 2^15-bin shared-memory ranges read them 4 or 8 times and a cluster
// histogram pays for remote shared-memory atomics.
//
// Replaces, for radix bits above 11, the reference's HSSWWCv4 / SSWWCv2
// scatters (sql-ops/cudautils/radix_partition.cu:689-1477); the per-(chunk,
// partition) tuple multisets are the same as every other scatter's.
#include <algorithm>

#include "common.cuh"
#include "kernels.h"

namespace fi {

namespace {

constexpr uint32_t kWideThreads = 256;
constexpr uint32_t kWideItems = 8;  // tuples per thread per tile
constexpr uint32_t kWideTile = kWideThreads * kWideItems;

// Chunk of input tuple i under the canonical chunking: chunk c spans
// [c * clen, (c + 1) * clen), the last chunk takes the rest (clen == 0
// leaves everything to the last chunk).
__device__ __forceinline__ uint32_t chunk_of(uint64_t i, uint64_t clen,
                                             uint32_t chunks) {
  if (clen == 0) return chunks - 1;
  const uint64_t c = i / clen;
  return c < chunks ? (uint32_t)c : chunks - 1;
}

// Next tile of the input for the whole CTA (a global counter; the value is
// broadcast through shared memory).  Tile ids stay below 2^32: a tile holds
// 2048 tuples and relations hold fewer than 2^43.
__device__ __forceinline__ uint32_t next_tile(uint32_t *counter,
                                              uint32_t *slot) {
  __syncthreads();  // every thread is done with the previous value
  if (threadIdx.x == 0) *slot = atomicAdd(counter, 1u);
  __syncthreads();
  return *slot;
}

// Claims a slot on counter `bin`: lanes of the warp with the same bin are
// grouped, the lowest adds the group size, each lane gets a distinct slot.
__device__ __forceinline__ uint32_t claim_slot(uint32_t *counters, uint64_t bin,
                                               bool active) {
  const uint32_t act = __ballot_sync(kFullMask, active);
  uint32_t slot = 0;
  if (active) {
    const uint32_t peers = __match_any_sync(act, bin);
    const uint32_t leader = __ffs(peers) - 1;
    uint32_t base = 0;
    if (lane_id() == leader) base = atomicAdd(&counters[bin], __popc(peers));
    base = __shfl_sync(act, base, leader);
    slot = base + __popc(peers & lanemask_lt());
  }
  return slot;
}

// Adds one to counter `bin` for every active lane, one reduction per group
// of lanes with the same bin.
__device__ __forceinline__ void count_bin(uint32_t *counters, uint64_t bin,
                                          bool active) {
  const uint32_t act = __ballot_sync(kFullMask, active);
  if (active) {
    const uint32_t peers = __match_any_sync(act, bin);
    if (lane_id() == __ffs(peers) - 1) atomicAdd(&counters[bin], __popc(peers));
  }
}

// rel[c * F + p] = cursors[c * F + p] - cursors[c * F]: each chunk's cursors
// relative to its first slot (below 2^32: a chunk and a contiguous relation
// hold fewer tuples).
__global__ void wide_cursor_init_kernel(const uint64_t *__restrict__ cursors,
                                        uint32_t *__restrict__ rel,
                                        uint64_t n, uint32_t radix_bits,
                                        uint32_t *tile_counter) {
  const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
  for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += stride) {
    const uint64_t first = (i >> radix_bits) << radix_bits;
    rel[i] = (uint32_t)(cursors[i] - cursors[first]);
  }
  if (blockIdx.x == 0 && threadIdx.x == 0) *tile_counter = 0;
}

template <typename K>
__global__ void __launch_bounds__(kWideThreads, 4)
    wide_scatter_kernel(const K *__restrict__ keys, const K *__restrict__ pays,
                        uint64_t len, uint64_t clen, uint32_t chunks,
                        uint32_t radix_bits, uint32_t ignore_bits,
                        const uint64_t *__restrict__ cursors,
                        uint32_t *__restrict__ rel_cursors,
                        Tuple<K> *__restrict__ out, uint64_t out_len,
                        uint32_t *tile_counter, int *status) {
  __shared__ uint32_t s_tile;
  const uint64_t mask = (((uint64_t)1 << radix_bits) - 1u) << ignore_bits;
  const uint64_t ntiles = (len + kWideTile - 1) / kWideTile;
  const uint32_t tid = threadIdx.x;
  for (;;) {
    const uint64_t t = next_tile(tile_counter, &s_tile);
    if (t >= ntiles) break;
    const uint64_t t0 = t * kWideTile;
    const uint32_t c0 = chunk_of(t0, clen, chunks);
    const uint64_t b1 = (c0 + 1 < chunks) ? (uint64_t)(c0 + 1) * clen : ~0ull;
    K k[kWideItems], v[kWideItems];
#pragma unroll
    for (uint32_t u = 0; u < kWideItems; ++u) {
      const uint64_t i = t0 + u * kWideThreads + tid;
      if (i < len) {
        k[u] = load_cs(keys + i);
        v[u] = load_cs(pays + i);
      }
    }
    uint64_t dst[kWideItems];
#pragma unroll
    for (uint32_t u = 0; u < kWideItems; ++u) {
      const uint64_t i = t0 + u * kWideThreads + tid;
      const bool act = i < len;
      const uint32_t c = (i < b1) ? c0 : chunk_of(i, clen, chunks);
      const uint64_t first = (uint64_t)c << radix_bits;
      const uint32_t p = act ? key_to_partition(k[u], mask, ignore_bits) : 0u;
      const uint32_t slot = claim_slot(rel_cursors, first | p, act);
      dst[u] = act ? cursors[first] + slot : ~0ull;
    }
#pragma unroll
    for (uint32_t u = 0; u < kWideItems; ++u) {
      if (t0 + u * kWideThreads + tid >= len) continue;
      if (dst[u] < out_len)
        store_tuple(out + dst[u], Tuple<K>{k[u], v[u]});
      else
        record_error(status, kDevErrCapacity);
    }
  }
}

template <typename K>
__global__ void __launch_bounds__(kWideThreads)
    wide_histogram_kernel(const K *__restrict__ keys, uint64_t len,
                          uint64_t clen, uint32_t chunks, uint32_t radix_bits,
                          uint32_t ignore_bits, uint32_t *__restrict__ hist,
                          uint32_t *tile_counter) {
  __shared__ uint32_t s_tile;
  const uint64_t mask = (((uint64_t)1 << radix_bits) - 1u) << ignore_bits;
  const uint64_t ntiles = (len + kWideTile - 1) / kWideTile;
  const uint32_t tid = threadIdx.x;
  for (;;) {
    const uint64_t t = next_tile(tile_counter, &s_tile);
    if (t >= ntiles) break;
    const uint64_t t0 = t * kWideTile;
    const uint32_t c0 = chunk_of(t0, clen, chunks);
    const uint64_t b1 = (c0 + 1 < chunks) ? (uint64_t)(c0 + 1) * clen : ~0ull;
    K k[kWideItems];
#pragma unroll
    for (uint32_t u = 0; u < kWideItems; ++u) {
      const uint64_t i = t0 + u * kWideThreads + tid;
      if (i < len) k[u] = load_cs(keys + i);
    }
#pragma unroll
    for (uint32_t u = 0; u < kWideItems; ++u) {
      const uint64_t i = t0 + u * kWideThreads + tid;
      const bool act = i < len;
      const uint32_t c = (i < b1) ? c0 : chunk_of(i, clen, chunks);
      const uint32_t p = act ? key_to_partition(k[u], mask, ignore_bits) : 0u;
      count_bin(hist, ((uint64_t)c << radix_bits) | p, act);
    }
  }
}

int resident_grid(const void *fn, uint32_t threads, uint32_t sm_count) {
  int per_sm = 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, fn, (int)threads, 0) !=
          cudaSuccess ||
      per_sm < 1)
    per_sm = 1;
  return per_sm * (int)sm_count;
}

}  // namespace

template <typename K>
cudaError_t launch_partition_wide(const K *keys, const K *pays, uint64_t len,
                                  uint32_t chunks, uint32_t radix_bits,
                                  uint32_t ignore_bits, const uint64_t *cursors,
                                  void *out, uint64_t out_len,
                                  uint32_t *rel_cursors,
                                  uint32_t *tile_counter, int *status,
                                  uint32_t sm_count, cudaStream_t stream) {
  constexpr uint64_t kAlignMask = ~((uint64_t)(kAlignBytes / sizeof(K)) - 1ull);
  const uint64_t clen = ((len + chunks - 1) / chunks) & kAlignMask;
  const uint64_t n = (uint64_t)chunks << radix_bits;
  const uint32_t init_grid = (uint32_t)std::min<uint64_t>((n + 255) / 256, 4u * sm_count);
  wide_cursor_init_kernel<<<init_grid, 256, 0, stream>>>(cursors, rel_cursors, n,
                                                         radix_bits, tile_counter);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return e;
  const int grid = resident_grid((const void *)wide_scatter_kernel<K>, kWideThreads,
                                 sm_count);
  wide_scatter_kernel<K><<<grid, kWideThreads, 0, stream>>>(
      keys, pays, len, clen, chunks, radix_bits, ignore_bits, cursors, rel_cursors,
      reinterpret_cast<Tuple<K> *>(out), out_len, tile_counter, status);
  return cudaGetLastError();
}

template <typename K>
cudaError_t launch_wide_chunk_histogram(const K *keys, uint64_t len, uint64_t clen,
                                        uint32_t chunks, uint32_t radix_bits,
                                        uint32_t ignore_bits, uint32_t *hist,
                                        uint32_t *tile_counter,
                                        uint32_t sm_count, cudaStream_t stream) {
  cudaError_t e = cudaMemsetAsync(tile_counter, 0, sizeof(uint32_t), stream);
  if (e != cudaSuccess) return e;
  const int grid = resident_grid((const void *)wide_histogram_kernel<K>, kWideThreads,
                                 sm_count);
  wide_histogram_kernel<K><<<grid, kWideThreads, 0, stream>>>(
      keys, len, clen, chunks, radix_bits, ignore_bits, hist, tile_counter);
  return cudaGetLastError();
}

#define FI_INSTANTIATE_WIDE(K)                                                   \
  template cudaError_t launch_partition_wide<K>(                                 \
      const K *, const K *, uint64_t, uint32_t, uint32_t, uint32_t,              \
      const uint64_t *, void *, uint64_t, uint32_t *, uint32_t *,                \
      int *, uint32_t, cudaStream_t);                                            \
  template cudaError_t launch_wide_chunk_histogram<K>(                           \
      const K *, uint64_t, uint64_t, uint32_t, uint32_t, uint32_t, uint32_t *,   \
      uint32_t *, uint32_t, cudaStream_t);

FI_INSTANTIATE_WIDE(int32_t)
FI_INSTANTIATE_WIDE(int64_t)

}  // namespace fi
