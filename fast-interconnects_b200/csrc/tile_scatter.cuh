// Shared-memory tile write-combining scatter (device code shared by the
// partition kernels and the join engine's second pass).
//
// A CTA walks its input in tiles of kThreads * kItems tuples.  The next
// tile's tuples are loaded into registers (evict-first) while the current
// tile is processed.  Each tile is counting-sorted by partition in shared
// memory (shared-memory atomic ranks + a block scan of the tile histogram)
// and written out in partition runs, so consecutive threads store
// consecutive tuples of a run.  Partially written 128-byte lines are
// completed by later tiles while they stay in L2.
#pragma once

#include "common.cuh"

namespace fi {

// Tile shapes.  Wide: 512 threads, one CTA per SM (the register double
// buffer takes ~100 registers per thread).  Dual: 256 threads, two CTAs per
// SM, so one CTA's barriers overlap the other's loads and stores.
template <typename K, uint32_t kThreads_, uint32_t kMinBlocks_>
struct TileShape {
  static constexpr uint32_t kThreads = kThreads_;
  static constexpr uint32_t kMinBlocks = kMinBlocks_;
  static constexpr uint32_t kItems = sizeof(K) == 8 ? 8 : 16;
  static constexpr uint32_t kTile = kThreads * kItems;
};
template <typename K>
using TileWide = TileShape<K, 512, 1>;
template <typename K>
using TileDual = TileShape<K, 256, 2>;

template <typename K, typename S>
size_t tile_scatter_smem(uint32_t F) {
  return (size_t)S::kTile * sizeof(Tuple<K>) +
         (size_t)(2 * F + 1 + 33) * sizeof(uint32_t);
}

// Source of tuples for the tile scatter: two columns.
template <typename K>
struct ColumnSource {
  const K *__restrict__ keys;
  const K *__restrict__ pays;
  __device__ __forceinline__ void load(uint64_t i, K &k, K &v) {
    k = load_cs(keys + i);
    v = load_cs(pays + i);
  }
};

// Source of tuples for the tile scatter: an array of tuples.
template <typename K>
struct TupleSource {
  const Tuple<K> *__restrict__ tuples;
  __device__ __forceinline__ void load(uint64_t i, K &k, K &v) {
    Tuple<K> t = load_tuple_cs(tuples + i);
    k = t.key;
    v = t.value;
  }
};

// Source of tuples for the tile scatter: a logical sequence made of several
// regions of an array of tuples (one first-pass partition spread over the
// chunks of a Chunked relation).  Logical index i lies in region r with
// pre[r] <= i < pre[r+1] at physical slot begin[r] + (i - pre[r]).  `pre`
// and `begin` live in shared memory; every thread keeps its current region's
// bounds in registers, which only move forward because each thread's indices
// increase.
template <typename K>
struct RegionSource {
  const Tuple<K> *__restrict__ tuples;
  const uint64_t *pre;    // [regions + 1]
  const uint64_t *begin;  // [regions]
  uint32_t regions;
  uint32_t r = 0;
  uint64_t lo = 0, hi = 0, base = 0;
  __device__ __forceinline__ RegionSource(const Tuple<K> *t, const uint64_t *p,
                                          const uint64_t *b, uint32_t n)
      : tuples(t), pre(p), begin(b), regions(n) {}
  __device__ __forceinline__ void load(uint64_t i, K &k, K &v) {
    if (i >= hi) {
      while (r + 1 < regions && pre[r + 1] <= i) ++r;
      lo = pre[r];
      hi = pre[r + 1];
      base = begin[r];
    }
    Tuple<K> t = load_tuple_cs(tuples + base + (i - lo));
    k = t.key;
    v = t.value;
  }
};

// Scatters src[begin, end) by partition into out, starting partition p at
// out[cur_base + cur[p]].  `cur` (F u32, relative to cur_base) and `toff`
// (F+1 u32, zero on entry and exit) live in shared memory.
template <typename K, typename S, typename Src>
__device__ __forceinline__ void tile_scatter_range(
    Src &src, uint64_t begin, uint64_t end, uint32_t F, uint64_t mask,
    uint32_t ignore_bits, uint32_t *cur, uint32_t *toff, uint32_t *scan_tmp,
    Tuple<K> *staged, Tuple<K> *__restrict__ out, uint64_t cur_base,
    uint64_t out_len, int *status) {
  constexpr uint32_t T = S::kThreads;
  constexpr uint32_t I = S::kItems;
  constexpr uint32_t kTile = S::kTile;
  const uint32_t tid = threadIdx.x;

  K ck[I], cv[I];
#pragma unroll
  for (uint32_t u = 0; u < I; ++u) {
    const uint64_t i = begin + (uint64_t)u * T + tid;
    if (i < end) src.load(i, ck[u], cv[u]);
  }

  for (uint64_t t0 = begin; t0 < end; t0 += kTile) {
    const uint32_t n_valid = (uint32_t)min((uint64_t)kTile, end - t0);
    const uint64_t t1 = t0 + kTile;
    K nk[I], nv[I];
#pragma unroll
    for (uint32_t u = 0; u < I; ++u) {
      const uint64_t i = t1 + (uint64_t)u * T + tid;
      if (i < end) src.load(i, nk[u], nv[u]);
    }

    // 1. rank every tuple inside its partition's run of the tile
    uint32_t pp[I], rk[I];
#pragma unroll
    for (uint32_t u = 0; u < I; ++u) {
      const bool act = (uint64_t)u * T + tid < n_valid;
      pp[u] = act ? key_to_partition(ck[u], mask, ignore_bits) : 0u;
      rk[u] = warp_aggregated_rank(toff, pp[u], act);
    }
    __syncthreads();
    // 2. run offsets inside the tile
    block_exclusive_scan_u32(toff, F, scan_tmp);
    if (tid == 0) toff[F] = n_valid;
    // 3. stage the tile sorted by partition
#pragma unroll
    for (uint32_t u = 0; u < I; ++u) {
      if ((uint64_t)u * T + tid < n_valid)
        staged[toff[pp[u]] + rk[u]] = Tuple<K>{ck[u], cv[u]};
    }
    __syncthreads();
    // 4. write the runs; tuple j of run p goes to cur[p] + (j - toff[p])
    for (uint32_t j = tid; j < n_valid; j += T) {
      const Tuple<K> t = staged[j];
      const uint32_t p = key_to_partition(t.key, mask, ignore_bits);
      const uint64_t dst = cur_base + cur[p] + (j - toff[p]);
      if (dst < out_len)
        store_tuple(out + dst, t);
      else
        record_error(status, kDevErrCapacity);
    }
    __syncthreads();
    // 5. advance the cursors (reads toff), then clear toff for the next tile
    for (uint32_t p = tid; p < F; p += T) cur[p] += toff[p + 1] - toff[p];
    __syncthreads();
    for (uint32_t p = tid; p <= F; p += T) toff[p] = 0;
    __syncthreads();
#pragma unroll
    for (uint32_t u = 0; u < I; ++u) {
      ck[u] = nk[u];
      cv[u] = nv[u];
    }
  }
}

}  // namespace fi
