// Histogram and prefix-sum kernels of the radix partitioner (sm_100a).
//
// Replaces gpu_chunked_prefix_sum, gpu_contiguous_prefix_sum,
// gpu_contiguous_prefix_sum_and_copy_with_payload and
// gpu_contiguous_prefix_sum_and_transform of the reference
// (sql-ops/cudautils/radix_partition.cu:40-467) with the same outputs.
//
// Design (B200):
//  * Histogram: every chunk is shared by `splits` CTAs so that the grid fills
//    all 148 SMs even with few chunks.  Keys stream in with 16-byte
//    evict-first vector loads; counts go to a shared-memory histogram through
//    plain shared atomics (the match.any aggregation of common.cuh measured
//    slower on B200, even for Zipf-skewed keys).  Fanouts above 2^15 do not
//    fit one CTA's shared memory: the bins are split into ranges of 2^15
//    and every (chunk, split) is read by one CTA per range (histogram_kernel),
//    the CTAs adjacent in the grid so the repeated reads mostly come from L2;
//    at 2^18 bins a thread-block cluster of 8 CTAs holds the histogram in
//    distributed shared memory and every key is read once
//    (histogram_cluster_kernel).  A chunk owned by a single
//    CTA is scanned in place and its offsets written directly (one launch);
//    otherwise the CTAs add their counts into a global per-chunk histogram
//    and a second kernel scans it.
//  * Contiguous offsets: instead of the reference's cooperative launch with
//    three grid-wide barriers, a second kernel scans the (partition, chunk)
//    counts with a single-pass decoupled look-back over tiles of partitions
//    (Merrill & Garland, "Single-pass Parallel Prefix Scan with Decoupled
//    Look-back", 2016): tile ids are taken from an atomic counter so a tile
//    only waits on tiles that are already running, and every wait is bounded.
#include <cooperative_groups.h>

#include "common.cuh"
#include "kernels.h"
#include "tma_scatter.cuh"

namespace fi {

constexpr uint32_t kHistThreads = 512;
constexpr uint32_t kHistUnroll = 4;
constexpr uint32_t kScanThreads = 1024;  // 32 chunk groups x kScanTile partitions

template <typename K>
struct Vec16;
template <>
struct Vec16<int64_t> {
  using type = longlong2;
  static constexpr uint32_t n = 2;
  __device__ static int64_t get(const longlong2 &v, uint32_t i) {
    return i == 0 ? v.x : v.y;
  }
};
template <>
struct Vec16<int32_t> {
  using type = int4;
  static constexpr uint32_t n = 4;
  __device__ static int32_t get(const int4 &v, uint32_t i) {
    return i == 0 ? v.x : (i == 1 ? v.y : (i == 2 ? v.z : v.w));
  }
};

// Calls f(key, active) for keys[begin, end) in warp-uniform iterations, so
// that f may use warp intrinsics.  16-byte vector loads when the column is
// 16-byte aligned; scalar loads for the ragged head and tail.
template <typename K, typename Fn>
__device__ __forceinline__ void for_each_key(const K *__restrict__ keys,
                                             uint64_t begin, uint64_t end,
                                             Fn &&f) {
  using VT = Vec16<K>;
  using V = typename VT::type;
  constexpr uint32_t kVec = VT::n;
  const uint32_t tid = threadIdx.x, nt = blockDim.x;
  uint64_t vb = (begin + kVec - 1) / kVec, ve = end / kVec;
  const bool aligned = (reinterpret_cast<uintptr_t>(keys) % 16) == 0;
  if (!aligned || vb >= ve) {
    for (uint64_t base = begin; base < end; base += nt) {
      uint64_t i = base + tid;
      bool act = i < end;
      f(act ? load_cs(keys + i) : K(0), act);
    }
    return;
  }
  {  // head: fewer than kVec elements
    uint64_t i = begin + tid;
    bool act = i < vb * kVec;
    f(act ? load_cs(keys + i) : K(0), act);
  }
  const V *vk = reinterpret_cast<const V *>(keys);
  for (uint64_t base = vb; base < ve; base += (uint64_t)nt * kHistUnroll) {
    V v[kHistUnroll];
    bool act[kHistUnroll];
#pragma unroll
    for (uint32_t u = 0; u < kHistUnroll; ++u) {
      uint64_t idx = base + (uint64_t)u * nt + tid;
      act[u] = idx < ve;
      if (act[u]) v[u] = __ldcs(vk + idx);
    }
#pragma unroll
    for (uint32_t u = 0; u < kHistUnroll; ++u)
#pragma unroll
      for (uint32_t e = 0; e < kVec; ++e)
        f(act[u] ? VT::get(v[u], e) : K(0), act[u]);
  }
  {  // tail
    uint64_t i = ve * kVec + tid;
    bool act = i < end;
    f(act ? load_cs(keys + i) : K(0), act);
  }
}

// Sub-range [sb, se) of chunk c handled by split s (16-byte aligned starts).
template <typename K>
__device__ __forceinline__ void split_range(uint64_t len, uint64_t clen,
                                            uint32_t chunks, uint32_t c,
                                            uint32_t splits, uint32_t s,
                                            uint64_t &sb, uint64_t &se) {
  constexpr uint64_t kVec = 16 / sizeof(K);
  const uint64_t cb = clen * c;
  const uint64_t ce = (c + 1 == chunks) ? len : cb + clen;
  const uint64_t n = ce - cb;
  const uint64_t per = ((n + splits - 1) / splits + kVec - 1) / kVec * kVec;
  sb = min(ce, cb + per * s);
  se = min(ce, sb + per);
}

// Shared-memory counters of one histogram CTA; larger fanouts are split into
// ranges of this many bins, one CTA per (chunk, split, range).  The CTAs of
// one chunk are adjacent in the grid, so their repeated reads of the same
// keys hit in L2.
constexpr uint32_t kHistSmemBinsLog2 = 15;

// Histogram of one chunk split, restricted to the bins
// [range*nbins, (range+1)*nbins), nbins = min(F, 2^15).  direct_offsets !=
// nullptr: the CTA owns the whole chunk and all bins (splits == ranges == 1)
// and writes the chunk's final offsets (radix_partition.cu:83-95); otherwise
// it adds its counts to g_hist[c*F+p].  With dst_key/dst_pay the columns are
// copied as well.
template <typename K>
__global__ void __launch_bounds__(kHistThreads)
    histogram_kernel(const K *__restrict__ keys, const K *__restrict__ pays,
                     K *__restrict__ dst_key, K *__restrict__ dst_pay,
                     uint64_t len, uint64_t clen, uint32_t chunks,
                     uint32_t splits, uint32_t ranges, uint32_t radix_bits,
                     uint32_t ignore_bits, uint32_t pad,
                     uint64_t *__restrict__ direct_offsets,
                     uint32_t *__restrict__ g_hist) {
  extern __shared__ uint32_t smem[];
  const uint32_t F = 1u << radix_bits;
  const uint32_t nbins = F / ranges;
  const uint64_t mask = static_cast<uint64_t>(F - 1u) << ignore_bits;
  uint32_t *cnt = smem;
  uint32_t *scan_tmp = smem + nbins;
  const uint32_t r = blockIdx.x % ranges;
  const uint32_t s = (blockIdx.x / ranges) % splits;
  const uint32_t c = blockIdx.x / (ranges * splits);
  const uint32_t bin_lo = r * nbins;
  uint64_t sb, se;
  split_range<K>(len, clen, chunks, c, splits, s, sb, se);

  for (uint32_t i = threadIdx.x; i < nbins; i += blockDim.x) cnt[i] = 0;
  __syncthreads();

  for_each_key(keys, sb, se, [&](K key, bool act) {
    const uint32_t b = key_to_partition(key, mask, ignore_bits) - bin_lo;
    warp_aggregated_count(cnt, b, act && b < nbins);
  });

  if (dst_key != nullptr && r == 0) {
    for (uint64_t i = sb + threadIdx.x; i < se; i += blockDim.x) {
      dst_key[i] = keys[i];
      dst_pay[i] = pays[i];
    }
  }
  __syncthreads();

  if (direct_offsets != nullptr) {
    block_exclusive_scan_u32(cnt, F, scan_tmp);
    const uint64_t chunk_base = (clen + (uint64_t)pad * F) * c;
    for (uint32_t p = threadIdx.x; p < F; p += blockDim.x)
      direct_offsets[(uint64_t)c * F + p] =
          (uint64_t)cnt[p] + chunk_base + (uint64_t)(p + 1) * pad;
  } else {
    uint32_t *gh = g_hist + (uint64_t)c * F + bin_lo;
    for (uint32_t p = threadIdx.x; p < nbins; p += blockDim.x)
      if (cnt[p] != 0) atomicAdd(&gh[p], cnt[p]);
  }
}

// Histogram of fanouts above 2^15 with a thread-block cluster: the
// cluster's R = F / 2^15 CTAs each hold 2^15 counters in shared memory, so
// together they hold the whole histogram in distributed shared memory.
// Every CTA reads its share of the (chunk, split) keys once and adds each
// key to the counter of the CTA that owns its bin, through the cluster's
// shared-memory window; then every CTA adds its own 2^15 counters to
// g_hist.  Each key is read once from HBM (the bin-range kernel above reads
// it R times).  Cluster barriers: after the counters are zeroed (before any
// remote add) and after the adds (before the flush and before any CTA may
// exit while its shared memory is still a target).
constexpr uint32_t kClusterThreads = 1024;

template <typename K>
__global__ void __launch_bounds__(kClusterThreads)
    histogram_cluster_kernel(const K *__restrict__ keys, uint64_t len,
                             uint64_t clen, uint32_t chunks, uint32_t splits,
                             uint32_t radix_bits, uint32_t ignore_bits,
                             uint32_t *__restrict__ g_hist) {
  namespace cg = cooperative_groups;
  cg::cluster_group cluster = cg::this_cluster();
  extern __shared__ uint32_t cnt[];  // [2^15]
  constexpr uint32_t kBins = 1u << kHistSmemBinsLog2;
  const uint32_t F = 1u << radix_bits;
  const uint32_t R = cluster.num_blocks(), q = cluster.block_rank();
  const uint64_t mask = static_cast<uint64_t>(F - 1u) << ignore_bits;
  const uint32_t cid = blockIdx.x / R;  // (chunk, split) of this cluster
  const uint32_t c = cid / splits, s = cid % splits;
  uint64_t sb, se;
  split_range<K>(len, clen, chunks, c, splits, s, sb, se);
  // this CTA's share of the cluster's keys (16-byte aligned starts)
  constexpr uint64_t kVec = 16 / sizeof(K);
  const uint64_t per = ((se - sb + R - 1) / R + kVec - 1) / kVec * kVec;
  const uint64_t qb = min(se, sb + per * q), qe = min(se, qb + per);
  for (uint32_t i = threadIdx.x; i < kBins; i += blockDim.x) cnt[i] = 0;
  cluster.sync();
  for_each_key(keys, qb, qe, [&](K key, bool act) {
    if (act) {
      const uint32_t b = key_to_partition(key, mask, ignore_bits);
      uint32_t *dst = cluster.map_shared_rank(cnt, b >> kHistSmemBinsLog2);
      atomicAdd(dst + (b & (kBins - 1u)), 1u);
    }
  });
  cluster.sync();
  uint32_t *gh = g_hist + (uint64_t)c * F + (uint64_t)q * kBins;
  for (uint32_t p = threadIdx.x; p < kBins; p += blockDim.x)
    if (cnt[p] != 0) atomicAdd(&gh[p], cnt[p]);
}

// Histogram of fanouts above 2^15 fed by TMA: one 1024-thread CTA per
// (chunk, split, bin range) holds the range's 2^15 counters (128 KB) and
// streams its split's keys through two 32 KB shared-memory stages with 1-D
// bulk copies (cp.async.bulk + mbarrier), so every SM keeps a tile in flight
// while it counts the previous one.  The range CTAs of one split are
// adjacent in the grid, so the rereads of each tile mostly come from L2.
// The bin-range kernel above reads the same keys with 512 threads and a few
// 16-byte loads in flight each and is latency-bound (2.0 ms for 2^16 bins,
// 7.8 ms for 2^18, over 512M keys).  Waits are bounded; a wait that gives up records
// kDevErrTimeout in *status (when given), drains the copies in flight and
// leaves the CTA's counts out.  Every range rereads the split's keys, so
// the cost grows with the ranges: 1.82 ms for two (2^16 bins), 3.61 ms for
// four (2^17) and 7.1-7.2 ms for eight (2^18) over 512M int64 keys, the
// same for uniform and Zipf-skewed keys.
template <typename K>
struct RangeTile {
  static constexpr uint32_t kThreads = 1024;
  static constexpr uint32_t kKeys = (32u << 10) / sizeof(K);  // one 32 KB stage
  static constexpr uint32_t kStages = 2;
};

template <typename K>
size_t range_tma_smem() {
  return 64 + RangeTile<K>::kStages * (size_t)(32u << 10) +
         ((size_t)sizeof(uint32_t) << kHistSmemBinsLog2);
}

template <typename K>
__global__ void __launch_bounds__(1024, 1)
    histogram_range_tma_kernel(const K *__restrict__ keys, uint64_t len,
                               uint64_t clen, uint32_t chunks, uint32_t splits,
                               uint32_t ranges, uint32_t radix_bits,
                               uint32_t ignore_bits, uint32_t *__restrict__ g_hist,
                               int *status) {
  using T = RangeTile<K>;
  constexpr uint32_t kBins = 1u << kHistSmemBinsLog2;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  uint64_t *bars = reinterpret_cast<uint64_t *>(smem_raw);
  K *stages = reinterpret_cast<K *>(smem_raw + 64);
  uint32_t *cnt = reinterpret_cast<uint32_t *>(smem_raw + 64 + T::kStages * (32u << 10));
  const uint32_t F = 1u << radix_bits;
  const uint64_t mask = static_cast<uint64_t>(F - 1u) << ignore_bits;
  const uint32_t r = blockIdx.x % ranges;
  const uint32_t sp = (blockIdx.x / ranges) % splits;
  const uint32_t c = blockIdx.x / (ranges * splits);
  const uint32_t bin_lo = r * kBins;
  uint64_t sb, se;
  split_range<K>(len, clen, chunks, c, splits, sp, sb, se);
  const uint32_t tid = threadIdx.x;
  for (uint32_t i = tid; i < kBins; i += blockDim.x) cnt[i] = 0;
  if (tid == 0) {
    for (uint32_t st = 0; st < T::kStages; ++st) mbar_init(&bars[st], 1);
    mbar_fence_init();
  }
  __syncthreads();
  // [sb, se) starts 16-byte aligned; each tile's 16-byte multiple comes by
  // TMA, the last tile's ragged end (under 16 bytes) by plain loads
  const uint64_t n_all = se > sb ? se - sb : 0;
  const uint64_t ntiles = (n_all + T::kKeys - 1) / T::kKeys;
  auto issue = [&](uint64_t t) {
    const uint64_t t0 = sb + t * T::kKeys;
    const uint32_t n = (uint32_t)min((uint64_t)T::kKeys, se - t0);
    const uint32_t bytes = (n * (uint32_t)sizeof(K)) & ~15u;
    uint64_t *bar = &bars[t % T::kStages];
    mbar_arrive_expect_tx(bar, bytes);
    if (bytes) bulk_g2s(stages + (t % T::kStages) * T::kKeys, keys + t0, bytes, bar);
  };
  if (tid == 0 && ntiles > 0) issue(0);
  bool counted = true;
  for (uint64_t t = 0; t < ntiles; ++t) {
    if (tid == 0 && t + 1 < ntiles) {
      fence_proxy_async_smem();  // every thread left that stage before the last barrier
      issue(t + 1);
    }
    const bool ok = mbar_wait(&bars[t % T::kStages], (uint32_t)((t / T::kStages) & 1u));
    if (__syncthreads_or(!ok)) {
      if (tid == 0) {
        record_error(status, kDevErrTimeout);
        tma_drain<T::kStages>(bars, t, ntiles);
      }
      __syncthreads();
      counted = false;
      break;
    }
    const uint64_t t0 = sb + t * T::kKeys;
    const uint32_t n = (uint32_t)min((uint64_t)T::kKeys, se - t0);
    const uint32_t n_tma = ((n * (uint32_t)sizeof(K)) & ~15u) / (uint32_t)sizeof(K);
    const K *stage = stages + (t % T::kStages) * T::kKeys;
    for (uint32_t i = tid; i < n; i += T::kThreads) {
      const K k = i < n_tma ? stage[i] : load_cs(keys + t0 + i);
      const uint32_t b = key_to_partition(k, mask, ignore_bits) - bin_lo;
      if (b < kBins) atomicAdd(&cnt[b], 1u);
    }
    __syncthreads();  // the stage is free for the copy of tile t + 2
  }
  if (!counted) return;
  uint32_t *gh = g_hist + (uint64_t)c * F + bin_lo;
  for (uint32_t p = tid; p < kBins; p += blockDim.x)
    if (cnt[p] != 0) atomicAdd(&gh[p], cnt[p]);
}

// Per-chunk scan of g_hist into Chunked offsets (one CTA per chunk), in
// tiles of kScanTileBins bins with a running carry.
constexpr uint32_t kScanTileBins = 8192;
__global__ void __launch_bounds__(1024)
    chunked_scan_kernel(const uint32_t *__restrict__ g_hist, uint32_t F,
                        uint64_t clen, uint32_t pad,
                        uint64_t *__restrict__ offsets) {
  extern __shared__ uint32_t smem[];
  const uint32_t nb = min(F, kScanTileBins);
  uint32_t *cnt = smem;
  uint32_t *scan_tmp = smem + nb;
  const uint32_t c = blockIdx.x;
  const uint64_t chunk_base = (clen + (uint64_t)pad * F) * c;
  uint64_t carry = 0;
  for (uint32_t t0 = 0; t0 < F; t0 += nb) {
    for (uint32_t p = threadIdx.x; p < nb; p += blockDim.x)
      cnt[p] = g_hist[(uint64_t)c * F + t0 + p];
    __syncthreads();
    const uint32_t total = block_exclusive_scan_u32(cnt, nb, scan_tmp);
    for (uint32_t p = threadIdx.x; p < nb; p += blockDim.x)
      offsets[(uint64_t)c * F + t0 + p] = carry + (uint64_t)cnt[p] + chunk_base +
                                          (uint64_t)(t0 + p + 1) * pad;
    carry += total;
    __syncthreads();
  }
}

// ---- decoupled look-back ---------------------------------------------------
// A tile's state word packs a 2-bit flag with a 62-bit value.
constexpr uint64_t kFlagAggregate = 1ull << 62;
constexpr uint64_t kFlagPrefix = 2ull << 62;
constexpr uint64_t kValueMask = (1ull << 62) - 1ull;

__device__ __forceinline__ void state_store(uint64_t *p, uint64_t v) {
  asm volatile("st.release.gpu.global.u64 [%0], %1;" ::"l"(p), "l"(v)
               : "memory");
}
__device__ __forceinline__ uint64_t state_load(const uint64_t *p) {
  uint64_t v;
  asm volatile("ld.acquire.gpu.global.u64 %0, [%1];"
               : "=l"(v)
               : "l"(p)
               : "memory");
  return v;
}

// Returns the exclusive prefix of tile t given its aggregate; thread 0 only.
__device__ uint64_t look_back(uint64_t *tile_state, uint32_t t,
                              uint64_t aggregate, int *status) {
  if (t == 0) {
    state_store(&tile_state[0], kFlagPrefix | aggregate);
    return 0;
  }
  state_store(&tile_state[t], kFlagAggregate | aggregate);
  uint64_t prefix = 0;
  int64_t j = (int64_t)t - 1;
  uint32_t polls = 0;
  while (j >= 0) {
    uint64_t s = state_load(&tile_state[j]);
    uint64_t flag = s & ~kValueMask;
    if (flag == 0) {
      if (++polls > kSpinLimit) {
        record_error(status, kDevErrTimeout);
        break;
      }
      spin_pause(polls);
      continue;
    }
    prefix += s & kValueMask;
    if (flag == kFlagPrefix) break;
    --j;
  }
  state_store(&tile_state[t], kFlagPrefix | (prefix + aggregate));
  return prefix;
}

// Contiguous offsets from per-chunk histograms g_hist[b*F+p]:
//   offsets[p]          = sum_{q<p} T[q] + (p+1)*pad,  T[q] = sum_b hist[b][q]
//   local_offsets[b][p] = offsets[p] + sum_{b'<b} hist[b'][p]
// (radix_partition.cu:160-198).  Tiles of kScanTile = 32 partitions chained
// by decoupled look-back, one 1024-thread CTA each: lane l of warp w sums
// partition l of the tile over w's contiguous group of chunks (coalesced
// across the lanes), the groups are scanned per partition in shared memory,
// and the same threads write the local offsets.  (With one partition per
// thread and tiles of 1024 partitions, 1024 partitions x 148 chunks took one
// CTA 39 us.)
__global__ void __launch_bounds__(kScanThreads)
    contiguous_scan_kernel(const uint32_t *__restrict__ g_hist, uint32_t grid,
                           uint32_t F, uint32_t pad, uint64_t base,
                           uint64_t *__restrict__ offsets,
                           uint64_t *__restrict__ local_offsets,
                           uint64_t *tile_state, uint32_t *tile_counter,
                           int *status) {
  static_assert(kScanTile == 32 && kScanThreads == 32 * kScanTile,
                "one warp per chunk group, one lane per partition");
  __shared__ uint32_t tile_s;
  __shared__ uint64_t prefix_s, tile_total_s;
  __shared__ uint64_t group[32][kScanTile + 1];  // [chunk group][partition]
  __shared__ uint64_t ptot[kScanTile];           // partition totals
  if (threadIdx.x == 0) tile_s = atomicAdd(tile_counter, 1u);
  __syncthreads();
  const uint32_t t = tile_s, w = threadIdx.x >> 5, l = lane_id();
  const uint32_t p = t * kScanTile + l;
  const bool act = p < F;
  const uint32_t per = (grid + 31) / 32;
  const uint32_t cb = min(grid, w * per), ce = min(grid, cb + per);
  uint64_t own = 0;
  if (act)
    for (uint32_t b = cb; b < ce; ++b) own += g_hist[(uint64_t)b * F + p];
  group[w][l] = own;
  __syncthreads();
  {  // warp w scans partition w of the tile over the 32 chunk groups (lanes)
    const uint64_t v = group[l][w];
    uint64_t x = v;
#pragma unroll
    for (uint32_t d = 1; d < 32; d <<= 1) {
      const uint64_t y = __shfl_up_sync(kFullMask, x, d);
      if (l >= d) x += y;
    }
    group[l][w] = x - v;  // exclusive over the chunk groups
    if (l == 31) ptot[w] = x;
  }
  __syncthreads();
  if (w == 0) {  // exclusive scan of the tile's partition totals
    const uint64_t v = ptot[l];
    uint64_t x = v;
#pragma unroll
    for (uint32_t d = 1; d < 32; d <<= 1) {
      const uint64_t y = __shfl_up_sync(kFullMask, x, d);
      if (l >= d) x += y;
    }
    ptot[l] = x - v;
    if (l == 31) tile_total_s = x;
  }
  __syncthreads();
  if (threadIdx.x == 0) prefix_s = look_back(tile_state, t, tile_total_s, status);
  __syncthreads();
  if (act) {
    const uint64_t start = base + prefix_s + ptot[l] + (uint64_t)(p + 1) * pad;
    if (w == 0) offsets[p] = start;
    uint64_t run = start + group[w][l];
    for (uint32_t b = cb; b < ce; ++b) {
      local_offsets[(uint64_t)b * F + p] = run;
      run += g_hist[(uint64_t)b * F + p];
    }
  }
}

// ---- prefix_sum_and_transform ---------------------------------------------
// Gathers partition `pid` of every source chunk (chunk order) into columns
// and histograms the gathered sequence per canonical chunk of `grid`
// (radix_partition.cu:323-410).  Chunk table in shared memory; each thread
// finds its source chunk by binary search over the chunk prefix sums.
template <typename K>
__global__ void __launch_bounds__(kHistThreads) transform_histogram_kernel(
    uint32_t pid, const Tuple<K> *__restrict__ src,
    const uint64_t *__restrict__ src_offsets, uint32_t src_chunks,
    uint32_t src_fanout, uint64_t src_padded_len, uint32_t src_pad,
    uint64_t dst_len, uint32_t grid, uint32_t splits, uint32_t ranges,
    uint32_t radix_bits, uint32_t ignore_bits, K *__restrict__ dst_key,
    K *__restrict__ dst_pay, uint32_t *__restrict__ g_hist, int *status) {
  extern __shared__ uint64_t smem64[];
  const uint32_t F = 1u << radix_bits;
  const uint32_t nbins = F / ranges;
  const uint64_t mask = static_cast<uint64_t>(F - 1u) << ignore_bits;
  uint64_t *ch_begin = smem64;                 // [src_chunks]
  uint64_t *ch_pre = smem64 + src_chunks;      // [src_chunks + 1]
  uint64_t *tmp64 = ch_pre + src_chunks + 1;   // [33]
  uint32_t *cnt = reinterpret_cast<uint32_t *>(tmp64 + 33);  // [nbins]

  // chunk table: begin and length of partition pid in every source chunk
  uint64_t local_len = 0;
  for (uint32_t c = threadIdx.x; c < src_chunks; c += blockDim.x) {
    uint64_t b = src_offsets[(uint64_t)c * src_fanout + pid];
    uint64_t e = (c + 1 == src_chunks && pid + 1 == src_fanout)
                     ? src_padded_len
                     : src_offsets[(uint64_t)c * src_fanout + pid + 1] - src_pad;
    ch_begin[c] = b;
    ch_pre[c] = e - b;  // length, scanned below
  }
  for (uint32_t i = threadIdx.x; i < nbins; i += blockDim.x) cnt[i] = 0;
  __syncthreads();
  if (threadIdx.x == 0) {
    uint64_t run = 0;
    for (uint32_t c = 0; c < src_chunks; ++c) {
      uint64_t l = ch_pre[c];
      ch_pre[c] = run;
      run += l;
    }
    ch_pre[src_chunks] = run;
  }
  __syncthreads();
  (void)local_len;
  uint64_t n = ch_pre[src_chunks];
  if (n > dst_len) {
    if (blockIdx.x == 0 && threadIdx.x == 0) record_error(status, kDevErrCapacity);
    n = dst_len;
  }
  constexpr uint64_t kAlignMask = ~((uint64_t)(kAlignBytes / sizeof(K)) - 1ull);
  const uint64_t clen = ((n + grid - 1) / grid) & kAlignMask;
  const uint32_t r = blockIdx.x % ranges;
  const uint32_t s = (blockIdx.x / ranges) % splits;
  const uint32_t b = blockIdx.x / (ranges * splits);
  const uint32_t bin_lo = r * nbins;
  uint64_t sb, se;
  split_range<K>(n, clen, grid, b, splits, s, sb, se);

  for (uint64_t base = sb; base < se; base += blockDim.x) {
    const uint64_t i = base + threadIdx.x;
    const bool act = i < se;
    K key = 0;
    if (act) {
      // last chunk c with ch_pre[c] <= i
      uint32_t lo = 0, hi = src_chunks;
      while (hi - lo > 1) {
        uint32_t mid = (lo + hi) >> 1;
        if (ch_pre[mid] <= i) lo = mid; else hi = mid;
      }
      Tuple<K> t = load_tuple_cs(src + ch_begin[lo] + (i - ch_pre[lo]));
      if (r == 0) {
        dst_key[i] = t.key;
        dst_pay[i] = t.value;
      }
      key = t.key;
    }
    const uint32_t bin = key_to_partition(key, mask, ignore_bits) - bin_lo;
    warp_aggregated_count(cnt, bin, act && bin < nbins);
  }
  __syncthreads();
  uint32_t *gh = g_hist + (uint64_t)b * F + bin_lo;
  for (uint32_t p = threadIdx.x; p < nbins; p += blockDim.x)
    if (cnt[p] != 0) atomicAdd(&gh[p], cnt[p]);
}

// ---- host launchers ---------------------------------------------------------
uint32_t hist_splits(uint32_t chunks, uint32_t sm_count) {
  // about two CTAs of kHistThreads per SM in total
  uint32_t want = 2u * sm_count;
  uint32_t s = (want + chunks - 1) / chunks;
  return s < 1 ? 1 : s;
}

// Number of 2^15-bin ranges the histogram of a fanout is split into.
static uint32_t hist_ranges(uint32_t radix_bits) {
  return radix_bits > kHistSmemBinsLog2 ? 1u << (radix_bits - kHistSmemBinsLog2)
                                        : 1u;
}

// Shared memory of one histogram CTA: its bins plus the scan's warp sums.
static size_t hist_smem(uint32_t radix_bits) {
  return (size_t)(((1u << radix_bits) / hist_ranges(radix_bits)) + 33) *
         sizeof(uint32_t);
}

static size_t scan_smem(uint32_t F) {
  return (size_t)((F < kScanTileBins ? F : kScanTileBins) + 33) *
         sizeof(uint32_t);
}

template <typename K>
static cudaError_t set_smem(const void *fn, size_t bytes) {
  return cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize,
                              (int)bytes);
}

// Histogram of a fanout above 2^15 into g_hist (zeroed by the caller): the
// TMA-fed bin-range kernel for a 16-byte aligned key column without a
// column copy; else, at 2^18 bins, the cluster kernel when the GPU can
// schedule its clusters; else the bin-range kernel.
template <typename K>
static cudaError_t launch_wide_histogram(const K *keys, const K *pays,
                                         K *dst_key, K *dst_pay, uint64_t len,
                                         uint64_t clen, uint32_t chunks,
                                         uint32_t splits, uint32_t radix_bits,
                                         uint32_t ignore_bits, uint32_t pad,
                                         uint32_t *g_hist, int *status,
                                         cudaStream_t stream) {
  const uint32_t ranges = hist_ranges(radix_bits);
  const size_t tsm = range_tma_smem<K>();
  // measured on B200, 512M int64 keys over 148 chunks: 1.82 ms at 2^16
  // bins, 3.61 ms at 2^17, 7.19 ms at 2^18 for uniform keys and 7.11 ms
  // for Zipf(1.5) keys (every range pass rereads the keys at ~4.8 TB/s);
  // the cluster kernel below takes 7.03 ms at 2^18 for uniform keys but
  // 9.5 ms for Zipf(1.0) and 19.0 ms for Zipf(1.5), whose hot bin
  // serialises the remote atomics
  if (dst_key == nullptr && reinterpret_cast<uintptr_t>(keys) % 16 == 0 &&
      tsm <= (size_t)device_max_smem_optin()) {
    cudaError_t e = set_smem<K>((const void *)histogram_range_tma_kernel<K>, tsm);
    if (e != cudaSuccess) return e;
    histogram_range_tma_kernel<K><<<chunks * splits * ranges, RangeTile<K>::kThreads,
                                    tsm, stream>>>(keys, len, clen, chunks, splits,
                                                   ranges, radix_bits, ignore_bits,
                                                   g_hist, status);
    return cudaGetLastError();
  }
  // measured on B200, 512M keys over 148 chunks: at 2^16 bins the two-range
  // kernel takes 2.0 ms and the cluster 3.0 ms (its remote shared-memory
  // atomics cost more than the second, mostly L2-served, key read); at 2^18
  // bins eight reads per key make the ranges slower (7.8 ms vs 7.0 ms).  One
  // global reduction per key into the chunk's histogram, CTAs taking tiles
  // in input order so that one or two chunks' histograms (1 MB each) take
  // the reductions from L2, measured slower still: 8.1 ms at 2^17 and 8.2
  // ms at 2^18 bins for uniform keys, 10.3-11.7 ms for Zipf 1.0-1.5 keys
  // (the hot bin's reductions serialise in one L2 slice)
  if (dst_key == nullptr && ranges == 8) {
    const size_t csm = (size_t)sizeof(uint32_t) << kHistSmemBinsLog2;
    cudaError_t e = cudaFuncSetAttribute(
        (const void *)histogram_cluster_kernel<K>,
        cudaFuncAttributeMaxDynamicSharedMemorySize, (int)csm);
    if (e == cudaSuccess) {
      cudaLaunchConfig_t cfg = {};
      cfg.gridDim = dim3(chunks * splits * ranges);
      cfg.blockDim = dim3(kClusterThreads);
      cfg.dynamicSmemBytes = csm;
      cfg.stream = stream;
      cudaLaunchAttribute attr[1];
      attr[0].id = cudaLaunchAttributeClusterDimension;
      attr[0].val.clusterDim.x = ranges;
      attr[0].val.clusterDim.y = 1;
      attr[0].val.clusterDim.z = 1;
      cfg.attrs = attr;
      cfg.numAttrs = 1;
      int clusters = 0;
      e = cudaOccupancyMaxActiveClusters(&clusters,
                                         (const void *)histogram_cluster_kernel<K>,
                                         &cfg);
      if (e == cudaSuccess && clusters > 0)
        return cudaLaunchKernelEx(&cfg, histogram_cluster_kernel<K>, keys, len,
                                  clen, chunks, splits, radix_bits, ignore_bits,
                                  g_hist);
    }
    cudaGetLastError();  // fall back to the bin ranges
  }
  const size_t sm = hist_smem(radix_bits);
  cudaError_t e = set_smem<K>((const void *)histogram_kernel<K>, sm);
  if (e != cudaSuccess) return e;
  histogram_kernel<K><<<chunks * splits * ranges, kHistThreads, sm, stream>>>(
      keys, pays, dst_key, dst_pay, len, clen, chunks, splits, ranges,
      radix_bits, ignore_bits, pad, nullptr, g_hist);
  return cudaGetLastError();
}

template <typename K>
cudaError_t launch_chunked_prefix_sum(const K *keys, uint64_t len,
                                      uint32_t chunks, uint32_t radix_bits,
                                      uint32_t ignore_bits, uint32_t pad,
                                      uint64_t *offsets, HistScratch s,
                                      uint32_t sm_count, cudaStream_t stream) {
  const uint32_t F = 1u << radix_bits;
  constexpr uint64_t kAlignMask = ~((uint64_t)(kAlignBytes / sizeof(K)) - 1ull);
  const uint64_t clen = ((len + chunks - 1) / chunks) & kAlignMask;
  const uint32_t splits = hist_splits(chunks, sm_count);
  const uint32_t ranges = hist_ranges(radix_bits);
  const size_t sm = hist_smem(radix_bits);
  cudaError_t e = set_smem<K>((const void *)histogram_kernel<K>, sm);
  if (e != cudaSuccess) return e;
  if (splits == 1 && ranges == 1) {
    histogram_kernel<K><<<chunks, kHistThreads, sm, stream>>>(
        keys, nullptr, nullptr, nullptr, len, clen, chunks, 1, 1, radix_bits,
        ignore_bits, pad, offsets, nullptr);
    return cudaGetLastError();
  }
  e = cudaMemsetAsync(s.hist, 0, (size_t)chunks * F * sizeof(uint32_t), stream);
  if (e != cudaSuccess) return e;
  if (ranges > 1) {
    e = launch_wide_histogram<K>(keys, nullptr, nullptr, nullptr, len, clen,
                                 chunks, splits, radix_bits, ignore_bits, pad,
                                 s.hist, s.status, stream);
  } else {
    histogram_kernel<K><<<chunks * splits, kHistThreads, sm, stream>>>(
        keys, nullptr, nullptr, nullptr, len, clen, chunks, splits, 1,
        radix_bits, ignore_bits, pad, nullptr, s.hist);
    e = cudaGetLastError();
  }
  if (e != cudaSuccess) return e;
  const size_t ssm = scan_smem(F);
  e = set_smem<K>((const void *)chunked_scan_kernel, ssm);
  if (e != cudaSuccess) return e;
  chunked_scan_kernel<<<chunks, 1024, ssm, stream>>>(s.hist, F, clen, pad,
                                                     offsets);
  return cudaGetLastError();
}

static cudaError_t launch_contiguous_scan(uint32_t F, uint32_t grid,
                                          uint32_t pad, uint64_t base,
                                          uint64_t *offsets,
                                          uint64_t *local_offsets,
                                          HistScratch s, cudaStream_t stream) {
  const uint32_t tiles = (F + kScanTile - 1) / kScanTile;
  cudaError_t e =
      cudaMemsetAsync(s.tile_state, 0, (size_t)tiles * sizeof(uint64_t), stream);
  if (e != cudaSuccess) return e;
  e = cudaMemsetAsync(s.tile_counter, 0, sizeof(uint32_t), stream);
  if (e != cudaSuccess) return e;
  contiguous_scan_kernel<<<tiles, kScanThreads, 0, stream>>>(
      s.hist, grid, F, pad, base, offsets, local_offsets, s.tile_state,
      s.tile_counter, s.status);
  return cudaGetLastError();
}

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
                                         cudaStream_t stream) {
  const uint32_t F = 1u << radix_bits;
  constexpr uint64_t kAlignMask = ~((uint64_t)(kAlignBytes / sizeof(K)) - 1ull);
  const uint64_t clen = ((len + grid - 1) / grid) & kAlignMask;
  const uint32_t splits = hist_splits(grid, sm_count);
  const uint32_t ranges = hist_ranges(radix_bits);
  const size_t sm = hist_smem(radix_bits);
  cudaError_t e = set_smem<K>((const void *)histogram_kernel<K>, sm);
  if (e != cudaSuccess) return e;
  e = cudaMemsetAsync(s.hist, 0, (size_t)grid * F * sizeof(uint32_t), stream);
  if (e != cudaSuccess) return e;
  if (ranges > 1) {
    e = launch_wide_histogram<K>(keys, pays, dst_key, dst_pay, len, clen, grid,
                                 splits, radix_bits, ignore_bits, pad, s.hist,
                                 s.status, stream);
    if (e != cudaSuccess) return e;
  } else {
    histogram_kernel<K><<<grid * splits, kHistThreads, sm, stream>>>(
        keys, pays, dst_key, dst_pay, len, clen, grid, splits, 1, radix_bits,
        ignore_bits, pad, nullptr, s.hist);
  }
  e = cudaGetLastError();
  if (e != cudaSuccess) return e;
  return launch_contiguous_scan(F, grid, pad, base, offsets, local_offsets, s,
                                stream);
}

template <typename K>
cudaError_t launch_prefix_sum_and_transform(
    uint32_t partition_id, const void *src_relation, const uint64_t *src_offsets,
    uint32_t src_chunks, uint32_t src_radix_bits, uint64_t src_padded_len,
    uint32_t src_pad, uint64_t dst_len, uint32_t grid, uint32_t radix_bits,
    uint32_t ignore_bits, uint32_t pad, K *dst_key, K *dst_pay,
    uint64_t *offsets, uint64_t *local_offsets, HistScratch s,
    uint32_t sm_count, cudaStream_t stream) {
  const uint32_t F = 1u << radix_bits;
  const uint32_t splits = hist_splits(grid, sm_count);
  const uint32_t ranges = hist_ranges(radix_bits);
  const size_t sm = (size_t)(2 * src_chunks + 1 + 33) * sizeof(uint64_t) +
                    (size_t)(F / ranges) * sizeof(uint32_t);
  cudaError_t e =
      set_smem<K>((const void *)transform_histogram_kernel<K>, sm);
  if (e != cudaSuccess) return e;
  e = cudaMemsetAsync(s.hist, 0, (size_t)grid * F * sizeof(uint32_t), stream);
  if (e != cudaSuccess) return e;
  transform_histogram_kernel<K>
      <<<grid * splits * ranges, kHistThreads, sm, stream>>>(
          partition_id, reinterpret_cast<const Tuple<K> *>(src_relation),
          src_offsets, src_chunks, 1u << src_radix_bits, src_padded_len,
          src_pad, dst_len, grid, splits, ranges, radix_bits, ignore_bits,
          dst_key, dst_pay, s.hist, s.status);
  e = cudaGetLastError();
  if (e != cudaSuccess) return e;
  return launch_contiguous_scan(F, grid, pad, 0, offsets, local_offsets, s,
                                stream);
}

#define FI_INSTANTIATE_PREFIX(K)                                               \
  template cudaError_t launch_chunked_prefix_sum<K>(                           \
      const K *, uint64_t, uint32_t, uint32_t, uint32_t, uint32_t, uint64_t *, \
      HistScratch, uint32_t, cudaStream_t);                                    \
  template cudaError_t launch_contiguous_prefix_sum<K>(                        \
      const K *, const K *, uint64_t, uint32_t, uint32_t, uint32_t, uint32_t,  \
      K *, K *, uint64_t *, uint64_t *, uint64_t, HistScratch, uint32_t,       \
      cudaStream_t);                                                           \
  template cudaError_t launch_prefix_sum_and_transform<K>(                     \
      uint32_t, const void *, const uint64_t *, uint32_t, uint32_t, uint64_t,  \
      uint32_t, uint64_t, uint32_t, uint32_t, uint32_t, uint32_t, K *, K *,    \
      uint64_t *, uint64_t *, HistScratch, uint32_t, cudaStream_t);

FI_INSTANTIATE_PREFIX(int32_t)
FI_INSTANTIATE_PREFIX(int64_t)

}  // namespace fi
