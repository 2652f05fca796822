// The radix-join execution method on one B200
// (radix-join/src/execution_methods/gpu_radix_join.rs:90-565).
//
// The reference runs pass 1 for R and S and then loops over the 2^b1
// first-pass partitions on two streams, issuing six launches per partition
// (two prefix_sum_and_transform gathers, two second-pass partitions, task
// assignment, join), i.e. about 3000 launches at 9+9 bits, each with a grid of
// half the GPU.  This engine instead runs every step over all partitions at
// once, so the whole join is about a dozen launches that each fill the GPU:
//
//   1. Chunked histograms + offsets of R and S on the first-pass bits.
//   2. Tile scatter of R and S into chunked AoS relations (pass 1).
//   3. Plan: per first-pass partition p1, its length (summed over chunks),
//      its start in the pass-2 output and its split into "pieces" of at most
//      piece_tuples(len) tuples.  Pieces are the unit of pass-2 work, so a
//      Zipf-hot partition is spread over many CTAs.
//   4. Piece histograms on the second-pass bits (reads the pass-1 output).
//   5. Cursors: per (p1, p2) the contiguous output offsets, per piece its
//      cursor inside each (p1, p2) sub-partition.
//   6. Tile scatter of every piece into the final layout, ordered by
//      (p1, p2) with no padding (this replaces the reference's AoS->SoA
//      transform copy plus the second-pass prefix sum and partition).
//   7. One shared-memory join over all 2^(b1+b2) partitions (join.cu), then
//      a reduction of the per-thread sums into {sum, count}.
// With a single pass (b2 absent) steps 3-6 are skipped and pass 1 uses the
// Contiguous layout, as the join requires.
#include <algorithm>
#include <cstring>
#include <thread>
#include <vector>

#include "../../include/fi_sqlops.h"
#include "api_internal.h"
#include "common.cuh"
#include "kernels.h"
#include "tile_scatter.cuh"
#include "tma_scatter.cuh"

namespace fi {

// Pass-2 piece length: about four pieces per SM, between 2^13 and 2^18
// tuples.  Measured on B200 (1024M x 1024M int64, 9+9 bits, per relation):
// 2^17 -> pass-2 histogram 3.01 ms, scatter 7.31 ms; 2^18 -> 2.93 and 7.02
// ms; 2^19 -> 3.08 and 6.91; 2^20 -> 3.05 and 6.85 (longer pieces amortise a
// scatter CTA's set-up, shorter ones give the histogram more CTAs).  Small
// relations need shorter pieces to fill the GPU: 16M int32 tuples at 6+6
// bits made only 64 pieces of 2^18 (pass-2 histogram 0.36 ms, scatter 0.22).
constexpr uint64_t kMaxPieceTuples = 1ull << 18;
constexpr uint64_t kMinPieceTuples = 1ull << 13;
inline uint64_t piece_tuples(uint64_t len, uint32_t sm_count) {
  const uint64_t want = len / (4ull * sm_count);
  uint64_t p = kMinPieceTuples;
  while (p < kMaxPieceTuples && 2 * p <= want) p *= 2;
  return p;
}
// First-pass chunks per SM and the pass-2 tile shape.  Measured on B200
// (1024M x 1024M int64, 9+9 bits): the wide shape (512 threads, 4096-tuple
// tiles, one CTA per SM) beats two 256-thread CTAs per SM with 2048-tuple
// tiles (pass-1 scatter 4.6 vs 3.4 TB/s), because longer partition runs per
// tile give better-coalesced stores.
constexpr uint32_t kChunksPerSm = 1;
template <typename K>
using Pass2Shape = TileWide<K>;
// Join launch when the plan leaves it open (join block 0).  Bucket
// chaining: the most CTAs per SM whose table still holds an average
// partition (join_auto_block): four of 256 threads for the 4K-tuple
// partitions of 1024M x 1024M int64 at 9+9 bits (join 7.48 ms, against 7.78
// ms with two CTAs of 512 and 9.75 ms with one of 1024), one of 1024 for the
// 16K-tuple int32 partitions of 16M x 16M at 10 bits (0.12 ms, against 2.0
// ms when the 256-thread tables are too small and every partition is joined
// in rounds).  Perfect hashing: two CTAs of 512, whose table must span the
// largest key of a partition: half the SM's shared memory holds ~14.5K
// int64 keys, the capacity of the reference's one-table-per-CTA sizing
// (radix-join/src/cuda_radix_join.rs:234-237).
constexpr uint32_t kJoinBlockPerfect = 512;

struct Pass2Plan {
  uint64_t *reg_pre;      // [F1][C1+1] prefix of the chunk regions of p1
  uint64_t *p1_base;      // [F1+1] start of p1 in the pass-2 output
  uint32_t *piece_first;  // [F1+1] first piece of p1
  uint32_t *hist;         // [max_pieces][F2]
  uint64_t *cursor;       // [max_pieces][F2]
  uint64_t *off2;         // [F1*F2 + 1]
  uint32_t piece_log2;    // tuples per piece = 2^piece_log2 (piece_tuples)
};

// Exclusive scan of a global u64 array by one CTA; a[n] gets the total.
__device__ void cta_scan_global_u64(uint64_t *a, uint32_t n, uint64_t *tmp) {
  uint64_t carry = 0;
  for (uint32_t base = 0; base < n; base += blockDim.x) {
    const uint32_t i = base + threadIdx.x;
    const uint64_t v = i < n ? a[i] : 0;
    uint64_t total;
    const uint64_t ex = block_exclusive_scan_u64(v, tmp, &total);
    if (i < n) a[i] = carry + ex;
    carry += total;
  }
  if (threadIdx.x == 0) a[n] = carry;
}

// Pass-2 plan, step 1: per first-pass partition p1 (32 per CTA, lane l of
// warp w taking p1 = 32 * blockIdx.x + l over w's contiguous group of
// chunks), the prefix of its chunk regions' lengths, its length and its
// piece count.  (One CTA walking 512 partitions x 148 chunks took 56 us.)
__global__ void __launch_bounds__(1024)
    pass2_regions_kernel(const uint64_t *__restrict__ off1, uint32_t C1,
                         uint32_t F1, uint64_t padded1, uint32_t pad,
                         Pass2Plan pl, uint64_t *piece_count_tmp) {
  __shared__ uint64_t group[32][33];  // [chunk group][partition of the CTA]
  const uint32_t w = threadIdx.x >> 5, l = lane_id();
  const uint32_t p1 = blockIdx.x * 32 + l;
  const bool act = p1 < F1;
  const uint64_t n_off = (uint64_t)C1 * F1;
  const uint32_t per = (C1 + 31) / 32;
  const uint32_t cb = min(C1, w * per), ce = min(C1, cb + per);
  auto region_len = [&](uint32_t c) {
    const uint64_t ofi = (uint64_t)c * F1 + p1;
    const uint64_t b = off1[ofi];
    const uint64_t e = (ofi + 1 < n_off) ? off1[ofi + 1] - pad : padded1;
    return e - b;
  };
  uint64_t own = 0;
  if (act)
    for (uint32_t c = cb; c < ce; ++c) own += region_len(c);
  group[w][l] = own;
  __syncthreads();
  {  // warp w: exclusive scan of partition w's 32 group sums
    const uint64_t v = group[l][w];
    uint64_t x = v;
#pragma unroll
    for (uint32_t d = 1; d < 32; d <<= 1) {
      const uint64_t y = __shfl_up_sync(kFullMask, x, d);
      if (l >= d) x += y;
    }
    group[l][w] = x - v;
  }
  __syncthreads();
  if (!act) return;
  uint64_t *rp = pl.reg_pre + (uint64_t)p1 * (C1 + 1);
  uint64_t run = group[w][l];
  for (uint32_t c = cb; c < ce; ++c) {
    rp[c] = run;
    run += region_len(c);
  }
  if (w == 31) {  // the last group ends at chunk C1 (or is empty)
    rp[C1] = run;
    pl.p1_base[p1] = run;
    piece_count_tmp[p1] = (run + (1ull << pl.piece_log2) - 1) >> pl.piece_log2;
  }
}

// Pass-2 plan, step 2 (one CTA): exclusive scans of the partition lengths
// (p1_base) and of the piece counts (piece_first).
__global__ void __launch_bounds__(1024)
    pass2_plan_kernel(uint32_t F1, Pass2Plan pl, uint64_t *piece_count_tmp) {
  __shared__ uint64_t tmp[33];
  cta_scan_global_u64(pl.p1_base, F1, tmp);
  __syncthreads();
  cta_scan_global_u64(piece_count_tmp, F1, tmp);
  __syncthreads();
  for (uint32_t p1 = threadIdx.x; p1 <= F1; p1 += blockDim.x)
    pl.piece_first[p1] = (uint32_t)piece_count_tmp[p1];
}

__device__ __forceinline__ uint32_t find_p1(const uint32_t *piece_first,
                                            uint32_t F1, uint32_t k) {
  uint32_t lo = 0, hi = F1;  // last p1 with piece_first[p1] <= k
  while (hi - lo > 1) {
    const uint32_t mid = (lo + hi) >> 1;
    if (piece_first[mid] <= k) lo = mid; else hi = mid;
  }
  return lo;
}

// Histogram of piece k on the second-pass bits.  It reads the whole pass-1
// tuples for their keys (16 bytes per tuple).  Measured on B200 and left
// out: pass 1 storing each tuple's second-pass digit as a u16 beside the
// tuple, for this histogram to read 2 bytes per tuple: the histogram went
// from 2.9 to 2.0 ms per relation (1024M int64), but the digit stores, two
// bytes each in short runs, made the pass-1 scatter 6.97 -> 12.0 ms.
template <typename K>
__global__ void __launch_bounds__(512)
    piece_histogram_kernel(const Tuple<K> *__restrict__ rel1,
                           const uint64_t *__restrict__ off1, uint32_t C1,
                           uint32_t F1, uint32_t F2, uint64_t mask2,
                           uint32_t ign2, Pass2Plan pl) {
  extern __shared__ uint32_t hist[];
  const uint32_t k = blockIdx.x;
  const uint32_t total = pl.piece_first[F1];
  if (k >= total) return;
  const uint32_t p1 = find_p1(pl.piece_first, F1, k);
  const uint64_t n = pl.p1_base[p1 + 1] - pl.p1_base[p1];
  const uint64_t s0 = (uint64_t)(k - pl.piece_first[p1]) << pl.piece_log2;
  const uint64_t s1 = min(n, s0 + ((uint64_t)1 << pl.piece_log2));
  for (uint32_t i = threadIdx.x; i < F2; i += blockDim.x) hist[i] = 0;
  __syncthreads();
  const uint64_t *rp = pl.reg_pre + (uint64_t)p1 * (C1 + 1);
  for (uint32_t c = 0; c < C1; ++c) {
    const uint64_t rb = rp[c], re = rp[c + 1];
    const uint64_t lo = max(rb, s0), hi = min(re, s1);
    if (lo >= hi) continue;
    const uint64_t phys = off1[(uint64_t)c * F1 + p1] + (lo - rb);
    const uint64_t cnt = hi - lo;
    // four independent key loads per thread in flight (one per thread left
    // the kernel latency-bound: 2.91 -> 2.66 ms per 1024M int64 relation)
    for (uint64_t base = 0; base < cnt; base += 4ull * blockDim.x) {
      K key[4];
#pragma unroll
      for (uint32_t u = 0; u < 4; ++u) {
        const uint64_t i = base + u * blockDim.x + threadIdx.x;
        key[u] = i < cnt ? __ldcs(&rel1[phys + i].key) : K(0);
      }
#pragma unroll
      for (uint32_t u = 0; u < 4; ++u) {
        const uint64_t i = base + u * blockDim.x + threadIdx.x;
        warp_aggregated_count(hist, key_to_partition(key[u], mask2, ign2), i < cnt);
      }
    }
  }
  __syncthreads();
  for (uint32_t i = threadIdx.x; i < F2; i += blockDim.x)
    pl.hist[(uint64_t)k * F2 + i] = hist[i];
}

// Output offsets per (p1, p2) and per-piece cursors; one CTA per p1.
__global__ void __launch_bounds__(1024)
    pass2_cursor_kernel(uint32_t F1, uint32_t F2, Pass2Plan pl) {
  extern __shared__ uint32_t tot[];  // [F2] + 33
  uint32_t *scan_tmp = tot + F2;
  const uint32_t p1 = blockIdx.x;
  const uint32_t kb = pl.piece_first[p1], ke = pl.piece_first[p1 + 1];
  for (uint32_t p2 = threadIdx.x; p2 < F2; p2 += blockDim.x) {
    uint32_t t = 0;
    for (uint32_t k = kb; k < ke; ++k) t += pl.hist[(uint64_t)k * F2 + p2];
    tot[p2] = t;
  }
  __syncthreads();
  block_exclusive_scan_u32(tot, F2, scan_tmp);
  const uint64_t base = pl.p1_base[p1];
  for (uint32_t p2 = threadIdx.x; p2 < F2; p2 += blockDim.x) {
    uint64_t run = base + tot[p2];
    pl.off2[(uint64_t)p1 * F2 + p2] = run;
    for (uint32_t k = kb; k < ke; ++k) {
      pl.cursor[(uint64_t)k * F2 + p2] = run;
      run += pl.hist[(uint64_t)k * F2 + p2];
    }
  }
  if (p1 + 1 == F1 && threadIdx.x == 0) pl.off2[(uint64_t)F1 * F2] = pl.p1_base[F1];
}

// Scatter of piece k into the (p1, p2)-ordered output.
template <typename K>
__global__ void __launch_bounds__(Pass2Shape<K>::kThreads, Pass2Shape<K>::kMinBlocks)
    pass2_scatter_kernel(const Tuple<K> *__restrict__ rel1,
                         const uint64_t *__restrict__ off1, uint32_t C1,
                         uint32_t F1, uint32_t F2, uint64_t mask2,
                         uint32_t ign2, Pass2Plan pl,
                         Tuple<K> *__restrict__ rel2, uint64_t rel2_len,
                         int *status) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  // region tables first (8-byte aligned), then the tile-scatter state
  uint64_t *reg_pre = reinterpret_cast<uint64_t *>(smem_raw);  // [C1 + 1]
  uint64_t *reg_begin = reg_pre + C1 + 1;                      // [C1]
  Tuple<K> *staged = reinterpret_cast<Tuple<K> *>(
      smem_raw + (((2 * (size_t)C1 + 1) * 8 + 15) & ~(size_t)15));
  uint32_t *toff = reinterpret_cast<uint32_t *>(staged + Pass2Shape<K>::kTile);
  uint32_t *cur = toff + F2 + 1;
  uint32_t *scan_tmp = cur + F2;
  const uint32_t k = blockIdx.x;
  const uint32_t total = pl.piece_first[F1];
  if (k >= total) return;
  const uint32_t p1 = find_p1(pl.piece_first, F1, k);
  const uint64_t n = pl.p1_base[p1 + 1] - pl.p1_base[p1];
  const uint64_t s0 = (uint64_t)(k - pl.piece_first[p1]) << pl.piece_log2;
  const uint64_t s1 = min(n, s0 + ((uint64_t)1 << pl.piece_log2));
  const uint64_t *cp = pl.cursor + (uint64_t)k * F2;
  const uint64_t base = cp[0];
  for (uint32_t p = threadIdx.x; p < F2; p += blockDim.x) {
    cur[p] = (uint32_t)(cp[p] - base);
    toff[p] = 0;
  }
  if (threadIdx.x == 0) toff[F2] = 0;
  const uint64_t *rp = pl.reg_pre + (uint64_t)p1 * (C1 + 1);
  for (uint32_t c = threadIdx.x; c <= C1; c += blockDim.x) {
    reg_pre[c] = rp[c];
    if (c < C1) reg_begin[c] = off1[(uint64_t)c * F1 + p1];
  }
  __syncthreads();
  // one logical range over all chunk regions of p1, so tiles stay full
  RegionSource<K> src(rel1, reg_pre, reg_begin, C1);
  tile_scatter_range<K, Pass2Shape<K>>(src, s0, s1, F2, mask2, ign2, cur, toff, scan_tmp,
                        staged, rel2, base, rel2_len, status);
}

// The same scatter fed by TMA bulk copies of the region segments (16-byte
// tuples only).  Shared memory: bars | reg_pre | reg_begin | stages | toff |
// cur | scan_tmp.
__host__ __device__ inline size_t pass2_tma_tables_bytes(uint32_t C1) {
  return (64 + (2 * (size_t)C1 + 1) * 8 + 127) & ~(size_t)127;
}

template <typename K>
__global__ void __launch_bounds__(TmaShape<K>::kThreads, 1)
    pass2_scatter_tma_kernel(const Tuple<K> *__restrict__ rel1,
                             const uint64_t *__restrict__ off1, uint32_t C1,
                             uint32_t F1, uint32_t F2, uint64_t mask2,
                             uint32_t ign2, Pass2Plan pl,
                             Tuple<K> *__restrict__ rel2, uint64_t rel2_len,
                             int *status) {
  using S = TmaShape<K>;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  uint64_t *bars = reinterpret_cast<uint64_t *>(smem_raw);
  uint64_t *reg_pre = bars + 8;             // [C1 + 1]
  uint64_t *reg_begin = reg_pre + C1 + 1;   // [C1]
  unsigned char *stages = smem_raw + pass2_tma_tables_bytes(C1);
  uint32_t *toff =
      reinterpret_cast<uint32_t *>(stages + S::kStages * tma_stage_bytes<K>());
  uint32_t *cur = toff + F2 + 1;
  uint32_t *scan_tmp = cur + F2;
  const uint32_t k = blockIdx.x;
  const uint32_t total = pl.piece_first[F1];
  if (k >= total) return;
  const uint32_t p1 = find_p1(pl.piece_first, F1, k);
  const uint64_t n = pl.p1_base[p1 + 1] - pl.p1_base[p1];
  const uint64_t s0 = (uint64_t)(k - pl.piece_first[p1]) << pl.piece_log2;
  const uint64_t s1 = min(n, s0 + ((uint64_t)1 << pl.piece_log2));
  const uint64_t *cp = pl.cursor + (uint64_t)k * F2;
  const uint64_t base = cp[0];
  for (uint32_t p = threadIdx.x; p < F2; p += blockDim.x)
    cur[p] = (uint32_t)(cp[p] - base);
  for (uint32_t p = threadIdx.x; p <= F2; p += blockDim.x) toff[p] = 0;
  const uint64_t *rp = pl.reg_pre + (uint64_t)p1 * (C1 + 1);
  for (uint32_t c = threadIdx.x; c <= C1; c += blockDim.x) {
    reg_pre[c] = rp[c];
    if (c < C1) reg_begin[c] = off1[(uint64_t)c * F1 + p1];
  }
  if (threadIdx.x == 0) {
    for (uint32_t s = 0; s < S::kStages; ++s) mbar_init(&bars[s], 1);
    mbar_fence_init();
  }
  __syncthreads();
  TmaRegionSource<K> src(rel1, reg_pre, reg_begin, C1);
  // A first-pass partition 8x the average is a Zipf-hot one: its tiles hold
  // long stretches of one key, so whole warps rank into one bin and one
  // atomic per warp replaces 32 (Zipf 1.5, 1024M x 1024M int64: pass-2
  // scatter 16.4 -> 14.1 ms).  Elsewhere the extra shuffle and vote cost
  // 3.5%, so ordinary partitions keep one atomic per tuple.
  if (n > 8 * (pl.p1_base[F1] / F1 + 1))
    tma_tile_scatter_range<K, TmaRegionSource<K>, true>(
        src, s0, s1, F2, mask2, ign2, cur, toff, scan_tmp, stages, bars, rel2,
        base, rel2_len, status);
  else
    tma_tile_scatter_range<K, TmaRegionSource<K>, false>(
        src, s0, s1, F2, mask2, ign2, cur, toff, scan_tmp, stages, bars, rel2,
        base, rel2_len, status);
}

template <typename K>
size_t pass2_tma_smem(uint32_t C1, uint32_t F2) {
  return pass2_tma_tables_bytes(C1) + tma_scatter_smem<K>(F2) - 64;
}

template <typename K>
size_t pass2_scatter_smem(uint32_t C1, uint32_t F2) {
  return (((2 * (size_t)C1 + 1) * 8 + 15) & ~(size_t)15) +
         tile_scatter_smem<K, Pass2Shape<K>>(F2);
}

// The join's per-thread sums, reduced in two launches: every CTA of
// partial_sums_kernel reduces its slice of `per` sums and leaves the
// partial in the slice's first element (only that CTA reads the slice), then
// one CTA of finish_result_kernel adds the partials.  (One CTA reducing all
// 151K sums of a 148 x 1024-thread join took 70 us.)
__global__ void __launch_bounds__(1024)
    partial_sums_kernel(int64_t *__restrict__ sums, uint64_t n, uint64_t per) {
  __shared__ uint64_t tmp[32];
  const uint64_t b0 = blockIdx.x * per, b1 = min(n, b0 + per);
  uint64_t s = 0;
  for (uint64_t i = b0 + threadIdx.x; i < b1; i += blockDim.x) s += (uint64_t)sums[i];
  s = block_reduce_u64(s, tmp);  // every thread's loads are done by now
  if (threadIdx.x == 0 && b0 < n) sums[b0] = (int64_t)s;
}

__global__ void __launch_bounds__(256)
    finish_result_kernel(const int64_t *__restrict__ sums, uint64_t n,
                         uint64_t per, const uint64_t *count,
                         fi_join_result *result) {
  __shared__ uint64_t tmp[32];
  uint64_t s = 0;
  for (uint64_t i = threadIdx.x; i * per < n; i += blockDim.x)
    s += (uint64_t)sums[i * per];
  s = block_reduce_u64(s, tmp);
  if (threadIdx.x == 0) {
    result->sum = (int64_t)s;
    result->count = *count;
  }
}

}  // namespace fi

using namespace fi;

struct fi_radix_join_engine {
  uint64_t max_build, max_probe;
  uint32_t tuple_bytes;   // largest tuple the buffers hold (8 or 16 bytes)
  int32_t bits1, bits2;   // current plan; bits2 < 0: single pass
  int32_t cap1, cap2;     // bits the buffers were sized for
  fi_hashing_scheme scheme;
  uint32_t join_block = 0;  // as planned; 0 = by scheme and partition size
  uint32_t scatter = 0;   // 0: TMA-fed where possible, 1: register-fed
  uint32_t sm_count, C1, F1, F2, max_pieces;
  DevBuf rel1[2], off1[2], loc1[2], rel2[2];
  DevBuf reg_pre[2], p1_base[2], piece_first[2], piece_tmp[2], hist2[2],
      cursor2[2], off2[2];
  DevBuf hist_scratch, tile_state, counters, status;
  DevBuf join_items, join_part, join_counters, join_tiles, join_sums, join_count;
  int scatter_variant() const {
    return scatter == 1 ? kScatterRegisters : kScatterAuto;
  }
  // join shape of a run over `build` tuples in `fanout` partitions
  template <typename K>
  uint32_t join_block_for(uint64_t build, uint32_t fanout) const {
    if (join_block) return join_block;
    return scheme == FI_HASHING_PERFECT ? kJoinBlockPerfect
                                        : join_auto_block<K>(build, fanout);
  }
  DevBuf in_cols[4];  // device copies of host input (run_host)
  uint64_t part_len[2] = {0, 0};  // lengths of the partitioned relations
  bool built = false;             // a build relation is partitioned
  // streamed pass 1 (run_streamed): a copy stream, two staging slots of
  // key and payload columns, their ready/free events, block-local cursors
  cudaStream_t copy_stream = nullptr;
  cudaEvent_t slot_ready[2] = {}, slot_free[2] = {};
  DevBuf stage_key[2], stage_pay[2], stream_loc, result_dev;
  // hybrid run: the CPU's first-pass relations and offsets in pinned memory
  void *host_rel[2] = {nullptr, nullptr};
  uint64_t *host_off[2] = {nullptr, nullptr};
  size_t host_rel_bytes[2] = {0, 0};
  uint64_t workspace = 0;
  cudaEvent_t events[FI_ENGINE_PHASE_EVENTS] = {};
  bool record = false;
  uint32_t launches = 0;

  void mark(int i, cudaStream_t st) {
    if (record) cudaEventRecord(events[i], st);
  }

  int alloc(DevBuf &b, size_t bytes, bool zero = false) {
    int rc = b.reserve(bytes, zero);
    if (rc == FI_OK) workspace += bytes;
    return rc;
  }
  HistScratch hs() {
    return HistScratch{(uint32_t *)hist_scratch.ptr, (uint64_t *)tile_state.ptr,
                       (uint32_t *)counters.ptr, (int *)status.ptr};
  }
  Pass2Plan plan(int r, uint64_t piece) {
    uint32_t lg = 0;
    while ((1ull << lg) < piece) ++lg;
    return Pass2Plan{(uint64_t *)reg_pre[r].ptr, (uint64_t *)p1_base[r].ptr,
                     (uint32_t *)piece_first[r].ptr, (uint32_t *)hist2[r].ptr,
                     (uint64_t *)cursor2[r].ptr, (uint64_t *)off2[r].ptr, lg};
  }
  void release_all() {
    for (int r = 0; r < 2; ++r) {
      rel1[r].release(); off1[r].release(); loc1[r].release(); rel2[r].release();
      reg_pre[r].release(); p1_base[r].release(); piece_first[r].release();
      piece_tmp[r].release(); hist2[r].release(); cursor2[r].release();
      off2[r].release();
    }
    hist_scratch.release(); tile_state.release(); counters.release();
    status.release(); join_items.release(); join_part.release();
    join_counters.release();
    join_tiles.release(); join_sums.release(); join_count.release();
    for (auto &b : in_cols) b.release();
    for (int i = 0; i < 2; ++i) {
      stage_key[i].release();
      stage_pay[i].release();
      if (slot_ready[i]) cudaEventDestroy(slot_ready[i]);
      if (slot_free[i]) cudaEventDestroy(slot_free[i]);
      slot_ready[i] = slot_free[i] = nullptr;
    }
    stream_loc.release();
    result_dev.release();
    for (int i = 0; i < 2; ++i) {
      if (host_rel[i]) cudaFreeHost(host_rel[i]);
      if (host_off[i]) cudaFreeHost(host_off[i]);
      host_rel[i] = nullptr;
      host_off[i] = nullptr;
      host_rel_bytes[i] = 0;
    }
    if (copy_stream) cudaStreamDestroy(copy_stream);
    copy_stream = nullptr;
  }
};

extern "C" int fi_radix_join_engine_new(uint64_t max_build_len,
                                        uint64_t max_probe_len,
                                        uint32_t tuple_bytes,
                                        fi_radix_bits radix_bits,
                                        fi_hashing_scheme hashing_scheme,
                                        fi_radix_join_engine **out) {
  if (!out) return set_error(FI_ERR_INVALID_ARGUMENT, "null output handle");
  *out = nullptr;
  if (tuple_bytes != 8 && tuple_bytes != 16)
    return set_error(FI_ERR_INVALID_ARGUMENT, "tuple_bytes must be 8 or 16");
  if (hashing_scheme != FI_HASHING_PERFECT &&
      hashing_scheme != FI_HASHING_BUCKET_CHAINING)
    return set_error(FI_ERR_UNSUPPORTED,
                     "the radix join supports Perfect and BucketChaining");
  const int32_t b1 = radix_bits.pass_bits[0], b2 = radix_bits.pass_bits[1];
  if (b1 < 0 || b1 > (int32_t)kMaxHistBits || b1 > (int32_t)kMaxTileBits ||
      b2 > 10 || radix_bits.pass_bits[2] >= 0)
    return set_error(FI_ERR_UNSUPPORTED,
                     "the engine supports one or two passes with at most 14 "
                     "first-pass and 10 second-pass bits");
  if (b2 >= 0 && b1 + b2 > 24)
    return set_error(FI_ERR_UNSUPPORTED, "at most 24 radix bits in total");
  auto *e = new fi_radix_join_engine();
  e->max_build = max_build_len;
  e->max_probe = max_probe_len;
  e->tuple_bytes = tuple_bytes;
  e->bits1 = e->cap1 = b1;
  e->bits2 = e->cap2 = b2;
  e->scheme = hashing_scheme;
  e->sm_count = (uint32_t)device_sm_count();
  e->C1 = e->sm_count * kChunksPerSm;
  e->F1 = 1u << b1;
  e->F2 = b2 >= 0 ? (1u << b2) : 1u;
  const uint64_t maxn = std::max(max_build_len, max_probe_len);
  // pieces of a relation of len <= maxn tuples: at most len / piece + F1,
  // and len / piece_tuples(len) stays below 8 per SM or maxn / 2^18
  e->max_pieces = (uint32_t)(std::max<uint64_t>(8ull * e->sm_count,
                                                 (maxn + kMaxPieceTuples - 1) /
                                                     kMaxPieceTuples) +
                             e->F1 + 1);
  const uint64_t pad = kPaddingBytes / tuple_bytes;
  const uint32_t pass1_chunks = b2 >= 0 ? e->C1 : 1;
  int rc = FI_OK;
  const uint64_t lens[2] = {max_build_len, max_probe_len};
  for (int r = 0; r < 2 && !rc; ++r) {
    rc = e->alloc(e->rel1[r], (lens[r] + (uint64_t)pass1_chunks * e->F1 * pad) *
                                  tuple_bytes);
    if (!rc) rc = e->alloc(e->off1[r], (size_t)e->C1 * e->F1 * 8);
    if (!rc) rc = e->alloc(e->loc1[r], (size_t)e->C1 * e->F1 * 8);
    if (!rc && b2 >= 0) {
      rc = e->alloc(e->rel2[r], std::max<uint64_t>(lens[r], 1) * tuple_bytes);
      if (!rc) rc = e->alloc(e->reg_pre[r], (size_t)e->F1 * (e->C1 + 1) * 8);
      if (!rc) rc = e->alloc(e->p1_base[r], (size_t)(e->F1 + 1) * 8);
      if (!rc) rc = e->alloc(e->piece_first[r], (size_t)(e->F1 + 1) * 4);
      if (!rc) rc = e->alloc(e->piece_tmp[r], (size_t)(e->F1 + 1) * 8);
      if (!rc) rc = e->alloc(e->hist2[r], (size_t)e->max_pieces * e->F2 * 4);
      if (!rc) rc = e->alloc(e->cursor2[r], (size_t)e->max_pieces * e->F2 * 8);
      if (!rc) rc = e->alloc(e->off2[r], ((size_t)e->F1 * e->F2 + 1) * 8);
    }
  }
  const uint32_t Fj = e->F1 * e->F2;
  if (!rc) rc = e->alloc(e->hist_scratch, (size_t)e->C1 * e->F1 * 4, true);
  if (!rc) rc = e->alloc(e->tile_state, ((size_t)e->F1 / kScanTile + 2) * 8, true);
  if (!rc) rc = e->alloc(e->counters, 16, true);
  if (!rc) rc = e->alloc(e->status, 16, true);
  if (!rc) rc = e->alloc(e->join_items, ((size_t)Fj + 1) * 4);
  // item capacity for the largest padding in tuples (8-byte tuples)
  if (!rc)
    rc = e->alloc(e->join_part,
                  (size_t)join_items_capacity(
                      Fj, max_probe_len + (uint64_t)e->F1 * (kPaddingBytes / 8)) *
                      4);
  if (!rc) rc = e->alloc(e->join_counters, 16, true);
  if (!rc) rc = e->alloc(e->join_tiles, ((size_t)Fj / 1024 + 2) * 8, true);
  // per-thread sums for every join shape (grid x block = SM x 1024)
  if (!rc) rc = e->alloc(e->join_sums, (size_t)e->sm_count * 1024 * 8);
  if (!rc) rc = e->alloc(e->join_count, 16);
  if (rc) {
    e->release_all();
    delete e;
    return rc;
  }
  *out = e;
  return FI_OK;
}

extern "C" void fi_radix_join_engine_free(fi_radix_join_engine *e) {
  if (!e) return;
  e->release_all();
  delete e;
}

extern "C" uint64_t fi_radix_join_engine_workspace_bytes(
    const fi_radix_join_engine *e) {
  return e ? e->workspace : 0;
}

extern "C" int fi_radix_join_engine_status(fi_radix_join_engine *e) {
  if (!e) return set_error(FI_ERR_INVALID_ARGUMENT, "null handle");
  return read_and_clear_status(e->status);
}

extern "C" int fi_radix_join_engine_status_async(fi_radix_join_engine *e,
                                                 int *host_status,
                                                 fi_stream_t stream) {
  if (!e || !host_status) return set_error(FI_ERR_INVALID_ARGUMENT, "null argument");
  cudaStream_t st = (cudaStream_t)stream;
  cudaError_t ce = cudaMemcpyAsync(host_status, e->status.ptr, sizeof(int),
                                   cudaMemcpyDeviceToHost, st);
  if (ce == cudaSuccess) ce = cudaMemsetAsync(e->status.ptr, 0, sizeof(int), st);
  if (ce != cudaSuccess) return cuda_error(ce, "status copy");
  return FI_OK;
}

#define FI_CK(expr, what)                                                      \
  do {                                                                         \
    cudaError_t e_ = (expr);                                                   \
    if (e_ != cudaSuccess) return cuda_error(e_, what);                        \
  } while (0)

// Second pass of relation r: from its pass-1 layout (C1 chunks of F1
// partitions, padded length padded1) into rel2[r], ordered by (p1, p2) with
// no padding.  Four launches: plan, piece histograms, cursors, scatter.
template <typename K>
static int engine_pass2(fi_radix_join_engine *e, int r, uint32_t C1,
                        uint64_t padded1, uint64_t len, cudaStream_t st) {
  const uint32_t F1 = e->F1, F2 = e->F2;
  const uint32_t b1 = (uint32_t)e->bits1;
  const uint32_t pad = kPaddingBytes / sizeof(Tuple<K>);
  const uint64_t mask2 = (uint64_t)(F2 - 1u) << b1;
  Pass2Plan pl = e->plan(r, piece_tuples(len, e->sm_count));
  pass2_regions_kernel<<<(F1 + 31) / 32, 1024, 0, st>>>(
      (const uint64_t *)e->off1[r].ptr, C1, F1, padded1, pad, pl,
      (uint64_t *)e->piece_tmp[r].ptr);
  pass2_plan_kernel<<<1, 1024, 0, st>>>(F1, pl, (uint64_t *)e->piece_tmp[r].ptr);
  FI_CK(cudaGetLastError(), "pass-2 plan");
  piece_histogram_kernel<K><<<e->max_pieces, 512, F2 * 4, st>>>(
      (const Tuple<K> *)e->rel1[r].ptr, (const uint64_t *)e->off1[r].ptr, C1, F1,
      F2, mask2, b1, pl);
  FI_CK(cudaGetLastError(), "pass-2 histogram");
  const size_t csm = (size_t)(F2 + 33) * 4;
  pass2_cursor_kernel<<<F1, 1024, csm, st>>>(F1, F2, pl);
  FI_CK(cudaGetLastError(), "pass-2 cursors");
  e->mark(3 + 4 * r, st);
  bool tma_done = false;
  if constexpr (sizeof(Tuple<K>) == 16) {
    // TMA-fed stages (the pass-1 relation is a 16-byte aligned allocation of
    // 16-byte tuples, so every region segment qualifies)
    const size_t tsm = pass2_tma_smem<K>(C1, F2);
    if (e->scatter == 0 && tsm <= (size_t)device_max_smem_optin()) {
      FI_CK(cudaFuncSetAttribute((const void *)pass2_scatter_tma_kernel<K>,
                                 cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)tsm),
            "smem attribute");
      pass2_scatter_tma_kernel<K><<<e->max_pieces, TmaShape<K>::kThreads, tsm, st>>>(
          (const Tuple<K> *)e->rel1[r].ptr, (const uint64_t *)e->off1[r].ptr, C1,
          F1, F2, mask2, b1, pl, (Tuple<K> *)e->rel2[r].ptr, len,
          (int *)e->status.ptr);
      tma_done = true;
    }
  }
  if (!tma_done) {
    const size_t ssm = pass2_scatter_smem<K>(C1, F2);
    FI_CK(cudaFuncSetAttribute((const void *)pass2_scatter_kernel<K>,
                               cudaFuncAttributeMaxDynamicSharedMemorySize,
                               (int)ssm),
          "smem attribute");
    pass2_scatter_kernel<K><<<e->max_pieces, Pass2Shape<K>::kThreads, ssm, st>>>(
        (const Tuple<K> *)e->rel1[r].ptr, (const uint64_t *)e->off1[r].ptr, C1, F1,
        F2, mask2, b1, pl, (Tuple<K> *)e->rel2[r].ptr, len, (int *)e->status.ptr);
  }
  FI_CK(cudaGetLastError(), "pass-2 scatter");
  e->mark(4 + 4 * r, st);
  e->launches += 5;  // regions, plan, piece histograms, cursors, scatter
  return FI_OK;
}

// Partitions relation r (0 = build, 1 = probe) into the layout the join
// reads: one Contiguous pass into rel1[r]/off1[r], or two passes into
// rel2[r]/off2[r].
template <typename K>
static int engine_partition(fi_radix_join_engine *e, int r, const K *key,
                            const K *pay, uint64_t len, cudaStream_t st) {
  const uint32_t C1 = e->C1, F1 = e->F1;
  const uint32_t b1 = (uint32_t)e->bits1;
  const uint32_t pad = kPaddingBytes / sizeof(Tuple<K>);
  if ((uint64_t)(len + C1 - 1) / C1 >= 0xffffffffull)
    return set_error(FI_ERR_INTEGER_OVERFLOW, "relation too large");
  if (e->bits2 < 0) {
    const uint64_t padded = len + (uint64_t)F1 * pad;
    FI_CK(launch_contiguous_prefix_sum<K>(
              key, nullptr, len, C1, b1, 0, pad, nullptr, nullptr,
              (uint64_t *)e->off1[r].ptr, (uint64_t *)e->loc1[r].ptr, 0,
              e->hs(), e->sm_count, st),
          "prefix sum");
    e->mark(1 + 4 * r, st);
    FI_CK(launch_partition<K>(key, pay, len, C1, b1, 0,
                              (const uint64_t *)e->loc1[r].ptr, e->rel1[r].ptr,
                              padded, e->scatter_variant(), (int *)e->status.ptr,
                              st),
          "partition");
    e->mark(2 + 4 * r, st);
    e->mark(3 + 4 * r, st);
    e->mark(4 + 4 * r, st);
    e->launches += 3;
  } else {
    const uint64_t padded1 = len + (uint64_t)C1 * F1 * pad;
    FI_CK(launch_chunked_prefix_sum<K>(key, len, C1, b1, 0, pad,
                                       (uint64_t *)e->off1[r].ptr, e->hs(),
                                       e->sm_count, st),
          "pass-1 prefix sum");
    e->mark(1 + 4 * r, st);
    FI_CK(launch_partition<K>(key, pay, len, C1, b1, 0,
                              (const uint64_t *)e->off1[r].ptr, e->rel1[r].ptr,
                              padded1, e->scatter_variant(), (int *)e->status.ptr,
                              st),
          "pass-1 partition");
    e->mark(2 + 4 * r, st);
    int rc = engine_pass2<K>(e, r, C1, padded1, len, st);
    if (rc) return rc;
    e->launches += (hist_splits(C1, e->sm_count) == 1 ? 1u : 2u) + 1;
  }
  e->part_len[r] = len;
  return FI_OK;
}

// Joins the partitioned build and probe relations and writes {sum, count}
// to the device `result`.
template <typename K>
static int engine_join(fi_radix_join_engine *e, fi_join_result *result,
                       cudaStream_t st) {
  FI_CK(cudaMemsetAsync(e->join_sums.ptr, 0, e->join_sums.size, st), "memset");
  FI_CK(cudaMemsetAsync(e->join_count.ptr, 0, 8, st), "memset");
  const int scheme = e->scheme == FI_HASHING_PERFECT ? 0 : 2;
  JoinScratch js{(uint32_t *)e->join_items.ptr, (uint32_t *)e->join_part.ptr,
                 (uint64_t *)e->join_tiles.ptr, (uint32_t *)e->join_counters.ptr,
                 (int *)e->status.ptr};
  const uint32_t jb =
      e->join_block_for<K>(e->part_len[0], e->bits2 < 0 ? e->F1 : e->F1 * e->F2);
  const uint32_t grid = e->sm_count * join_ctas_per_sm(jb);
  if (e->bits2 < 0) {
    const uint32_t pad = kPaddingBytes / sizeof(Tuple<K>);
    const uint64_t padded[2] = {e->part_len[0] + (uint64_t)e->F1 * pad,
                                e->part_len[1] + (uint64_t)e->F1 * pad};
    FI_CK(launch_radix_join<K>(e->rel1[0].ptr, (const uint64_t *)e->off1[0].ptr,
                               padded[0], pad, e->rel1[1].ptr,
                               (const uint64_t *)e->off1[1].ptr, padded[1], pad,
                               e->F1, (uint32_t)e->bits1, scheme, grid, jb,
                               (int64_t *)e->join_sums.ptr,
                               (uint64_t *)e->join_count.ptr, js, e->sm_count,
                               st),
          "join");
  } else {
    FI_CK(launch_radix_join<K>(e->rel2[0].ptr, (const uint64_t *)e->off2[0].ptr,
                               e->part_len[0], 0, e->rel2[1].ptr,
                               (const uint64_t *)e->off2[1].ptr, e->part_len[1], 0,
                               e->F1 * e->F2, (uint32_t)(e->bits1 + e->bits2),
                               scheme, grid, jb, (int64_t *)e->join_sums.ptr,
                               (uint64_t *)e->join_count.ptr, js, e->sm_count,
                               st),
          "join");
  }
  e->mark(9, st);
  const uint64_t nsums = (uint64_t)grid * jb;
  const uint64_t per = (nsums + e->sm_count - 1) / e->sm_count;
  partial_sums_kernel<<<(uint32_t)((nsums + per - 1) / per), 1024, 0, st>>>(
      (int64_t *)e->join_sums.ptr, nsums, per);
  finish_result_kernel<<<1, 256, 0, st>>>((const int64_t *)e->join_sums.ptr, nsums,
                                          per, (const uint64_t *)e->join_count.ptr,
                                          result);
  FI_CK(cudaGetLastError(), "result");
  e->launches += 4;  // join plan, join, partial sums, result
  e->mark(10, st);
  return FI_OK;
}

template <typename K>
static int engine_check(fi_radix_join_engine *e, int r, const K *key,
                        const K *pay, uint64_t len) {
  if (!e) return set_error(FI_ERR_INVALID_ARGUMENT, "null handle");
  if (2 * sizeof(K) > e->tuple_bytes)
    return set_error(FI_ERR_INVALID_ARGUMENT,
                     "tuples larger than the engine was built for");
  if (len > (r == 0 ? e->max_build : e->max_probe))
    return set_error(FI_ERR_INVALID_ARGUMENT,
                     "relation larger than the engine's workspace");
  if (len > 0 && (!key || !pay))
    return set_error(FI_ERR_INVALID_ARGUMENT, "null column");
  return FI_OK;
}

template <typename K>
static int engine_run(fi_radix_join_engine *e, const K *bk, const K *bp,
                      uint64_t bn, const K *pk, const K *pp, uint64_t pn,
                      fi_join_result *result, cudaStream_t st) {
  int rc = engine_check<K>(e, 0, bk, bp, bn);
  if (!rc) rc = engine_check<K>(e, 1, pk, pp, pn);
  if (rc) return rc;
  if (!result) return set_error(FI_ERR_INVALID_ARGUMENT, "null result");
  e->launches = 0;
  e->mark(0, st);
  rc = engine_partition<K>(e, 0, bk, bp, bn, st);
  if (!rc) rc = engine_partition<K>(e, 1, pk, pp, pn, st);
  if (!rc) e->built = true;
  if (!rc) rc = engine_join<K>(e, result, st);
  return rc;
}

// Build once, probe many: the build relation stays partitioned in the
// engine until the next build, and every probe joins a probe relation (or a
// slice of one) against it.
template <typename K>
static int engine_build(fi_radix_join_engine *e, const K *key, const K *pay,
                        uint64_t len, cudaStream_t st) {
  int rc = engine_check<K>(e, 0, key, pay, len);
  if (rc) return rc;
  e->launches = 0;
  e->mark(0, st);
  rc = engine_partition<K>(e, 0, key, pay, len, st);
  e->built = rc == FI_OK;
  return rc;
}

template <typename K>
static int engine_probe(fi_radix_join_engine *e, const K *key, const K *pay,
                        uint64_t len, fi_join_result *result, cudaStream_t st) {
  int rc = engine_check<K>(e, 1, key, pay, len);
  if (rc) return rc;
  if (!result) return set_error(FI_ERR_INVALID_ARGUMENT, "null result");
  if (!e->built) return set_error(FI_ERR_INVALID_ARGUMENT, "probe before build");
  e->launches = 0;
  rc = engine_partition<K>(e, 1, key, pay, len, st);
  if (!rc) rc = engine_join<K>(e, result, st);
  return rc;
}

extern "C" int fi_radix_join_engine_set_events(fi_radix_join_engine *e,
                                               void **events,
                                               uint32_t n_events) {
  if (!e) return set_error(FI_ERR_INVALID_ARGUMENT, "null handle");
  if (!events) {
    e->record = false;
    return FI_OK;
  }
  if (n_events < FI_ENGINE_PHASE_EVENTS)
    return set_error(FI_ERR_INVALID_ARGUMENT, "need %d events",
                     FI_ENGINE_PHASE_EVENTS);
  for (int i = 0; i < FI_ENGINE_PHASE_EVENTS; ++i)
    if (!events[i])
      return set_error(FI_ERR_INVALID_ARGUMENT, "event %d is not a created event", i);
  for (int i = 0; i < FI_ENGINE_PHASE_EVENTS; ++i)
    e->events[i] = (cudaEvent_t)events[i];
  e->record = true;
  return FI_OK;
}

extern "C" uint32_t fi_radix_join_engine_last_launches(
    const fi_radix_join_engine *e) {
  return e ? e->launches : 0;
}

extern "C" int fi_radix_join_engine_run_int32(
    fi_radix_join_engine *e, const int32_t *build_key, const int32_t *build_pay,
    uint64_t build_len, const int32_t *probe_key, const int32_t *probe_pay,
    uint64_t probe_len, fi_join_result *result, fi_stream_t stream) {
  return engine_run<int32_t>(e, build_key, build_pay, build_len, probe_key,
                             probe_pay, probe_len, result, (cudaStream_t)stream);
}
extern "C" int fi_radix_join_engine_run_int64(
    fi_radix_join_engine *e, const int64_t *build_key, const int64_t *build_pay,
    uint64_t build_len, const int64_t *probe_key, const int64_t *probe_pay,
    uint64_t probe_len, fi_join_result *result, fi_stream_t stream) {
  return engine_run<int64_t>(e, build_key, build_pay, build_len, probe_key,
                             probe_pay, probe_len, result, (cudaStream_t)stream);
}

template <typename K>
static int engine_run_streamed(fi_radix_join_engine *e, const K *bk,
                               const K *bp, uint64_t bn, const K *pk,
                               const K *pp, uint64_t pn, uint64_t block_tuples,
                               fi_join_result *result, cudaStream_t st);
uint64_t host_stream_block(uint64_t maxn, uint32_t c1);

// Host columns.  With two passes the columns are streamed block by block
// (engine_run_streamed), so the copy of one block overlaps the first pass of
// the one before and the host link is the only bound; one pass copies the
// columns whole and runs the in-memory join.  Same results either way.
template <typename K>
static int engine_run_host(fi_radix_join_engine *e, const K *build_key,
                           const K *build_pay, uint64_t build_len,
                           const K *probe_key, const K *probe_pay,
                           uint64_t probe_len, fi_join_result *result,
                           cudaStream_t st) {
  if (!e || !result) return set_error(FI_ERR_INVALID_ARGUMENT, "null argument");
  if (e->bits2 >= 0)
    return engine_run_streamed<K>(
        e, build_key, build_pay, build_len, probe_key, probe_pay, probe_len,
        host_stream_block(std::max(build_len, probe_len), e->C1), result, st);
  const K *src[4] = {build_key, build_pay, probe_key, probe_pay};
  const uint64_t lens[4] = {build_len, build_len, probe_len, probe_len};
  for (int i = 0; i < 4; ++i) {
    int rc = e->in_cols[i].reserve(std::max<uint64_t>(lens[i], 1) * sizeof(K), false);
    if (rc) return rc;
    FI_CK(cudaMemcpyAsync(e->in_cols[i].ptr, src[i], lens[i] * sizeof(K),
                          cudaMemcpyHostToDevice, st),
          "host-to-device copy");
  }
  DevBuf dres;
  int rc = dres.reserve(sizeof(fi_join_result), false);
  if (rc) return rc;
  rc = engine_run<K>(e, (const K *)e->in_cols[0].ptr, (const K *)e->in_cols[1].ptr,
                     build_len, (const K *)e->in_cols[2].ptr,
                     (const K *)e->in_cols[3].ptr, probe_len,
                     (fi_join_result *)dres.ptr, st);
  if (rc == FI_OK) {
    cudaError_t ce = cudaMemcpyAsync(result, dres.ptr, sizeof(fi_join_result),
                                     cudaMemcpyDeviceToHost, st);
    if (ce == cudaSuccess) ce = cudaStreamSynchronize(st);
    if (ce != cudaSuccess) rc = cuda_error(ce, "result copy");
  }
  dres.release();
  return rc;
}

extern "C" int fi_radix_join_engine_run_host_int32(
    fi_radix_join_engine *e, const int32_t *build_key, const int32_t *build_pay,
    uint64_t build_len, const int32_t *probe_key, const int32_t *probe_pay,
    uint64_t probe_len, fi_join_result *result, fi_stream_t stream) {
  return engine_run_host<int32_t>(e, build_key, build_pay, build_len, probe_key,
                                  probe_pay, probe_len, result, (cudaStream_t)stream);
}
extern "C" int fi_radix_join_engine_run_host_int64(
    fi_radix_join_engine *e, const int64_t *build_key, const int64_t *build_pay,
    uint64_t build_len, const int64_t *probe_key, const int64_t *probe_pay,
    uint64_t probe_len, fi_join_result *result, fi_stream_t stream) {
  return engine_run_host<int64_t>(e, build_key, build_pay, build_len, probe_key,
                                  probe_pay, probe_len, result, (cudaStream_t)stream);
}

extern "C" int fi_radix_join_engine_build_int32(fi_radix_join_engine *e,
                                                const int32_t *build_key,
                                                const int32_t *build_pay,
                                                uint64_t build_len,
                                                fi_stream_t stream) {
  return engine_build<int32_t>(e, build_key, build_pay, build_len,
                               (cudaStream_t)stream);
}
extern "C" int fi_radix_join_engine_build_int64(fi_radix_join_engine *e,
                                                const int64_t *build_key,
                                                const int64_t *build_pay,
                                                uint64_t build_len,
                                                fi_stream_t stream) {
  return engine_build<int64_t>(e, build_key, build_pay, build_len,
                               (cudaStream_t)stream);
}
extern "C" int fi_radix_join_engine_probe_int32(
    fi_radix_join_engine *e, const int32_t *probe_key, const int32_t *probe_pay,
    uint64_t probe_len, fi_join_result *result, fi_stream_t stream) {
  return engine_probe<int32_t>(e, probe_key, probe_pay, probe_len, result,
                               (cudaStream_t)stream);
}
extern "C" int fi_radix_join_engine_probe_int64(
    fi_radix_join_engine *e, const int64_t *probe_key, const int64_t *probe_pay,
    uint64_t probe_len, fi_join_result *result, fi_stream_t stream) {
  return engine_probe<int64_t>(e, probe_key, probe_pay, probe_len, result,
                               (cudaStream_t)stream);
}

// ---- per-run plan -------------------------------------------------------------
extern "C" int fi_radix_join_engine_set_plan(fi_radix_join_engine *e,
                                             const fi_join_plan *plan) {
  if (!e || !plan) return set_error(FI_ERR_INVALID_ARGUMENT, "null argument");
  const int32_t b1 = plan->radix_bits.pass_bits[0];
  const int32_t b2 = plan->radix_bits.pass_bits[1];
  if (b1 < 0 || b1 > e->cap1 || plan->radix_bits.pass_bits[2] >= 0)
    return set_error(FI_ERR_INVALID_ARGUMENT,
                     "first-pass bits must lie in [0, %d], the engine's size",
                     e->cap1);
  if (b2 >= 0 && (e->cap2 < 0 || b2 > e->cap2))
    return set_error(FI_ERR_INVALID_ARGUMENT,
                     "second-pass bits exceed the engine's size");
  if (plan->hashing_scheme != FI_HASHING_PERFECT &&
      plan->hashing_scheme != FI_HASHING_BUCKET_CHAINING)
    return set_error(FI_ERR_UNSUPPORTED,
                     "the radix join supports Perfect and BucketChaining");
  const uint32_t jb = plan->join_block;
  if (jb != 0 && jb != 256 && jb != 512 && jb != 1024)
    return set_error(FI_ERR_INVALID_ARGUMENT,
                     "join_block must be 0 (by partition size), 256, 512 or 1024");
  if (plan->scatter > 1)
    return set_error(FI_ERR_INVALID_ARGUMENT, "unknown scatter variant");
  e->bits1 = b1;
  e->bits2 = b2;
  e->F1 = 1u << b1;
  e->F2 = b2 >= 0 ? (1u << b2) : 1u;
  e->scheme = plan->hashing_scheme;
  e->join_block = jb;
  e->scatter = plan->scatter;
  e->built = false;  // a resident build side used the old plan
  return FI_OK;
}

// ---- out-of-core: first pass streamed from host memory ----------------------
// The relations stay in host memory; pass 1 reads them over the host link
// exactly once.  The input is cut into blocks of B tuples.  Block j is copied
// into one of two device staging slots on a copy stream while the compute
// stream partitions block j-1 out of the other slot, so the link and the
// partitioning overlap.  Each block is partitioned on its own, with the
// Contiguous layout over SM-count sub-chunks, into its own region of the
// pass-1 relation: region base j*(B + F1*pad), i.e. the pass-1 relation is a
// Chunked layout whose chunks are the blocks.  Pass 2 and the join then run
// in HBM exactly as in the in-memory engine.  The nearest reference pieces
// are the chunked multi-stream copy of numa-gpu/src/runtime/cuda.rs:891-985
// and the cache-and-spill staging of gpu_triton_join.rs:391-470; the
// reference has no streamed radix join.
constexpr uint64_t kStreamBlockDefault = 1ull << 26;  // tuples per block
constexpr uint64_t kStreamBlockAlign = 1ull << 16;

// Block size for run_host: the default, or larger when a relation would
// otherwise need more blocks than the engine has pass-1 chunks.
uint64_t host_stream_block(uint64_t maxn, uint32_t c1) {
  uint64_t b = (maxn + c1 - 1) / c1;
  b = (b + kStreamBlockAlign - 1) / kStreamBlockAlign * kStreamBlockAlign;
  return std::max(b, kStreamBlockDefault);
}

template <typename K>
static int engine_stream_pass1(fi_radix_join_engine *e, int r, const K *key,
                               const K *pay, uint64_t len, uint64_t B,
                               uint32_t nb, uint64_t *blk, cudaStream_t st) {
  const uint32_t F1 = e->F1;
  const uint32_t pad = kPaddingBytes / sizeof(Tuple<K>);
  const uint64_t padded1 = len + (uint64_t)nb * F1 * pad;
  for (uint32_t j = 0; j < nb; ++j, ++*blk) {
    const int slot = (int)(*blk & 1);
    const uint64_t n = std::min<uint64_t>(B, len - (uint64_t)j * B);
    K *sk = (K *)e->stage_key[slot].ptr, *sp = (K *)e->stage_pay[slot].ptr;
    // the slot's previous block must be partitioned before the copy
    // overwrites it
    if (*blk >= 2)
      FI_CK(cudaStreamWaitEvent(e->copy_stream, e->slot_free[slot], 0),
            "stream wait");
    FI_CK(cudaMemcpyAsync(sk, key + (uint64_t)j * B, n * sizeof(K),
                          cudaMemcpyHostToDevice, e->copy_stream),
          "host-to-device copy");
    FI_CK(cudaMemcpyAsync(sp, pay + (uint64_t)j * B, n * sizeof(K),
                          cudaMemcpyHostToDevice, e->copy_stream),
          "host-to-device copy");
    FI_CK(cudaEventRecord(e->slot_ready[slot], e->copy_stream), "event record");
    FI_CK(cudaStreamWaitEvent(st, e->slot_ready[slot], 0), "stream wait");
    FI_CK(launch_contiguous_prefix_sum<K>(
              sk, nullptr, n, e->sm_count, (uint32_t)e->bits1, 0, pad, nullptr,
              nullptr, (uint64_t *)e->off1[r].ptr + (uint64_t)j * F1,
              (uint64_t *)e->stream_loc.ptr,
              (uint64_t)j * (B + (uint64_t)F1 * pad), e->hs(), e->sm_count, st),
          "pass-1 prefix sum");
    FI_CK(launch_partition<K>(sk, sp, n, e->sm_count, (uint32_t)e->bits1, 0,
                              (const uint64_t *)e->stream_loc.ptr,
                              e->rel1[r].ptr, padded1, e->scatter_variant(),
                              (int *)e->status.ptr, st),
          "pass-1 partition");
    FI_CK(cudaEventRecord(e->slot_free[slot], st), "event record");
    e->launches += 3;
  }
  return FI_OK;
}

template <typename K>
static int engine_run_streamed(fi_radix_join_engine *e, const K *bk,
                               const K *bp, uint64_t bn, const K *pk,
                               const K *pp, uint64_t pn, uint64_t block_tuples,
                               fi_join_result *result, cudaStream_t st) {
  int rc = engine_check<K>(e, 0, bk, bp, bn);
  if (!rc) rc = engine_check<K>(e, 1, pk, pp, pn);
  if (rc) return rc;
  if (!result) return set_error(FI_ERR_INVALID_ARGUMENT, "null result");
  if (e->bits2 < 0)
    return set_error(FI_ERR_UNSUPPORTED,
                     "the streamed join needs two radix passes (the first pass "
                     "is partitioned block by block)");
  uint64_t B = block_tuples ? block_tuples : kStreamBlockDefault;
  B = (B + kStreamBlockAlign - 1) / kStreamBlockAlign * kStreamBlockAlign;
  const uint64_t maxn = std::max(bn, pn);
  if (maxn > 0 && B > maxn)
    B = (maxn + kStreamBlockAlign - 1) / kStreamBlockAlign * kStreamBlockAlign;
  const uint64_t lens[2] = {bn, pn};
  uint32_t nb[2];
  for (int r = 0; r < 2; ++r) {
    const uint64_t blocks = (lens[r] + B - 1) / B;
    if (blocks > e->C1)
      return set_error(FI_ERR_INVALID_ARGUMENT,
                       "block_tuples = %llu cuts a relation into %llu blocks; "
                       "at most %u are supported, use larger blocks",
                       (unsigned long long)B, (unsigned long long)blocks, e->C1);
    nb[r] = (uint32_t)blocks;
  }
  if (bn == 0 || pn == 0) {
    const fi_join_result zero{0, 0};
    std::memcpy(result, &zero, sizeof zero);
    return FI_OK;
  }
  // lazily set up the copy stream, events and staging slots
  if (!e->copy_stream)
    FI_CK(cudaStreamCreateWithFlags(&e->copy_stream, cudaStreamNonBlocking),
          "stream create");
  for (int i = 0; i < 2; ++i) {
    if (!e->slot_ready[i])
      FI_CK(cudaEventCreateWithFlags(&e->slot_ready[i], cudaEventDisableTiming),
            "event create");
    if (!e->slot_free[i])
      FI_CK(cudaEventCreateWithFlags(&e->slot_free[i], cudaEventDisableTiming),
            "event create");
    rc = e->stage_key[i].reserve(B * sizeof(K), false);
    if (!rc) rc = e->stage_pay[i].reserve(B * sizeof(K), false);
    if (rc) return rc;
  }
  rc = e->stream_loc.reserve((size_t)e->sm_count * e->F1 * 8, false);
  if (!rc) rc = e->result_dev.reserve(sizeof(fi_join_result), false);
  if (rc) return rc;

  e->launches = 0;
  e->mark(0, st);
  const K *keys[2] = {bk, pk}, *pays[2] = {bp, pp};
  const uint32_t pad = kPaddingBytes / sizeof(Tuple<K>);
  uint64_t blk = 0;
  for (int r = 0; r < 2; ++r) {
    e->mark(1 + 4 * r, st);
    rc = engine_stream_pass1<K>(e, r, keys[r], pays[r], lens[r], B, nb[r], &blk,
                                st);
    if (rc) return rc;
    e->mark(2 + 4 * r, st);
    const uint64_t padded1 = lens[r] + (uint64_t)nb[r] * e->F1 * pad;
    rc = engine_pass2<K>(e, r, nb[r], padded1, lens[r], st);
    if (rc) return rc;
    e->part_len[r] = lens[r];
  }
  e->built = true;
  rc = engine_join<K>(e, (fi_join_result *)e->result_dev.ptr, st);
  if (rc) return rc;
  FI_CK(cudaMemcpyAsync(result, e->result_dev.ptr, sizeof(fi_join_result),
                        cudaMemcpyDeviceToHost, st),
        "result copy");
  FI_CK(cudaStreamSynchronize(st), "synchronize");
  return FI_OK;
}

// Hybrid join (radix-join/src/execution_methods/cpu_partitioned_radix_join.rs:
// 118-769): the first pass runs on the CPU, one canonical chunk per host
// thread (cpu_partition.cu, write-combining scatter) into pinned memory; the
// partitioned relation and its Chunked offsets are copied to the device and
// the GPU runs the second pass and the join.  The CPU partitions S while
// the GPU copies R and runs its second pass.  Synchronous.
template <typename K>
static int engine_run_hybrid(fi_radix_join_engine *e, const K *bk, const K *bp,
                             uint64_t bn, const K *pk, const K *pp, uint64_t pn,
                             uint32_t threads, fi_join_result *result,
                             cudaStream_t st) {
  int rc = engine_check<K>(e, 0, bk, bp, bn);
  if (!rc) rc = engine_check<K>(e, 1, pk, pp, pn);
  if (rc) return rc;
  if (!result) return set_error(FI_ERR_INVALID_ARGUMENT, "null result");
  if (e->bits2 < 0)
    return set_error(FI_ERR_UNSUPPORTED,
                     "the hybrid join runs the second pass on the GPU; it needs "
                     "two radix passes");
  if (threads == 0) threads = std::max(1u, std::thread::hardware_concurrency());
  const uint32_t C = std::min(threads, e->C1);
  const uint32_t F1 = e->F1, b1 = (uint32_t)e->bits1;
  const uint64_t pad = kPaddingBytes / sizeof(Tuple<K>);
  const uint64_t lens[2] = {bn, pn};
  const K *keys[2] = {bk, pk}, *pays[2] = {bp, pp};
  for (int r = 0; r < 2; ++r) {
    const size_t need = (size_t)(lens[r] + (uint64_t)C * F1 * pad) * sizeof(Tuple<K>);
    if (e->host_rel_bytes[r] < need) {
      if (e->host_rel[r]) cudaFreeHost(e->host_rel[r]);
      e->host_rel[r] = nullptr;
      e->host_rel_bytes[r] = 0;
      FI_CK(cudaHostAlloc(&e->host_rel[r], need, cudaHostAllocDefault),
            "pinned host relation");
      e->host_rel_bytes[r] = need;
    }
    if (!e->host_off[r])
      FI_CK(cudaHostAlloc((void **)&e->host_off[r], (size_t)e->C1 * e->F1 * 8,
                          cudaHostAllocDefault),
            "pinned host offsets");
  }
  e->launches = 0;
  e->mark(0, st);
  for (int r = 0; r < 2; ++r) {
    const uint64_t padded1 = lens[r] + (uint64_t)C * F1 * pad;
    // R's copy may still be running while S is partitioned: each relation
    // has its own pinned buffer
    std::vector<int> rcs(C, FI_OK);
    std::vector<std::thread> pool;
    pool.reserve(C);
    for (uint32_t c = 0; c < C; ++c)
      pool.emplace_back([&, c]() {
        fi_cpu_radix_partitioner *p = nullptr;
        int x = fi_cpu_radix_partitioner_new(FI_CPU_HISTOGRAM_CHUNKED,
                                             FI_CPU_PARTITION_SWWC, b1, &p);
        uint64_t *off = e->host_off[r] + (size_t)c * F1;
        if (!x)
          x = sizeof(K) == 4
                  ? fi_cpu_prefix_sum_int32(p, (const int32_t *)keys[r], lens[r], c, C, 0, off)
                  : fi_cpu_prefix_sum_int64(p, (const int64_t *)keys[r], lens[r], c, C, 0, off);
        if (!x)
          x = sizeof(K) == 4
                  ? fi_cpu_partition_int32(p, (const int32_t *)keys[r],
                                           (const int32_t *)pays[r], lens[r], c, C, 0,
                                           off, e->host_rel[r], padded1)
                  : fi_cpu_partition_int64(p, (const int64_t *)keys[r],
                                           (const int64_t *)pays[r], lens[r], c, C, 0,
                                           off, e->host_rel[r], padded1);
        fi_cpu_radix_partitioner_free(p);
        rcs[c] = x;
      });
    for (auto &t : pool) t.join();
    for (uint32_t c = 0; c < C; ++c)
      if (rcs[c]) return set_error(rcs[c], "CPU first pass of relation %d failed", r);
    e->mark(1 + 4 * r, st);
    FI_CK(cudaMemcpyAsync(e->off1[r].ptr, e->host_off[r], (size_t)C * F1 * 8,
                          cudaMemcpyHostToDevice, st),
          "offsets copy");
    FI_CK(cudaMemcpyAsync(e->rel1[r].ptr, e->host_rel[r],
                          (size_t)padded1 * sizeof(Tuple<K>), cudaMemcpyHostToDevice, st),
          "relation copy");
    e->mark(2 + 4 * r, st);
    rc = engine_pass2<K>(e, r, C, padded1, lens[r], st);
    if (rc) return rc;
    e->part_len[r] = lens[r];
  }
  e->built = true;
  rc = e->result_dev.reserve(sizeof(fi_join_result), false);
  if (rc) return rc;
  rc = engine_join<K>(e, (fi_join_result *)e->result_dev.ptr, st);
  if (rc) return rc;
  FI_CK(cudaMemcpyAsync(result, e->result_dev.ptr, sizeof(fi_join_result),
                        cudaMemcpyDeviceToHost, st),
        "result copy");
  FI_CK(cudaStreamSynchronize(st), "synchronize");
  return FI_OK;
}

extern "C" int fi_radix_join_engine_run_hybrid_int32(
    fi_radix_join_engine *e, const int32_t *build_key, const int32_t *build_pay,
    uint64_t build_len, const int32_t *probe_key, const int32_t *probe_pay,
    uint64_t probe_len, uint32_t threads, fi_join_result *result,
    fi_stream_t stream) {
  return engine_run_hybrid<int32_t>(e, build_key, build_pay, build_len, probe_key,
                                    probe_pay, probe_len, threads, result,
                                    (cudaStream_t)stream);
}
extern "C" int fi_radix_join_engine_run_hybrid_int64(
    fi_radix_join_engine *e, const int64_t *build_key, const int64_t *build_pay,
    uint64_t build_len, const int64_t *probe_key, const int64_t *probe_pay,
    uint64_t probe_len, uint32_t threads, fi_join_result *result,
    fi_stream_t stream) {
  return engine_run_hybrid<int64_t>(e, build_key, build_pay, build_len, probe_key,
                                    probe_pay, probe_len, threads, result,
                                    (cudaStream_t)stream);
}

extern "C" int fi_radix_join_engine_run_streamed_int32(
    fi_radix_join_engine *e, const int32_t *build_key, const int32_t *build_pay,
    uint64_t build_len, const int32_t *probe_key, const int32_t *probe_pay,
    uint64_t probe_len, uint64_t block_tuples, fi_join_result *result,
    fi_stream_t stream) {
  return engine_run_streamed<int32_t>(e, build_key, build_pay, build_len,
                                      probe_key, probe_pay, probe_len,
                                      block_tuples, result, (cudaStream_t)stream);
}
extern "C" int fi_radix_join_engine_run_streamed_int64(
    fi_radix_join_engine *e, const int64_t *build_key, const int64_t *build_pay,
    uint64_t build_len, const int64_t *probe_key, const int64_t *probe_pay,
    uint64_t probe_len, uint64_t block_tuples, fi_join_result *result,
    fi_stream_t stream) {
  return engine_run_streamed<int64_t>(e, build_key, build_pay, build_len,
                                      probe_key, probe_pay, probe_len,
                                      block_tuples, result, (cudaStream_t)stream);
}
