// Tile write-combining scatter fed by TMA bulk copies (sm_100a).
//
// Same algorithm as tile_scatter.cuh, but the next tile is brought into a
// shared-memory stage by the Tensor Memory Accelerator (cp.async.bulk, 1-D,
// completion tracked by an mbarrier) instead of into registers.  That frees
// ~60 registers per thread, so a CTA runs 1024 threads (32 warps per SM
// instead of 16) to hide the shared-memory latency of ranking and staging,
// and the loads of tile t+1 stay in flight for the whole of tile t.
//
// Each tile is sorted in place in its own stage (tuples held in registers
// across the scan), so two stages of 6144 int64 tuples fit where two stages
// plus a separate staging tile of 4096 did.  Measured on B200 (1024M x 1024M
// int64 join, 9+9 bits): pass-1 scatter 7.59 -> 6.96 ms and pass-2 scatter
// 8.13 -> 7.38 ms per relation against the 4096-tuple tiles with a staging
// tile; 7040-tuple tiles (the shared-memory limit) gave 6.92 ms.  Slower
// variants, measured: a two-barrier scan in which every thread sums the warp
// totals (-16%), a double-buffered tile histogram cleared during the
// write-out (-2%), two 512-thread CTAs per SM with 2048-tuple tiles (-28%:
// shorter runs per partition), TMA bulk stores of the runs (-12%), a second
// pass writing separate key and payload columns so that the join reads
// build keys only (second-pass scatter 8.1 -> 12.4 ms per relation for a
// join 0.1 ms faster: each run splits into two runs of half the bytes), two
// barriers fewer per tile (alternating tile histograms, per-run write
// offsets, one bounds check per run: -4%), and warp specialisation (16
// warps ranking and sorting tile t+1 while 16 write out tile t, three
// 4096-tuple buffers handed over by mbarriers: 7.58 and 7.81 ms, no gain:
// the sorting work, not the serialisation of the phases, bounds the SM),
// and an L2 bulk prefetch of tile t+2 issued with the copy of tile t+1
// (pass 1 6.97 -> 7.09 ms, pass 2 7.01 -> 7.30 ms: the loads were not late).
// An ablation on 2^30 int64 tuples (9 bits, 4096-tuple tiles) located the
// time: without the global stores 6.1 of 7.6 ms remain, without the
// write-out loop 5.1, without the staging 3.9.
//
// Requirements checked by the host before choosing this path: 16-byte
// aligned column/relation bases, tuples of 16 bytes for AoS sources, and a
// fanout small enough that the two stages fit shared memory.
// Every mbarrier wait is bounded; a wait that gives up records
// kDevErrTimeout, waits (bounded) for the copy it issued and returns.
#pragma once

#include "common.cuh"

namespace fi {

__device__ __forceinline__ uint32_t smem_u32(const void *p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ void mbar_init(uint64_t *bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)),
               "r"(count)
               : "memory");
}

__device__ __forceinline__ void mbar_fence_init() {
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t *bar,
                                                      uint32_t bytes) {
  asm volatile(
      "mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(
          smem_u32(bar)),
      "r"(bytes)
      : "memory");
}

// Global -> shared bulk copy of `bytes` (multiple of 16, both addresses
// 16-byte aligned), completing transaction bytes on `bar`.
__device__ __forceinline__ void bulk_g2s(void *dst, const void *src,
                                         uint32_t bytes, uint64_t *bar) {
  asm volatile(
      "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes "
      "[%0], [%1], %2, [%3];" ::"r"(smem_u32(dst)),
      "l"(src), "r"(bytes), "r"(smem_u32(bar))
      : "memory");
}

// Orders this thread's earlier generic-proxy shared-memory accesses before
// later async-proxy (TMA) accesses.
__device__ __forceinline__ void fence_proxy_async_smem() {
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint64_t *bar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n .reg .pred p;\n"
      " mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n"
      " selp.u32 %0, 1, 0, p;\n}"
      : "=r"(ok)
      : "r"(smem_u32(bar)), "r"(parity)
      : "memory");
  return ok != 0;
}

// Bounded wait for phase `parity` of `bar`; false when it gave up.
__device__ __forceinline__ bool mbar_wait(uint64_t *bar, uint32_t parity) {
  for (uint32_t i = 0; i < kSpinLimit; ++i) {
    if (mbar_try_wait(bar, parity)) return true;
    if (i > 8) __nanosleep(128);
  }
  return false;
}


// Bounded waits for the copies of tiles t and t+1 (if any), the ones a CTA
// may still have in flight when a wait gave up.  Out of line: inlined into
// the scatter, the error path made the second-pass kernel spill registers
// (4% slower).
template <uint32_t kStages>
__device__ __noinline__ void tma_drain(uint64_t *bars, uint64_t t, uint64_t ntiles) {
  const uint64_t last = t + 2 < ntiles ? t + 2 : ntiles;
  for (uint64_t tt = t; tt < last; ++tt)
    for (uint32_t round = 0;
         round < 4 && !mbar_wait(&bars[tt % kStages], (uint32_t)((tt / kStages) & 1u));
         ++round) {
    }
}

template <typename K>
struct TmaShape {
  static constexpr uint32_t kThreads = 1024;
  static constexpr uint32_t kItems = sizeof(K) == 8 ? 6 : 12;
  static constexpr uint32_t kTile = kThreads * kItems;
  static constexpr uint32_t kStages = 2;
};

// Bytes of one input stage.
template <typename K>
constexpr size_t tma_stage_bytes() {
  return (size_t)TmaShape<K>::kTile * 2 * sizeof(K);
}

// Shared memory: [bars (64 B)] [stages] [toff F+1] [cur F] [warp_tmp 33]
// (a tile is sorted in place in its own stage)
template <typename K>
size_t tma_scatter_smem(uint32_t F) {
  return 64 + TmaShape<K>::kStages * tma_stage_bytes<K>() +
         (size_t)(2 * F + 1 + 33) * sizeof(uint32_t);
}

// Column source: tile [t0, t0+n) of two columns -> stage {keys[kTile],
// pays[kTile]}.  The 16-byte multiple prefix comes by TMA, the rest (at most
// 16/sizeof(K)-1 tuples) by plain loads in get().
template <typename K>
struct TmaColumnSource {
  const K *__restrict__ keys;
  const K *__restrict__ pays;
  // thread 0: issue the copies of tile [t0, t0+n) into `stage`
  __device__ __forceinline__ void issue(uint64_t t0, uint32_t n, void *stage,
                                        uint64_t *bar) {
    const uint32_t bytes = (n * (uint32_t)sizeof(K)) & ~15u;
    K *sk = reinterpret_cast<K *>(stage);
    K *sp = sk + TmaShape<K>::kTile;
    mbar_arrive_expect_tx(bar, 2 * bytes);
    if (bytes) {
      bulk_g2s(sk, keys + t0, bytes, bar);
      bulk_g2s(sp, pays + t0, bytes, bar);
    }
  }
  __device__ __forceinline__ void get(const void *stage, uint64_t t0,
                                      uint32_t n, uint32_t i, K &k, K &v) const {
    const uint32_t n_tma = ((n * (uint32_t)sizeof(K)) & ~15u) / (uint32_t)sizeof(K);
    if (i < n_tma) {
      const K *sk = reinterpret_cast<const K *>(stage);
      k = sk[i];
      v = sk[TmaShape<K>::kTile + i];
    } else {
      k = load_cs(keys + t0 + i);
      v = load_cs(pays + t0 + i);
    }
  }
};

// Region source (16-byte tuples only): logical index i of a sequence made of
// regions of a tuple array (see RegionSource in tile_scatter.cuh).  Thread 0
// walks the regions of each tile and issues one bulk copy per segment.
template <typename K>
struct TmaRegionSource {
  static_assert(sizeof(Tuple<K>) == 16, "TMA region source needs 16-byte tuples");
  const Tuple<K> *__restrict__ tuples;
  const uint64_t *pre;    // [regions + 1], shared memory
  const uint64_t *begin;  // [regions], shared memory
  uint32_t regions;
  uint32_t r = 0;  // thread 0's current region
  __device__ __forceinline__ TmaRegionSource(const Tuple<K> *t, const uint64_t *p,
                                             const uint64_t *b, uint32_t n)
      : tuples(t), pre(p), begin(b), regions(n) {}
  __device__ __forceinline__ void issue(uint64_t t0, uint32_t n, void *stage,
                                        uint64_t *bar) {
    Tuple<K> *st = reinterpret_cast<Tuple<K> *>(stage);
    mbar_arrive_expect_tx(bar, n * 16u);
    uint64_t i = t0;
    const uint64_t e = t0 + n;
    while (i < e) {
      while (r + 1 < regions && pre[r + 1] <= i) ++r;
      const uint64_t seg_end = min(e, pre[r + 1]);
      const uint32_t cnt = (uint32_t)(seg_end - i);
      bulk_g2s(st + (i - t0), tuples + begin[r] + (i - pre[r]), cnt * 16u, bar);
      i = seg_end;
    }
  }
  __device__ __forceinline__ void get(const void *stage, uint64_t, uint32_t,
                                      uint32_t i, K &k, K &v) const {
    const Tuple<K> t = reinterpret_cast<const Tuple<K> *>(stage)[i];
    k = t.key;
    v = t.value;
  }
};

// Scatters logical src[begin, end) by partition: partition p's tuples go to
// out[cur_base + cur[p]], out[cur_base + cur[p] + 1], ...  Shared memory:
// `cur` (F u32, relative to cur_base), `toff` (tile histogram, F+1 u32, zero
// on entry and exit), `warp_tmp` (33 u32), `stages` (kStages input stages)
// and `bars` (one mbarrier per stage, initialised with count 1).  A tile is
// sorted in place: every thread holds its tuples in registers across the
// scan, then writes them back into the tile's own stage in partition order,
// so no separate staging buffer is needed and the stages can be 50% longer.
// Called once per barrier initialisation by all threads; thread 0 issues
// the copies.
// The partition of a key: its radix digit (key_to_partition).
template <typename K>
struct RadixDigit {
  uint64_t mask;
  uint32_t ignore_bits;
  __device__ __forceinline__ uint32_t operator()(K k) const {
    return key_to_partition(k, mask, ignore_bits);
  }
};

// The scatter for any partition function `part` (key -> [0, F)).
template <typename K, typename Src, typename Part, bool kUniformWarps = false>
__device__ __forceinline__ void tma_tile_scatter_by(
    Src &src, uint64_t begin, uint64_t end, uint32_t F, const Part part,
    uint32_t *cur, uint32_t *toff, uint32_t *warp_tmp,
    unsigned char *stages, uint64_t *bars, Tuple<K> *__restrict__ out,
    uint64_t cur_base, uint64_t out_len, int *status) {
  using S = TmaShape<K>;
  constexpr uint32_t T = S::kThreads, I = S::kItems, kTile = S::kTile;
  constexpr size_t kStageBytes = tma_stage_bytes<K>();
  const uint32_t tid = threadIdx.x;
  if (begin >= end) return;
  const uint64_t ntiles = (end - begin + kTile - 1) / kTile;

  if (tid == 0) {
    const uint32_t n0 = (uint32_t)min((uint64_t)kTile, end - begin);
    src.issue(begin, n0, stages, &bars[0]);
  }
  for (uint64_t t = 0; t < ntiles; ++t) {
    const uint32_t s = (uint32_t)(t % S::kStages);
    const uint32_t parity = (uint32_t)((t / S::kStages) & 1u);
    const uint64_t t0 = begin + t * kTile;
    const uint32_t n_valid = (uint32_t)min((uint64_t)kTile, end - t0);
    // prefetch the next tile into the other stage; tile t-1 finished with it
    // (every thread fenced its accesses before the last barrier of t-1)
    if (tid == 0 && t + 1 < ntiles) {
      const uint64_t t1 = t0 + kTile;
      const uint32_t s1 = (uint32_t)((t + 1) % S::kStages);
      fence_proxy_async_smem();
      src.issue(t1, (uint32_t)min((uint64_t)kTile, end - t1),
                stages + s1 * kStageBytes, &bars[s1]);
    }
    const bool ok = mbar_wait(&bars[s], parity);
    unsigned char *stage = stages + s * kStageBytes;

    // 1. rank every tuple inside its partition's run of the tile
    K ck[I], cv[I];
    uint32_t pp[I], rk[I];
#pragma unroll
    for (uint32_t u = 0; u < I; ++u) {
      const uint32_t i = u * T + tid;
      const bool act = ok && i < n_valid;
      if (act) src.get(stage, t0, n_valid, i, ck[u], cv[u]);
      pp[u] = act ? part(ck[u]) : 0u;
      rk[u] = kUniformWarps ? warp_uniform_rank(toff, pp[u], act)
                            : warp_aggregated_rank(toff, pp[u], act);
    }
    // barrier 1: every tuple of the stage is in registers; also the vote on
    // a wait that gave up
    if (__syncthreads_or(!ok)) {
      if (tid == 0) {
        record_error(status, kDevErrTimeout);
        // Drain before the CTA's shared memory is released: wait (bounded)
        // for both copies this CTA may still have in flight, tile t's (whose
        // wait gave up) and tile t+1's.  A copy that outlasts these waits as
        // well is reported by the timeout status above.
        tma_drain<S::kStages>(bars, t, ntiles);
      }
      __syncthreads();
      return;
    }
    // 2. run offsets inside the tile
    block_exclusive_scan_u32(toff, F, warp_tmp);
    // 3. write the tile back into its stage, sorted by partition
    Tuple<K> *staged = reinterpret_cast<Tuple<K> *>(stage);
#pragma unroll
    for (uint32_t u = 0; u < I; ++u)
      if (u * T + tid < n_valid) staged[toff[pp[u]] + rk[u]] = Tuple<K>{ck[u], cv[u]};
    __syncthreads();
    // 4. write the runs: tuple j of run p goes to cur[p] + (j - toff[p])
    for (uint32_t j = tid; j < n_valid; j += T) {
      const Tuple<K> tp = staged[j];
      const uint32_t p = part(tp.key);
      const uint64_t dst = cur_base + (uint32_t)(cur[p] + (j - toff[p]));
      if (dst < out_len)
        store_tuple(out + dst, tp);
      else
        record_error(status, kDevErrCapacity);
    }
    fence_proxy_async_smem();  // this stage's generic accesses before its refill
    __syncthreads();
    // 5. advance the cursors, then clear the tile histogram
    for (uint32_t p = tid; p < F; p += T) {
      const uint32_t next = (p + 1 < F) ? toff[p + 1] : n_valid;
      cur[p] += next - toff[p];
    }
    __syncthreads();
    for (uint32_t p = tid; p <= F; p += T) toff[p] = 0;
    __syncthreads();
  }
}

// The scatter by the radix digit (mask, ignore_bits).
template <typename K, typename Src, bool kUniformWarps = false>
__device__ __forceinline__ void tma_tile_scatter_range(
    Src &src, uint64_t begin, uint64_t end, uint32_t F, uint64_t mask,
    uint32_t ignore_bits, uint32_t *cur, uint32_t *toff, uint32_t *warp_tmp,
    unsigned char *stages, uint64_t *bars, Tuple<K> *__restrict__ out,
    uint64_t cur_base, uint64_t out_len, int *status) {
  tma_tile_scatter_by<K, Src, RadixDigit<K>, kUniformWarps>(
      src, begin, end, F, RadixDigit<K>{mask, ignore_bits}, cur, toff, warp_tmp,
      stages, bars, out, cur_base, out_len, status);
}

}  // namespace fi
