// Device-side vocabulary shared by all sm_100a kernels of the radix-partition
// and hash-join path.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

namespace fi {

// sql-ops/build.rs:46,58,72: ALIGN_BYTES, PADDING_BYTES and the bucket count
// of the reference's shared-memory bucket-chaining join.
constexpr uint32_t kAlignBytes = 128;
constexpr uint32_t kPaddingBytes = 128;
constexpr uint32_t kRefChainingBuckets = 2048;

constexpr uint32_t kWarp = 32;
constexpr uint32_t kFullMask = 0xffffffffu;

// Error codes a kernel can record in a device status word (same numbering as
// the C ABI's FI_ERR_*).
constexpr int kDevErrTimeout = -5;
constexpr int kDevErrCapacity = -7;

// Upper bound of polls for every device-side wait; with the nanosleep
// back-off below this is roughly two seconds.
constexpr uint32_t kSpinLimit = 1u << 21;

// Tuple<K, V> of the reference (sql-ops/include/gpu_common.h:48-103).  The
// alignment lets one 8- or 16-byte vector instruction move a whole tuple.
template <typename K>
struct alignas(2 * sizeof(K)) Tuple {
  K key;
  K value;
};

template <typename K>
__host__ __device__ constexpr K null_key() {
  return static_cast<K>(-1);
}

// key_to_partition (sql-ops/include/gpu_radix_partition.h:122-127): the key
// is widened to u64 (sign-extending int32, as static_cast<unsigned long long>
// does), masked and shifted; the result is truncated to u32.
template <typename K>
__device__ __forceinline__ uint32_t key_to_partition(K key, uint64_t mask,
                                                     uint32_t ignore_bits) {
  return static_cast<uint32_t>(
      (static_cast<uint64_t>(static_cast<int64_t>(key)) & mask) >> ignore_bits);
}

// Multiply-shift hash with Knuth's golden-ratio factor, the reference's
// default hash (sql-ops/include/gpu_common.h:144-168,216).  Requires
// log2_buckets >= 1.
template <typename K>
__device__ __forceinline__ uint32_t mult_shift_hash(K value,
                                                    uint32_t log2_buckets);
template <>
__device__ __forceinline__ uint32_t mult_shift_hash<int32_t>(
    int32_t value, uint32_t log2_buckets) {
  return (static_cast<uint32_t>(value) * 2654435769u) >> (32u - log2_buckets);
}
template <>
__device__ __forceinline__ uint32_t mult_shift_hash<int64_t>(
    int64_t value, uint32_t log2_buckets) {
  return static_cast<uint32_t>(
      (static_cast<uint64_t>(value) * 11400714819323198485ull) >>
      (64u - log2_buckets));
}

// ---- vector loads / stores of whole tuples --------------------------------
__device__ __forceinline__ Tuple<int64_t> load_tuple(const Tuple<int64_t> *p) {
  longlong2 v = *reinterpret_cast<const longlong2 *>(p);
  return {v.x, v.y};
}
__device__ __forceinline__ Tuple<int32_t> load_tuple(const Tuple<int32_t> *p) {
  int2 v = *reinterpret_cast<const int2 *>(p);
  return {v.x, v.y};
}
// Streaming (evict-first) variants for data read exactly once.
__device__ __forceinline__ Tuple<int64_t> load_tuple_cs(const Tuple<int64_t> *p) {
  longlong2 v = __ldcs(reinterpret_cast<const longlong2 *>(p));
  return {v.x, v.y};
}
__device__ __forceinline__ Tuple<int32_t> load_tuple_cs(const Tuple<int32_t> *p) {
  int2 v = __ldcs(reinterpret_cast<const int2 *>(p));
  return {v.x, v.y};
}
__device__ __forceinline__ void store_tuple(Tuple<int64_t> *p, Tuple<int64_t> t) {
  *reinterpret_cast<longlong2 *>(p) = make_longlong2(t.key, t.value);
}
__device__ __forceinline__ void store_tuple(Tuple<int32_t> *p, Tuple<int32_t> t) {
  *reinterpret_cast<int2 *>(p) = make_int2(t.key, t.value);
}

template <typename K>
__device__ __forceinline__ K load_cs(const K *p) {
  return __ldcs(p);
}

__device__ __forceinline__ uint32_t lane_id() { return threadIdx.x & 31u; }

__device__ __forceinline__ uint32_t lanemask_lt() {
  uint32_t m;
  asm("mov.u32 %0, %%lanemask_lt;" : "=r"(m));
  return m;
}

// Warp-aggregated shared-memory increment: lanes with equal `bin` are grouped
// with match.any, the lowest lane adds the group size, and every lane gets a
// distinct rank.  Lanes with active == false take no part (they return 0).
// This keeps heavily skewed keys (Zipf) from serialising on one counter.
//
// FI_WARP_AGGREGATE = 0 (the default) selects plain shared-memory atomics,
// one per lane.  Measured on B200 at 2^28 x 2^28 int64 tuples, plain atomics
// made the histograms and tile scatters ~1.8x faster than the match.any
// aggregation for uniform keys AND for Zipf(1.5) keys (38% of them equal):
// the shared-memory atomic unit resolves same-address lanes faster than the
// match instruction costs.
#ifndef FI_WARP_AGGREGATE
#define FI_WARP_AGGREGATE 0
#endif
__device__ __forceinline__ uint32_t warp_aggregated_rank(uint32_t *counters,
                                                         uint32_t bin,
                                                         bool active) {
#if !FI_WARP_AGGREGATE
  return active ? atomicAdd(&counters[bin], 1u) : 0u;
#endif
  const uint32_t act = __ballot_sync(kFullMask, active);
  uint32_t rank = 0;
  if (active) {
    const uint32_t peers = __match_any_sync(act, bin);
    const uint32_t leader = __ffs(peers) - 1;
    uint32_t base = 0;
    if (lane_id() == leader) base = atomicAdd(&counters[bin], __popc(peers));
    base = __shfl_sync(act, base, leader);
    rank = base + __popc(peers & lanemask_lt());
  }
  return rank;
}

// Rank with one shared atomic per warp when all 32 lanes are active and
// share one bin (a tile inside a Zipf-hot partition), else one per lane.
__device__ __forceinline__ uint32_t warp_uniform_rank(uint32_t *counters,
                                                      uint32_t bin, bool active) {
  const uint32_t b0 = __shfl_sync(kFullMask, bin, 0);
  if (__all_sync(kFullMask, active && bin == b0)) {
    uint32_t base = 0;
    if (lane_id() == 0) base = atomicAdd(&counters[bin], 32u);
    return __shfl_sync(kFullMask, base, 0) + lane_id();
  }
  return active ? atomicAdd(&counters[bin], 1u) : 0u;
}

// Same as warp_aggregated_rank without a result (histograms).
__device__ __forceinline__ void warp_aggregated_count(uint32_t *counters,
                                                      uint32_t bin,
                                                      bool active) {
#if !FI_WARP_AGGREGATE
  if (active) atomicAdd(&counters[bin], 1u);
  return;
#endif
  const uint32_t act = __ballot_sync(kFullMask, active);
  if (active) {
    const uint32_t peers = __match_any_sync(act, bin);
    if (lane_id() == __ffs(peers) - 1) atomicAdd(&counters[bin], __popc(peers));
  }
}

// ---- block-wide exclusive scan ------------------------------------------
// Exclusive scan over `n` u32 values in shared memory, in place; returns the
// total.  Every thread of the block must call it.  `warp_tmp` must hold 33
// u32.  Values are summed in u32 (callers keep totals below 2^32).
__device__ inline uint32_t block_exclusive_scan_u32(uint32_t *data, uint32_t n,
                                                    uint32_t *warp_tmp) {
  const uint32_t tid = threadIdx.x, nthreads = blockDim.x;
  const uint32_t per = (n + nthreads - 1) / nthreads;
  const uint32_t begin = min(n, tid * per), end = min(n, begin + per);
  uint32_t local = 0;
  for (uint32_t i = begin; i < end; ++i) local += data[i];
  // inclusive warp scan of the per-thread sums
  uint32_t x = local;
#pragma unroll
  for (uint32_t d = 1; d < 32; d <<= 1) {
    uint32_t y = __shfl_up_sync(kFullMask, x, d);
    if (lane_id() >= d) x += y;
  }
  const uint32_t warp = tid >> 5, nwarps = (nthreads + 31) >> 5;
  if (lane_id() == 31) warp_tmp[warp] = x;
  __syncthreads();
  if (warp == 0) {
    uint32_t w = lane_id() < nwarps ? warp_tmp[lane_id()] : 0u;
    uint32_t wi = w;
#pragma unroll
    for (uint32_t d = 1; d < 32; d <<= 1) {
      uint32_t y = __shfl_up_sync(kFullMask, wi, d);
      if (lane_id() >= d) wi += y;
    }
    if (lane_id() < nwarps) warp_tmp[lane_id()] = wi - w;  // exclusive
    if (lane_id() == 31) warp_tmp[32] = wi;                // total
  }
  __syncthreads();
  uint32_t run = warp_tmp[warp] + x - local;
  for (uint32_t i = begin; i < end; ++i) {
    uint32_t v = data[i];
    data[i] = run;
    run += v;
  }
  const uint32_t total = warp_tmp[32];
  __syncthreads();
  return total;
}

// 64-bit block reduction (sum); every thread must call it; `tmp` holds 32
// u64.  The result is valid in all threads.
__device__ inline uint64_t block_reduce_u64(uint64_t v, uint64_t *tmp) {
#pragma unroll
  for (uint32_t d = 16; d > 0; d >>= 1) v += __shfl_down_sync(kFullMask, v, d);
  const uint32_t warp = threadIdx.x >> 5, nwarps = (blockDim.x + 31) >> 5;
  __syncthreads();
  if (lane_id() == 0) tmp[warp] = v;
  __syncthreads();
  uint64_t s = 0;
  for (uint32_t w = 0; w < nwarps; ++w) s += tmp[w];
  __syncthreads();
  return s;
}

// Block-wide exclusive scan of one u64 per thread; returns the exclusive
// value, *total gets the block total.  tmp holds 33 u64.
__device__ inline uint64_t block_exclusive_scan_u64(uint64_t v, uint64_t *tmp,
                                             uint64_t *total) {
  uint64_t x = v;
#pragma unroll
  for (uint32_t d = 1; d < 32; d <<= 1) {
    uint64_t y = __shfl_up_sync(kFullMask, x, d);
    if (lane_id() >= d) x += y;
  }
  const uint32_t warp = threadIdx.x >> 5, nwarps = (blockDim.x + 31) >> 5;
  if (lane_id() == 31) tmp[warp] = x;
  __syncthreads();
  if (warp == 0) {
    uint64_t w = lane_id() < nwarps ? tmp[lane_id()] : 0ull;
    uint64_t wi = w;
#pragma unroll
    for (uint32_t d = 1; d < 32; d <<= 1) {
      uint64_t y = __shfl_up_sync(kFullMask, wi, d);
      if (lane_id() >= d) wi += y;
    }
    if (lane_id() < nwarps) tmp[lane_id()] = wi - w;
    if (lane_id() == 31) tmp[32] = wi;
  }
  __syncthreads();
  uint64_t r = tmp[warp] + x - v;
  *total = tmp[32];
  __syncthreads();
  return r;
}

// Records the first device-side error in a status word.
__device__ __forceinline__ void record_error(int *status, int code) {
  if (status) atomicCAS(status, 0, code);
}

// Bounded back-off for polling loops.
__device__ __forceinline__ void spin_pause(uint32_t iter) {
  __nanosleep(iter < 64 ? 32 : 1024);
}

}  // namespace fi
