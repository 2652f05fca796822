// No-partitioning hash join in device memory (sm_100a).
//
// Replaces gpu_ht_build_linearprobing_*, gpu_ht_probe_aggregate_linearprobing_*,
// gpu_ht_build[_selective]_perfect_* and gpu_ht_probe_aggregate_perfect_* of
// the reference (sql-ops/cudautils/no_partitioning_join.cu:39-379) with the
// same table layout (HtEntry = Tuple<K, K>, null key = all ones), the same
// multiply-shift hash and the same results:
//  * linear probing: insert at hash(key) mod 2^floor(log2(size)) by CAS on the
//    key (for int32 on the packed 8-byte entry), moving forward on collision;
//    a probe adds its payload for every matching slot until an empty slot;
//  * perfect: ht[key] = (key, value); a probe matches when ht[key].key == key.
// B200 specifics: whole entries are read with one 8/16-byte load, probe keys
// and payloads with evict-first loads, and keys outside [0, size) are skipped
// by the perfect scheme instead of addressing out of bounds.
//
// Measured on B200 (Blanas: 16M x 256M int64, 1184 x 256 threads), in input
// order: linear probing builds in 1.0 ms and probes in 11.1 ms (a
// 2^25-entry, 512 MB table: one random access per probe, far beyond the
// 126 MB L2), perfect hashing probes in 4.7 ms (16M + 1 entries); grouped by
// table region (below, the default), the linear-probing build takes 0.57 ms
// and the probe 4.2-4.5 ms, the perfect probe 3.2 ms.  In input order, four
// tuples per thread with their table loads issued together made it no
// faster (11.7 ms), nor did
// loading a window of 4 slots (64 B) per step instead of slot by slot (11.0
// ms): the probe is bound by the rate of random HBM accesses (about 30 G/s
// reach DRAM in both schemes), and the perfect table is faster because it is
// half the size, so twice as much of it stays in L2.  The table size
// matters more: the hash masks with 2^floor(log2(size)) (as the reference
// does), so a size that is not a power of two can fill the table to near
// 1 (Kim, 128e6 keys in 2^27 slots: 27 ms per probe against 5.8 ms in 2^28).
#include <algorithm>

#include "common.cuh"
#include "kernels.h"
#include "tma_scatter.cuh"

namespace fi {

__device__ __forceinline__ uint32_t log2_floor_u64(uint64_t x) {
  return 63u - (uint32_t)__clzll((long long)x);
}

// Every byte set to 0xff, like the reference's cuMemsetD32 of the null key
// (no_partitioning_join.rs:603-613): the int32 linear-probing insert compares
// the whole 8-byte entry with all ones.
template <typename K>
__global__ void ht_init_kernel(Tuple<K> *ht, uint64_t n) {
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n;
       i += (uint64_t)gridDim.x * blockDim.x)
    store_tuple(ht + i, Tuple<K>{null_key<K>(), null_key<K>()});
}

__device__ __forceinline__ void lp_insert(Tuple<int32_t> *ht, uint32_t lg,
                                          int32_t key, int32_t pay) {
  const uint64_t n = 1ull << lg, m = n - 1;
  uint64_t idx = lg ? mult_shift_hash<int32_t>(key, lg) : 0;
  const unsigned long long nul = 0xffffffffffffffffull;
  const unsigned long long entry =
      (static_cast<unsigned long long>(static_cast<uint32_t>(key))) |
      (static_cast<unsigned long long>(static_cast<uint32_t>(pay)) << 32);
  for (uint64_t i = 0; i < n; ++i, idx = (idx + 1) & m) {
    unsigned long long old =
        atomicCAS(reinterpret_cast<unsigned long long *>(ht + idx), nul, entry);
    if (old == nul) return;
  }
}

__device__ __forceinline__ void lp_insert(Tuple<int64_t> *ht, uint32_t lg,
                                          int64_t key, int64_t pay) {
  const uint64_t n = 1ull << lg, m = n - 1;
  uint64_t idx = lg ? mult_shift_hash<int64_t>(key, lg) : 0;
  const unsigned long long nul = 0xffffffffffffffffull;
  for (uint64_t i = 0; i < n; ++i, idx = (idx + 1) & m) {
    unsigned long long old = atomicCAS(
        reinterpret_cast<unsigned long long *>(&ht[idx].key), nul,
        static_cast<unsigned long long>(key));
    if (old == nul) {
      ht[idx].value = pay;
      return;
    }
  }
}

template <typename K>
__global__ void ht_build_lp_kernel(Tuple<K> *ht, uint64_t size,
                                   const K *__restrict__ key,
                                   const K *__restrict__ pay, uint64_t len) {
  const uint32_t lg = log2_floor_u64(size);
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < len;
       i += (uint64_t)gridDim.x * blockDim.x)
    lp_insert(ht, lg, load_cs(key + i), load_cs(pay + i));
}

template <typename K>
__global__ void ht_build_perfect_kernel(Tuple<K> *ht, uint64_t size,
                                        const K *__restrict__ key,
                                        const K *__restrict__ pay,
                                        uint64_t len, bool selective) {
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < len;
       i += (uint64_t)gridDim.x * blockDim.x) {
    const K k = load_cs(key + i);
    if (selective && k == null_key<K>()) continue;
    const uint64_t slot = static_cast<uint64_t>(static_cast<int64_t>(k));
    if (slot < size) store_tuple(ht + slot, Tuple<K>{k, load_cs(pay + i)});
  }
}

template <typename K>
__global__ void ht_probe_lp_kernel(const Tuple<K> *__restrict__ ht,
                                   uint64_t size, const K *__restrict__ key,
                                   const K *__restrict__ pay, uint64_t len,
                                   uint64_t *__restrict__ result) {
  const uint32_t lg = log2_floor_u64(size);
  const uint64_t n = 1ull << lg, m = n - 1;
  const uint64_t gid = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
  uint64_t sum = 0;
  for (uint64_t i = gid; i < len; i += (uint64_t)gridDim.x * blockDim.x) {
    const K k = load_cs(key + i);
    const K v = load_cs(pay + i);
    uint64_t idx = lg ? mult_shift_hash<K>(k, lg) : 0;
    for (uint64_t s = 0; s < n; ++s, idx = (idx + 1) & m) {
      const Tuple<K> e = load_tuple(ht + idx);
      if (e.key == k)
        sum += static_cast<uint64_t>(static_cast<int64_t>(v));
      else if (e.key == null_key<K>())
        break;
    }
  }
  result[gid] += sum;
}

template <typename K>
__global__ void ht_probe_perfect_kernel(const Tuple<K> *__restrict__ ht,
                                        uint64_t size,
                                        const K *__restrict__ key,
                                        const K *__restrict__ pay,
                                        uint64_t len,
                                        uint64_t *__restrict__ result) {
  const uint64_t gid = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
  uint64_t sum = 0;
  for (uint64_t i = gid; i < len; i += (uint64_t)gridDim.x * blockDim.x) {
    const K k = load_cs(key + i);
    const uint64_t slot = static_cast<uint64_t>(static_cast<int64_t>(k));
    if (slot < size && ht[slot].key == k)
      sum += static_cast<uint64_t>(static_cast<int64_t>(load_cs(pay + i)));
  }
  result[gid] += sum;
}

// ---- region-ordered probing and building ---------------------------------
// A table far larger than L2 is probed at random: every probe reaches HBM
// (Blanas, 2^25 int64 slots: 24 G probes/s, 11 ms).  Grouping the probe
// tuples by the table region their first slot lies in (the top region_bits
// bits of the slot) and probing group by group keeps the active region
// (a few MB) in L2, so the table is read from HBM about once per slice.  The
// grouping is one streamed pass: per-(chunk, region) counts, their scan, and
// the TMA tile scatter of tma_scatter.cuh by region into a scratch buffer
// (one chunk per SM; a per-tile variant with one global claim per (tile,
// region) run serves columns that are not 16-byte aligned).  The sum does
// not depend on the order.  The build side is grouped the same way, and its
// inserts take tiles in order, so the table lines they write stay in L2
// until their region is done.  A heavily skewed probe slice is left in
// input order (region_chunk_scan_kernel).  Measured on B200, per 128M int64
// probes into a 512 MB table: counts 0.23 ms, scatter 0.92 ms (0.71 of the
// copy peak; 1.42 ms with the per-tile claims), probe 1.12 ms (32-byte
// windows; 1.17 ms slot by slot).

// Slot of a probe's first access: the hash (linear probing) or the key
// (perfect; keys outside [0, size) probe nothing and go to the last region).
template <typename K>
__device__ __forceinline__ uint32_t probe_region(K key, int scheme, uint32_t lg,
                                                 uint64_t size, uint32_t shift,
                                                 uint32_t regions) {
  uint64_t slot;
  if (scheme == 1) {
    slot = lg ? mult_shift_hash<K>(key, lg) : 0;
  } else {
    slot = static_cast<uint64_t>(static_cast<int64_t>(key));
    if (slot >= size) return regions - 1;
  }
  const uint64_t r = slot >> shift;
  return r < regions ? (uint32_t)r : regions - 1;
}

constexpr uint32_t kRegionThreads = 512;
constexpr uint32_t kRegionItems = 8;
constexpr uint32_t kRegionTile = kRegionThreads * kRegionItems;

// Region counts.  With few regions every warp counts into its own copy of
// the counters (copies = warps; one copy for more than kPrivateRegions
// regions), so 512 threads do not all collide on a few shared counters;
// four keys per thread are loaded before they are counted.
constexpr uint32_t kPrivateRegions = 256;

template <typename K>
__global__ void __launch_bounds__(kRegionThreads)
    region_histogram_kernel(const K *__restrict__ key, uint64_t len, int scheme,
                            uint32_t lg, uint64_t size, uint32_t shift,
                            uint32_t regions, uint32_t copies,
                            uint32_t *__restrict__ counts) {
  extern __shared__ uint32_t rh[];  // [copies][regions]
  for (uint32_t r = threadIdx.x; r < regions * copies; r += blockDim.x) rh[r] = 0;
  __syncthreads();
  uint32_t *mine = rh + (copies > 1 ? (threadIdx.x >> 5) * regions : 0);
  const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
  for (uint64_t b = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; b < len;
       b += 4 * stride) {
    K k[4];
#pragma unroll
    for (uint32_t u = 0; u < 4; ++u)
      if (b + u * stride < len) k[u] = load_cs(key + b + u * stride);
#pragma unroll
    for (uint32_t u = 0; u < 4; ++u)
      if (b + u * stride < len)
        atomicAdd(&mine[probe_region(k[u], scheme, lg, size, shift, regions)], 1u);
  }
  __syncthreads();
  for (uint32_t r = threadIdx.x; r < regions; r += blockDim.x) {
    uint32_t c = 0;
    for (uint32_t w = 0; w < copies; ++w) c += rh[w * regions + r];
    if (c) atomicAdd(&counts[r], c);
  }
}

// One CTA: exclusive scan of the region counts into the claim cursors.
__global__ void __launch_bounds__(1024)
    region_scan_kernel(const uint32_t *__restrict__ counts, uint32_t regions,
                       uint32_t *__restrict__ cursors) {
  extern __shared__ uint32_t rs[];  // [regions] + 33
  for (uint32_t r = threadIdx.x; r < regions; r += blockDim.x) rs[r] = counts[r];
  __syncthreads();
  block_exclusive_scan_u32(rs, regions, rs + regions);
  for (uint32_t r = threadIdx.x; r < regions; r += blockDim.x) cursors[r] = rs[r];
}

// Tiles of the probe columns sorted by region in shared memory; each
// (tile, region) run claims its slots with one global atomic and is stored
// as consecutive tuples.  Shared memory: staged [kRegionTile] tuples |
// toff [regions + 1] | gbase [regions] | scan_tmp [33].
template <typename K>
__global__ void __launch_bounds__(kRegionThreads)
    region_scatter_kernel(const K *__restrict__ key, const K *__restrict__ pay,
                          uint64_t len, int scheme, uint32_t lg, uint64_t size,
                          uint32_t shift, uint32_t regions,
                          uint32_t *__restrict__ cursors,
                          Tuple<K> *__restrict__ out) {
  extern __shared__ __align__(16) unsigned char rsm[];
  Tuple<K> *staged = reinterpret_cast<Tuple<K> *>(rsm);
  uint32_t *toff = reinterpret_cast<uint32_t *>(staged + kRegionTile);
  uint32_t *gbase = toff + regions + 1;
  uint32_t *scan_tmp = gbase + regions;
  const uint32_t tid = threadIdx.x;
  for (uint32_t r = tid; r <= regions; r += blockDim.x) toff[r] = 0;
  for (uint64_t t0 = (uint64_t)blockIdx.x * kRegionTile; t0 < len;
       t0 += (uint64_t)gridDim.x * kRegionTile) {
    const uint32_t n = (uint32_t)min((uint64_t)kRegionTile, len - t0);
    K k[kRegionItems], v[kRegionItems];
    uint32_t rg[kRegionItems], rk[kRegionItems];
    __syncthreads();  // the previous tile's write-out is done with toff
#pragma unroll
    for (uint32_t u = 0; u < kRegionItems; ++u) {
      const uint32_t j = u * kRegionThreads + tid;
      const bool act = j < n;
      if (act) {
        k[u] = load_cs(key + t0 + j);
        v[u] = load_cs(pay + t0 + j);
      }
      rg[u] = act ? probe_region(k[u], scheme, lg, size, shift, regions) : 0u;
      // lanes of a warp with the same region take one shared atomic: with
      // tens of regions most of a warp's lanes share a few counters
      const uint32_t am = __ballot_sync(kFullMask, act);
      rk[u] = 0;
      if (act) {
        const uint32_t peers = __match_any_sync(am, rg[u]);
        const uint32_t leader = __ffs(peers) - 1;
        uint32_t base = 0;
        if (lane_id() == leader) base = atomicAdd(&toff[rg[u]], __popc(peers));
        rk[u] = __shfl_sync(am, base, leader) + __popc(peers & lanemask_lt());
      }
    }
    __syncthreads();
    block_exclusive_scan_u32(toff, regions, scan_tmp);
    if (tid == 0) toff[regions] = n;
    __syncthreads();
    for (uint32_t r = tid; r < regions; r += blockDim.x) {
      const uint32_t c = toff[r + 1] - toff[r];
      if (c) gbase[r] = atomicAdd(&cursors[r], c);
    }
#pragma unroll
    for (uint32_t u = 0; u < kRegionItems; ++u)
      if (u * kRegionThreads + tid < n) staged[toff[rg[u]] + rk[u]] = Tuple<K>{k[u], v[u]};
    __syncthreads();
    for (uint32_t j = tid; j < n; j += blockDim.x) {
      const Tuple<K> t = staged[j];
      const uint32_t r = probe_region(t.key, scheme, lg, size, shift, regions);
      store_tuple(out + gbase[r] + (j - toff[r]), t);
    }
    __syncthreads();
    for (uint32_t r = tid; r <= regions; r += blockDim.x) toff[r] = 0;
  }
}

// The same grouping in chunks, without global atomics in the scatter: every
// CTA of the TMA tile scatter (tma_scatter.cuh) owns one contiguous chunk of
// the slice and writes its run of each region at a cursor fixed by a
// per-(chunk, region) histogram.  The output is region-major (region r holds
// chunk 0's tuples of r, then chunk 1's, ...).
// Region of a key's first slot (probe_region), one functor per scheme so
// that the scatter keeps few values live.  Linear probing: the top
// region_bits bits of the multiply-shift product, which are the top bits of
// the lg-bit hash (region_bits <= lg).  Perfect: the key's slot >> shift,
// keys outside [0, size) in the last region.
template <typename K>
struct LinearRegion {
  uint32_t bits;
  __device__ __forceinline__ uint32_t operator()(K k) const {
    return mult_shift_hash<K>(k, bits);
  }
};
template <typename K>
struct PerfectRegion {
  uint64_t size;
  uint32_t shift, regions;
  __device__ __forceinline__ uint32_t operator()(K k) const {
    const uint64_t slot = static_cast<uint64_t>(static_cast<int64_t>(k));
    if (slot >= size) return regions - 1;
    const uint64_t r = slot >> shift;
    return r < regions ? (uint32_t)r : regions - 1;
  }
};

// Per-(chunk, region) counts into counts[chunk][regions] (zero on entry);
// `per_chunk` CTAs share a chunk, four loads per thread in flight.
template <typename K, typename Part>
__global__ void __launch_bounds__(kRegionThreads)
    region_chunk_histogram_kernel(const K *__restrict__ key, uint64_t len,
                                  uint64_t clen, uint32_t chunks,
                                  uint32_t per_chunk, Part part, uint32_t regions,
                                  uint32_t copies, uint32_t *__restrict__ counts) {
  extern __shared__ uint32_t rh[];  // [copies][regions]
  for (uint32_t r = threadIdx.x; r < regions * copies; r += blockDim.x) rh[r] = 0;
  __syncthreads();
  const uint32_t c = blockIdx.x / per_chunk, sub = blockIdx.x % per_chunk;
  const uint64_t cb = clen * c, ce = (c + 1 == chunks) ? len : cb + clen;
  uint32_t *mine = rh + (copies > 1 ? (threadIdx.x >> 5) * regions : 0);
  const uint64_t stride = (uint64_t)per_chunk * blockDim.x;
  for (uint64_t b = cb + (uint64_t)sub * blockDim.x + threadIdx.x; b < ce;
       b += 4 * stride) {
    K k[4];
#pragma unroll
    for (uint32_t u = 0; u < 4; ++u)
      if (b + u * stride < ce) k[u] = load_cs(key + b + u * stride);
#pragma unroll
    for (uint32_t u = 0; u < 4; ++u)
      if (b + u * stride < ce) atomicAdd(&mine[part(k[u])], 1u);
  }
  __syncthreads();
  for (uint32_t r = threadIdx.x; r < regions; r += blockDim.x) {
    uint32_t t = 0;
    for (uint32_t w = 0; w < copies; ++w) t += rh[w * regions + r];
    if (t) atomicAdd(&counts[(uint64_t)c * regions + r], t);
  }
}

// One CTA: cursors[c][r] = (tuples of regions < r) + (tuples of region r in
// chunks < c), the region-major start of chunk c's run of region r.
// With `skip` set, a slice whose largest region holds more than a quarter
// of its tuples is not grouped: *skip = 1 tells the scatter and the probe
// to use input order (such skew already concentrates the probes on a few
// table lines; measured on 256M int64 Zipf(1.5) probes: 3.80 ms grouped,
// 1.31 ms in input order; Zipf(1.0), whose largest region holds ~8%, is
// faster grouped: 4.15 against 6.73 ms).
__global__ void __launch_bounds__(1024)
    region_chunk_scan_kernel(const uint32_t *__restrict__ counts, uint32_t chunks,
                             uint32_t regions, uint64_t *__restrict__ cursors,
                             uint64_t n, uint32_t *skip) {
  extern __shared__ uint32_t tot[];  // [regions] + 33
  __shared__ uint32_t biggest;
  if (threadIdx.x == 0) biggest = 0;
  __syncthreads();
  for (uint32_t r = threadIdx.x; r < regions; r += blockDim.x) {
    uint32_t t = 0;
    for (uint32_t c = 0; c < chunks; ++c) t += counts[(uint64_t)c * regions + r];
    tot[r] = t;
    atomicMax(&biggest, t);
  }
  __syncthreads();
  if (skip && threadIdx.x == 0) *skip = (uint64_t)biggest * 4 > n ? 1u : 0u;
  block_exclusive_scan_u32(tot, regions, tot + regions);
  for (uint32_t r = threadIdx.x; r < regions; r += blockDim.x) {
    uint64_t run = tot[r];
    for (uint32_t c = 0; c < chunks; ++c) {
      cursors[(uint64_t)c * regions + r] = run;
      run += counts[(uint64_t)c * regions + r];
    }
  }
}

// The TMA tile scatter of chunk blockIdx.x by region.  Shared memory as
// tma_tile_scatter_kernel's: bars | stages | toff | cur | scan_tmp.
template <typename K, typename Part>
__global__ void __launch_bounds__(TmaShape<K>::kThreads, 1)
    region_tma_scatter_kernel(const K *__restrict__ keys, const K *__restrict__ pays,
                              uint64_t len, uint64_t clen, uint32_t chunks,
                              Part part, uint32_t F,
                              const uint64_t *__restrict__ cursors,
                              Tuple<K> *__restrict__ out, uint64_t out_len,
                              int *status, const uint32_t *skip) {
  using S = TmaShape<K>;
  if (skip && *skip) return;  // the slice stays in input order
  extern __shared__ __align__(16) unsigned char smem_raw[];
  uint64_t *bars = reinterpret_cast<uint64_t *>(smem_raw);
  unsigned char *stages = smem_raw + 64;
  uint32_t *toff =
      reinterpret_cast<uint32_t *>(stages + S::kStages * tma_stage_bytes<K>());
  uint32_t *cur = toff + F + 1;
  uint32_t *scan_tmp = cur + F;
  const uint32_t c = blockIdx.x;
  const uint64_t cb = clen * c, ce = (c + 1 == chunks) ? len : cb + clen;
  // region-major cursors never lie below the chunk's run of region 0
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
  tma_tile_scatter_by<K, TmaColumnSource<K>, Part>(
      src, cb, ce, F, part, cur, toff, scan_tmp, stages, bars, out, base, out_len,
      status);
}

// The probes of a grouped slice, in order: every probe as in
// ht_probe_{lp,perfect}_kernel.  With the region in L2, the probe is bound
// by the L1's one request per uncoalesced load, so linear probing reads the
// table in 32-byte aligned windows (2 int64 or 4 int32 entries) with one
// 256-bit load each, instead of slot by slot; a window starts at the hash
// slot's window and the scan still ends at the first empty slot or after
// 2^lg slots.  (Four probes per thread with their first loads issued
// together measured slower, 1.17 -> 1.34 ms per 128M int64 probes: 52
// registers halve the resident threads.)
__device__ __forceinline__ void load_window32(const void *p, unsigned long long &a,
                                              unsigned long long &b,
                                              unsigned long long &c,
                                              unsigned long long &d) {
  asm volatile("ld.global.v4.u64 {%0, %1, %2, %3}, [%4];"
               : "=l"(a), "=l"(b), "=l"(c), "=l"(d)
               : "l"(p));
}

// Entry i of a 32-byte window held as four u64 words.
template <typename K>
struct Window32;
template <>
struct Window32<int64_t> {
  static constexpr uint32_t kSlots = 2;
  unsigned long long w[4];
  __device__ __forceinline__ int64_t key(uint32_t i) const {
    return static_cast<int64_t>(i == 0 ? w[0] : w[2]);
  }
};
template <>
struct Window32<int32_t> {
  static constexpr uint32_t kSlots = 4;
  unsigned long long w[4];
  __device__ __forceinline__ int32_t key(uint32_t i) const {
    const unsigned long long e = i == 0 ? w[0] : i == 1 ? w[1] : i == 2 ? w[2] : w[3];
    return static_cast<int32_t>(static_cast<uint32_t>(e));  // key: low half
  }
};

// kWindowed: the table base is 32-byte aligned (else slot by slot, W = 1).
constexpr uint32_t kProbeThreads = 256;

template <typename K, bool kWindowed>
__global__ void ht_probe_grouped_kernel(const Tuple<K> *__restrict__ ht,
                                        uint64_t size, int scheme,
                                        const Tuple<K> *__restrict__ probes,
                                        const K *__restrict__ key,
                                        const K *__restrict__ pay,
                                        const uint32_t *skip, uint64_t len,
                                        uint64_t *__restrict__ result,
                                        uint64_t result_len) {
  // a skewed slice was left in input order: probe the columns instead
  const bool in_order = *skip != 0;
  using Win = Window32<K>;
  constexpr uint32_t W = kWindowed ? Win::kSlots : 1;
  const uint32_t lg = log2_floor_u64(size);
  const uint64_t n = 1ull << lg, m = n - 1;
  const uint64_t gid = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
  uint64_t sum = 0;
  for (uint64_t i = gid; i < len; i += (uint64_t)gridDim.x * blockDim.x) {
    Tuple<K> p;
    if (in_order) {
      p.key = load_cs(key + i);
      p.value = load_cs(pay + i);
    } else {
      p = load_tuple_cs(probes + i);
    }
    const uint64_t v = static_cast<uint64_t>(static_cast<int64_t>(p.value));
    if (scheme == 1) {
      const uint64_t idx = mult_shift_hash<K>(p.key, lg);  // lg >= W here
      uint64_t w = idx & ~(uint64_t)(W - 1);
      // slots of the first window before the hash slot are not scanned
      uint32_t valid = ((1u << W) - 1) & ~((1u << (uint32_t)(idx - w)) - 1);
      uint64_t left = n;
      // a probe of the null key matches every empty slot and never stops
      // early (as in the slot-by-slot loop)
      const bool stop_on_null = p.key != null_key<K>();
      for (;;) {
        Win win;
        if (kWindowed)
          load_window32(ht + w, win.w[0], win.w[1], win.w[2], win.w[3]);
        uint32_t match = 0, empty = 0;
#pragma unroll
        for (uint32_t s = 0; s < W; ++s) {
          const K k = kWindowed ? win.key(s) : ht[w].key;
          match |= (uint32_t)(k == p.key) << s;
          empty |= (uint32_t)(k == null_key<K>()) << s;
        }
        const uint32_t cnt = (uint32_t)__popc(valid);
        if (left <= cnt) {  // the scan ends inside this window: n slots
          uint32_t keep = valid, c = (uint32_t)left;
          while (__popc(keep) > (int)c) keep &= ~(1u << (31 - __clz(keep)));
          valid = keep;
        }
        const uint32_t stop = stop_on_null ? (empty & valid) : 0u;
        if (stop) {
          const uint32_t before = (stop & (0u - stop)) - 1;  // below the first empty slot
          sum += v * (uint64_t)__popc(match & valid & before);
          break;
        }
        sum += v * (uint64_t)__popc(match & valid);
        if (left <= cnt) break;
        left -= cnt;
        w = (w + W) & m;
        valid = (1u << W) - 1;
      }
    } else {
      const uint64_t slot = static_cast<uint64_t>(static_cast<int64_t>(p.key));
      if (slot < size && ht[slot].key == p.key) sum += v;
    }
  }
  // the library's own grid: thread sums land modulo the caller's
  // grid * block entries of result_set, whose total is the join's sum
  if (sum)
    atomicAdd(reinterpret_cast<unsigned long long *>(result + gid % result_len),
              static_cast<unsigned long long>(sum));
}

// Region bits of a table: regions of at most kRegionBytes; 0 when the whole
// table fits kRegionBytes (then the probe needs no grouping).
#ifndef FI_REGION_MB
#define FI_REGION_MB 8
#endif
constexpr uint64_t kRegionBytes = (uint64_t)FI_REGION_MB << 20;
constexpr uint32_t kMaxRegionBits = 12;

uint32_t ht_region_bits(uint64_t size, uint32_t entry_bytes) {
  uint32_t lg = 63u - (uint32_t)__builtin_clzll(size);
  uint64_t slots = 1ull << lg;
  uint32_t b = 0;
  while (b < kMaxRegionBits && b < lg && (slots >> b) * entry_bytes > kRegionBytes) ++b;
  return b;
}

// Region scratch: [status: one int, padded to kRegionStatusWords u32]
// [counts: chunks x regions u32] [cursors: chunks x regions u64], with
// chunks = the SM count (at most kMaxRegionChunks).  The status sits at the
// start, so it stays in place whatever region count later calls use.  The
// per-tile path uses 2 x regions u32 after the status.
size_t ht_region_scratch_bytes(uint32_t region_bits) {
  return kRegionStatusWords * sizeof(uint32_t) +
         ((size_t)kMaxRegionChunks << region_bits) * (sizeof(uint32_t) + sizeof(uint64_t));
}

// The chunked grouping (TMA path) by region function `part`: per-(chunk,
// region) counts, their region-major scan, the TMA tile scatter.
template <typename K, typename Part>
static cudaError_t group_chunked(Part part, const K *key, const K *pay, uint64_t n,
                                 uint32_t region_bits, Tuple<K> *out,
                                 uint32_t *region_scratch, uint32_t chunks,
                                 uint32_t *skip, cudaStream_t stream) {
  const uint32_t regions = 1u << region_bits;
  const size_t tma_sm = tma_scatter_smem<K>(regions);
  int *status = reinterpret_cast<int *>(region_scratch);
  uint32_t *counts = region_scratch + kRegionStatusWords;
  uint64_t *cursors = reinterpret_cast<uint64_t *>(
      counts + ((size_t)kMaxRegionChunks << region_bits));
  // chunk starts on 128-byte boundaries; the last chunk takes the rest
  constexpr uint64_t kAlignMask = ~((uint64_t)(kAlignBytes / sizeof(K)) - 1ull);
  const uint64_t clen = ((n + chunks - 1) / chunks) & kAlignMask;
  cudaError_t e = cudaFuncSetAttribute((const void *)region_tma_scatter_kernel<K, Part>,
                                       cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       (int)tma_sm);
  if (e != cudaSuccess) return e;
  e = cudaMemsetAsync(counts, 0, (size_t)chunks * regions * sizeof(uint32_t), stream);
  if (e != cudaSuccess) return e;
  const uint32_t copies = regions <= kPrivateRegions ? kRegionThreads / 32 : 1;
  const uint32_t per_chunk = 2;
  region_chunk_histogram_kernel<K, Part><<<chunks * per_chunk, kRegionThreads,
                                           (size_t)regions * copies * sizeof(uint32_t),
                                           stream>>>(key, n, clen, chunks, per_chunk,
                                                     part, regions, copies, counts);
  region_chunk_scan_kernel<<<1, 1024, (regions + 33) * sizeof(uint32_t), stream>>>(
      counts, chunks, regions, cursors, n, skip);
  region_tma_scatter_kernel<K, Part><<<chunks, TmaShape<K>::kThreads, tma_sm, stream>>>(
      key, pay, n, clen, chunks, part, regions, cursors, out, n, status, skip);
  return cudaGetLastError();
}

// Groups tuples [0, n) of the two columns by table region into `out`
// (region order; the order inside a region is the order in which tiles claim
// their runs): region counts, their scan, and the tile scatter.
template <typename K>
static cudaError_t group_by_region(int scheme, uint64_t ht_size, const K *key,
                                   const K *pay, uint64_t n, uint32_t region_bits,
                                   Tuple<K> *out, uint32_t *region_scratch,
                                   uint32_t sm_count, uint32_t *skip,
                                   cudaStream_t stream) {
  const uint32_t lg = 63u - (uint32_t)__builtin_clzll(ht_size);
  const uint32_t regions = 1u << region_bits;
  // linear probing: regions of the hash range 2^lg; perfect: of the key
  // range [0, size), rounded up to a power of two
  uint32_t range_bits = lg;
  if (scheme != 1 && (1ull << lg) < ht_size) ++range_bits;
  const uint32_t shift = range_bits > region_bits ? range_bits - region_bits : 0;
  // chunked TMA path: 16-byte aligned columns, the scatter's shared memory
  // within the opt-in limit, one chunk per SM
  const size_t tma_sm = tma_scatter_smem<K>(regions);
  const uint32_t chunks = std::min<uint32_t>(sm_count, kMaxRegionChunks);
  if (((reinterpret_cast<uintptr_t>(key) | reinterpret_cast<uintptr_t>(pay)) % 16) == 0 &&
      tma_sm <= (size_t)device_max_smem_optin() && chunks > 0) {
    if (scheme == 1)
      return group_chunked<K>(LinearRegion<K>{region_bits}, key, pay, n, region_bits,
                              out, region_scratch, chunks, skip, stream);
    return group_chunked<K>(PerfectRegion<K>{ht_size, shift, regions}, key, pay, n,
                            region_bits, out, region_scratch, chunks, skip, stream);
  }
  // the per-tile path always groups
  if (skip) {
    cudaError_t e = cudaMemsetAsync(skip, 0, sizeof(uint32_t), stream);
    if (e != cudaSuccess) return e;
  }
  uint32_t *counts = region_scratch + kRegionStatusWords, *cursors = counts + regions;
  const size_t scatter_smem = (size_t)kRegionTile * sizeof(Tuple<K>) +
                              ((size_t)2 * regions + 1 + 33) * sizeof(uint32_t);
  cudaError_t e = cudaFuncSetAttribute((const void *)region_scatter_kernel<K>,
                                       cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       (int)scatter_smem);
  if (e != cudaSuccess) return e;
  e = cudaMemsetAsync(counts, 0, regions * sizeof(uint32_t), stream);
  if (e != cudaSuccess) return e;
  const uint32_t copies = regions <= kPrivateRegions ? kRegionThreads / 32 : 1;
  region_histogram_kernel<K><<<2 * sm_count, kRegionThreads,
                               (size_t)regions * copies * sizeof(uint32_t), stream>>>(
      key, n, scheme, lg, ht_size, shift, regions, copies, counts);
  region_scan_kernel<<<1, 1024, (regions + 33) * sizeof(uint32_t), stream>>>(
      counts, regions, cursors);
  region_scatter_kernel<K><<<2 * sm_count, kRegionThreads, scatter_smem, stream>>>(
      key, pay, n, scheme, lg, ht_size, shift, regions, cursors, out);
  return cudaGetLastError();
}

template <typename K>
cudaError_t launch_ht_probe_grouped(int scheme, const void *ht, uint64_t ht_size,
                                    const K *key, const K *pay, uint64_t len,
                                    uint64_t *result, uint32_t grid, uint32_t block,
                                    uint32_t region_bits, void *tuples,
                                    uint32_t *region_scratch, uint64_t slice,
                                    uint32_t sm_count, cudaStream_t stream) {
  Tuple<K> *out = static_cast<Tuple<K> *>(tuples);
  uint32_t *skip = region_scratch + 2;  // after the status and the build's counter
  // The library's launch shape, whatever the caller's probe grid: probes
  // served from L2 need every SM full of warps to hide its latency (the
  // caller's grid * block still sizes result_set).
  int per_sm = 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(
          &per_sm, (const void *)ht_probe_grouped_kernel<K, true>,
          (int)kProbeThreads, 0) != cudaSuccess ||
      per_sm < 1)
    per_sm = 1;
  const uint32_t probe_grid = (uint32_t)per_sm * sm_count;
  const uint64_t result_len = (uint64_t)grid * block;
  for (uint64_t s0 = 0; s0 < len; s0 += slice) {
    const uint64_t n = min(slice, len - s0);
    cudaError_t e = group_by_region<K>(scheme, ht_size, key + s0, pay + s0, n,
                                       region_bits, out, region_scratch, sm_count,
                                       skip, stream);
    if (e != cudaSuccess) return e;
    if (reinterpret_cast<uintptr_t>(ht) % 32 == 0)
      ht_probe_grouped_kernel<K, true><<<probe_grid, kProbeThreads, 0, stream>>>(
          static_cast<const Tuple<K> *>(ht), ht_size, scheme, out, key + s0,
          pay + s0, skip, n, result, result_len);
    else
      ht_probe_grouped_kernel<K, false><<<probe_grid, kProbeThreads, 0, stream>>>(
          static_cast<const Tuple<K> *>(ht), ht_size, scheme, out, key + s0,
          pay + s0, skip, n, result, result_len);
    e = cudaGetLastError();
    if (e != cudaSuccess) return e;
  }
  return cudaSuccess;
}

// Inserts of a grouped slice, in order: every insert as in
// ht_build_{lp,perfect}_kernel.  The CTAs take tiles of the slice in order
// from a global counter, so the inserts in flight stay within one or two
// regions and the lines they write stay in L2 until the region is done (in
// a grid-stride loop the warps drift apart over hundreds of iterations,
// and a profile of Kim's 128e6 int32 inserts showed an L2 hit rate of 12%
// and every table line read three times from HBM: 7.0 GB read for 3 GB of
// table and tuples, 4.0 ms).  Each thread issues the first CAS of its
// kBuildItems inserts together, then follows the collisions one by one.
constexpr uint32_t kBuildThreads = 256;
constexpr uint32_t kBuildItems = 4;
constexpr uint32_t kBuildTile = kBuildThreads * kBuildItems;

__device__ __forceinline__ unsigned long long lp_entry(int32_t key, int32_t pay) {
  return (static_cast<unsigned long long>(static_cast<uint32_t>(key))) |
         (static_cast<unsigned long long>(static_cast<uint32_t>(pay)) << 32);
}

// First insert attempt at slot idx: CAS of the packed entry (int32) or of
// the key (int64); returns the old word (the null word on success).
__device__ __forceinline__ unsigned long long lp_try(Tuple<int32_t> *ht, uint64_t idx,
                                                     int32_t key, int32_t pay) {
  return atomicCAS(reinterpret_cast<unsigned long long *>(ht + idx),
                   0xffffffffffffffffull, lp_entry(key, pay));
}
__device__ __forceinline__ unsigned long long lp_try(Tuple<int64_t> *ht, uint64_t idx,
                                                     int64_t key, int64_t) {
  return atomicCAS(reinterpret_cast<unsigned long long *>(&ht[idx].key),
                   0xffffffffffffffffull, static_cast<unsigned long long>(key));
}
// After a successful lp_try: the int64 payload goes in beside the key.
__device__ __forceinline__ void lp_done(Tuple<int32_t> *, uint64_t, int32_t) {}
__device__ __forceinline__ void lp_done(Tuple<int64_t> *ht, uint64_t idx, int64_t pay) {
  ht[idx].value = pay;
}

template <typename K>
__global__ void __launch_bounds__(kBuildThreads)
    ht_build_grouped_kernel(Tuple<K> *ht, uint64_t size, int scheme,
                            bool selective, const Tuple<K> *__restrict__ tuples,
                            uint64_t len, uint32_t *tile_counter) {
  __shared__ uint32_t s_tile;
  const uint32_t lg = log2_floor_u64(size);
  const uint64_t n = 1ull << lg, m = n - 1;
  const uint64_t ntiles = (len + kBuildTile - 1) / kBuildTile;
  const uint32_t tid = threadIdx.x;
  for (;;) {
    __syncthreads();  // every thread has read the previous tile id
    if (tid == 0) s_tile = atomicAdd(tile_counter, 1u);
    __syncthreads();
    const uint64_t t = s_tile;
    if (t >= ntiles) break;
    const uint64_t t0 = t * kBuildTile;
    Tuple<K> tp[kBuildItems];
    bool act[kBuildItems];
#pragma unroll
    for (uint32_t u = 0; u < kBuildItems; ++u) {
      const uint64_t i = t0 + u * kBuildThreads + tid;
      act[u] = i < len;
      if (act[u]) tp[u] = load_tuple_cs(tuples + i);
    }
    if (scheme != 1) {
#pragma unroll
      for (uint32_t u = 0; u < kBuildItems; ++u) {
        if (!act[u] || (selective && tp[u].key == null_key<K>())) continue;
        const uint64_t slot = static_cast<uint64_t>(static_cast<int64_t>(tp[u].key));
        if (slot < size) store_tuple(ht + slot, tp[u]);
      }
      continue;
    }
    uint64_t idx[kBuildItems];
    unsigned long long old[kBuildItems];
#pragma unroll
    for (uint32_t u = 0; u < kBuildItems; ++u) {
      idx[u] = lg ? mult_shift_hash<K>(tp[u].key, lg) : 0;
      if (act[u]) old[u] = lp_try(ht, idx[u], tp[u].key, tp[u].value);
    }
#pragma unroll
    for (uint32_t u = 0; u < kBuildItems; ++u) {
      if (!act[u]) continue;
      // the first slot was tried; at most n - 1 more, as lp_insert
      for (uint64_t s = 1; old[u] != 0xffffffffffffffffull && s < n; ++s) {
        idx[u] = (idx[u] + 1) & m;
        old[u] = lp_try(ht, idx[u], tp[u].key, tp[u].value);
      }
      if (old[u] == 0xffffffffffffffffull) lp_done(ht, idx[u], tp[u].value);
    }
  }
}

template <typename K>
cudaError_t launch_ht_build_grouped(int scheme, bool selective, void *ht,
                                    uint64_t ht_size, const K *key, const K *pay,
                                    uint64_t len, uint32_t grid, uint32_t block,
                                    uint32_t region_bits, void *tuples,
                                    uint32_t *region_scratch, uint64_t slice,
                                    uint32_t sm_count, cudaStream_t stream) {
  Tuple<K> *out = static_cast<Tuple<K> *>(tuples);
  // resident CTAs of the in-order build (grid and block of the caller do
  // not apply: the kernel's shape keeps its inserts in order)
  int per_sm = 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(
          &per_sm, (const void *)ht_build_grouped_kernel<K>, (int)kBuildThreads, 0) !=
          cudaSuccess ||
      per_sm < 1)
    per_sm = 1;
  const uint32_t build_grid = (uint32_t)per_sm * sm_count;
  for (uint64_t s0 = 0; s0 < len; s0 += slice) {
    const uint64_t n = min(slice, len - s0);
    cudaError_t e = group_by_region<K>(scheme, ht_size, key + s0, pay + s0, n,
                                       region_bits, out, region_scratch, sm_count,
                                       nullptr, stream);
    if (e != cudaSuccess) return e;
    uint32_t *tile_counter = region_scratch + 1;  // after the status word
    e = cudaMemsetAsync(tile_counter, 0, sizeof(uint32_t), stream);
    if (e != cudaSuccess) return e;
    ht_build_grouped_kernel<K><<<build_grid, kBuildThreads, 0, stream>>>(
        static_cast<Tuple<K> *>(ht), ht_size, scheme, selective, out, n,
        tile_counter);
    e = cudaGetLastError();
    if (e != cudaSuccess) return e;
  }
  return cudaSuccess;
}

template <typename K>
cudaError_t launch_ht_init(void *ht, uint64_t entries, cudaStream_t stream) {
  const uint64_t want = (entries + 255) / 256;
  const uint32_t grid = (uint32_t)(want < 148u * 32u ? want : 148u * 32u);
  if (grid == 0) return cudaSuccess;
  ht_init_kernel<K><<<grid, 256, 0, stream>>>(reinterpret_cast<Tuple<K> *>(ht),
                                              entries);
  return cudaGetLastError();
}

template <typename K>
cudaError_t launch_ht_build(int scheme, bool selective, void *ht,
                            uint64_t ht_size, const K *key, const K *pay,
                            uint64_t len, uint32_t grid, uint32_t block,
                            cudaStream_t stream) {
  if (scheme == 1)
    ht_build_lp_kernel<K><<<grid, block, 0, stream>>>(
        reinterpret_cast<Tuple<K> *>(ht), ht_size, key, pay, len);
  else
    ht_build_perfect_kernel<K><<<grid, block, 0, stream>>>(
        reinterpret_cast<Tuple<K> *>(ht), ht_size, key, pay, len, selective);
  return cudaGetLastError();
}

template <typename K>
cudaError_t launch_ht_probe_sum(int scheme, const void *ht, uint64_t ht_size,
                                const K *key, const K *pay, uint64_t len,
                                uint64_t *result, uint32_t grid, uint32_t block,
                                cudaStream_t stream) {
  if (scheme == 1)
    ht_probe_lp_kernel<K><<<grid, block, 0, stream>>>(
        reinterpret_cast<const Tuple<K> *>(ht), ht_size, key, pay, len, result);
  else
    ht_probe_perfect_kernel<K><<<grid, block, 0, stream>>>(
        reinterpret_cast<const Tuple<K> *>(ht), ht_size, key, pay, len, result);
  return cudaGetLastError();
}

#define FI_INSTANTIATE_HT(K)                                                   \
  template cudaError_t launch_ht_probe_grouped<K>(                             \
      int, const void *, uint64_t, const K *, const K *, uint64_t, uint64_t *, \
      uint32_t, uint32_t, uint32_t, void *, uint32_t *, uint64_t, uint32_t,    \
      cudaStream_t);                                                           \
  template cudaError_t launch_ht_build_grouped<K>(                             \
      int, bool, void *, uint64_t, const K *, const K *, uint64_t, uint32_t,   \
      uint32_t, uint32_t, void *, uint32_t *, uint64_t, uint32_t, cudaStream_t); \
  template cudaError_t launch_ht_init<K>(void *, uint64_t, cudaStream_t);      \
  template cudaError_t launch_ht_build<K>(int, bool, void *, uint64_t,         \
                                          const K *, const K *, uint64_t,      \
                                          uint32_t, uint32_t, cudaStream_t);   \
  template cudaError_t launch_ht_probe_sum<K>(                                 \
      int, const void *, uint64_t, const K *, const K *, uint64_t, uint64_t *, \
      uint32_t, uint32_t, cudaStream_t);

FI_INSTANTIATE_HT(int32_t)
FI_INSTANTIATE_HT(int64_t)

}  // namespace fi
