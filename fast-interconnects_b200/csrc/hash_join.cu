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
// Measured on B200 (Blanas: 16M x 256M int64, 1184 x 256 threads): linear
// probing builds in 1.0 ms and probes in 11.1 ms (a 2^25-entry, 512 MB
// table: one random access per probe, far beyond the 126 MB L2), perfect
// hashing probes in 4.7 ms (16M + 1 entries).  Four tuples per thread with
// their table loads issued together made it no faster (11.7 ms), nor did
// loading a window of 4 slots (64 B) per step instead of slot by slot (11.0
// ms): the probe is bound by the rate of random HBM accesses (about 30 G/s
// reach DRAM in both schemes), and the perfect table is faster because it is
// half the size, so twice as much of it stays in L2.  The table size
// matters more: the hash masks with 2^floor(log2(size)) (as the reference
// does), so a size that is not a power of two can fill the table to near
// 1 (Kim, 128e6 keys in 2^27 slots: 27 ms per probe against 5.8 ms in 2^28).
#include "common.cuh"
#include "kernels.h"

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

// ---- region-ordered probing ------------------------------------------------
// A table far larger than L2 is probed at random: every probe reaches HBM
// (Blanas, 2^25 int64 slots: 24 G probes/s, 11 ms).  Grouping the probe
// tuples by the table region their first slot lies in (the top region_bits
// bits of the slot) and probing group by group keeps the active region
// (a few MB) in L2, so the table is read from HBM about once per slice.  The
// grouping is one streamed pass (a histogram of region ids and a tile
// scatter into a scratch buffer); the sum does not depend on the order.

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

// The probes of a grouped slice, in order: every probe as in
// ht_probe_{lp,perfect}_kernel.
template <typename K>
__global__ void ht_probe_grouped_kernel(const Tuple<K> *__restrict__ ht,
                                        uint64_t size, int scheme,
                                        const Tuple<K> *__restrict__ probes,
                                        uint64_t len,
                                        uint64_t *__restrict__ result) {
  const uint32_t lg = log2_floor_u64(size);
  const uint64_t n = 1ull << lg, m = n - 1;
  const uint64_t gid = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
  uint64_t sum = 0;
  for (uint64_t i = gid; i < len; i += (uint64_t)gridDim.x * blockDim.x) {
    const Tuple<K> p = load_tuple_cs(probes + i);
    if (scheme == 1) {
      uint64_t idx = lg ? mult_shift_hash<K>(p.key, lg) : 0;
      for (uint64_t s = 0; s < n; ++s, idx = (idx + 1) & m) {
        const Tuple<K> e = load_tuple(ht + idx);
        if (e.key == p.key)
          sum += static_cast<uint64_t>(static_cast<int64_t>(p.value));
        else if (e.key == null_key<K>())
          break;
      }
    } else {
      const uint64_t slot = static_cast<uint64_t>(static_cast<int64_t>(p.key));
      if (slot < size && ht[slot].key == p.key)
        sum += static_cast<uint64_t>(static_cast<int64_t>(p.value));
    }
  }
  result[gid] += sum;
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

size_t ht_region_scratch_bytes(uint32_t region_bits) {
  return ((size_t)2 << region_bits) * sizeof(uint32_t);
}

template <typename K>
cudaError_t launch_ht_probe_grouped(int scheme, const void *ht, uint64_t ht_size,
                                    const K *key, const K *pay, uint64_t len,
                                    uint64_t *result, uint32_t grid, uint32_t block,
                                    uint32_t region_bits, void *tuples,
                                    uint32_t *region_scratch, uint64_t slice,
                                    uint32_t sm_count, cudaStream_t stream) {
  const uint32_t lg = 63u - (uint32_t)__builtin_clzll(ht_size);
  const uint32_t regions = 1u << region_bits;
  // linear probing: regions of the hash range 2^lg; perfect: of the key
  // range [0, size), rounded up to a power of two
  uint32_t range_bits = lg;
  if (scheme != 1 && (1ull << lg) < ht_size) ++range_bits;
  const uint32_t shift = range_bits > region_bits ? range_bits - region_bits : 0;
  uint32_t *counts = region_scratch, *cursors = region_scratch + regions;
  Tuple<K> *out = static_cast<Tuple<K> *>(tuples);
  const size_t scatter_smem = (size_t)kRegionTile * sizeof(Tuple<K>) +
                              ((size_t)2 * regions + 1 + 33) * sizeof(uint32_t);
  cudaError_t e = cudaFuncSetAttribute((const void *)region_scatter_kernel<K>,
                                       cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       (int)scatter_smem);
  if (e != cudaSuccess) return e;
  for (uint64_t s0 = 0; s0 < len; s0 += slice) {
    const uint64_t n = min(slice, len - s0);
    e = cudaMemsetAsync(counts, 0, regions * sizeof(uint32_t), stream);
    if (e != cudaSuccess) return e;
    const uint32_t copies = regions <= kPrivateRegions ? kRegionThreads / 32 : 1;
    region_histogram_kernel<K><<<2 * sm_count, kRegionThreads,
                                 (size_t)regions * copies * sizeof(uint32_t), stream>>>(
        key + s0, n, scheme, lg, ht_size, shift, regions, copies, counts);
    region_scan_kernel<<<1, 1024, (regions + 33) * sizeof(uint32_t), stream>>>(
        counts, regions, cursors);
    region_scatter_kernel<K><<<2 * sm_count, kRegionThreads, scatter_smem, stream>>>(
        key + s0, pay + s0, n, scheme, lg, ht_size, shift, regions, cursors, out);
    ht_probe_grouped_kernel<K><<<grid, block, 0, stream>>>(
        static_cast<const Tuple<K> *>(ht), ht_size, scheme, out, n, result);
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
