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
