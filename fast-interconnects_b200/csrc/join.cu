// Per-partition shared-memory radix join (sm_100a).
//
// Replaces gpu_radix_join_assign_tasks, gpu_join_aggregate_smem_perfect_* and
// gpu_join_aggregate_smem_chaining_* of the reference
// (sql-ops/cudautils/radix_join.cu:58-332).  The query is
//     SELECT SUM(s.value) FROM r JOIN s ON r.key = s.key
// evaluated partition by partition; partition p of a Contiguous relation spans
// [off[p], off[p+1] - pad) and the last one ends at the relation's length.
//
// B200 design:
//  * Work items instead of static partition ranges: every partition whose
//    build and probe sides are both non-empty becomes ceil(|S_p| / W) items
//    (W probe tuples each).  A planning kernel counts the items and scans
//    them (decoupled look-back).  Persistent CTAs take items from an atomic
//    counter, so a Zipf-skewed partition is probed by many CTAs instead of
//    one, and CTAs never idle while work is left.
//  * The build side of an item's partition is loaded into shared memory (up
//    to the 227 KB opt-in size): a bucket-chaining table (heads + next links
//    + keys) or a perfect-hash array indexed by key >> ignore_bits.  A CTA
//    keeps its table when its next item belongs to the same partition.
//    Build values are not stored: the aggregate only reads s.value.
//  * A build side larger than the table is joined in rounds (each round
//    builds a slice and probes the item), so capacity is never exceeded
//    (the reference asserts instead).
//  * Probe tuples stream in with 16-byte evict-first loads, several per
//    thread in flight.
//  * Each thread adds its sum into result_set[global thread] (the reference's
//    output convention, cuda_radix_join.rs:15-30); match counts are reduced
//    per CTA and added to one u64.
#include "common.cuh"
#include "kernels.h"

namespace fi {

constexpr uint32_t kPlanThreads = 1024;
constexpr uint32_t kProbeUnroll = 4;
constexpr uint32_t kChainLog2Buckets = 13;  // 8192 buckets
constexpr uint32_t kEnd = 0xffffffffu;
constexpr uint32_t kCtrlSmem = 256;  // bytes reserved for control variables

// ---- reference greedy task assignment --------------------------------------
// Same result as gpu_radix_join_assign_tasks (radix_join.cu:58-98), with the
// probe offsets staged through shared memory in windows so that the
// sequential loop reads shared instead of global memory.
__global__ void __launch_bounds__(1024)
    assign_tasks_kernel(const uint64_t *__restrict__ probe_offsets,
                        uint32_t probe_len, uint32_t probe_pad, uint32_t F,
                        uint32_t grid, uint32_t *__restrict__ tasks) {
  constexpr uint32_t kWin = 4096;
  __shared__ uint64_t win[kWin + 1];
  const uint32_t probe_tuples = probe_len - probe_pad * F;
  const uint32_t avg = (probe_tuples + grid - 1u) / grid;
  uint32_t task_id = 1u, task_size = 0u;
  if (threadIdx.x == 0) tasks[0] = 0u;
  for (uint32_t w0 = 0; w0 < F; w0 += kWin) {
    const uint32_t n = min(kWin, F - w0);
    __syncthreads();
    for (uint32_t i = threadIdx.x; i <= n; i += blockDim.x)
      win[i] = (w0 + i < F) ? probe_offsets[w0 + i] : 0ull;
    __syncthreads();
    if (threadIdx.x == 0) {
      for (uint32_t i = 0; i < n && task_id < grid; ++i) {
        const uint32_t p = w0 + i;
        const uint32_t upper =
            (p + 1 < F) ? (uint32_t)(win[i + 1] - probe_pad) : probe_len;
        task_size += (uint32_t)(upper - (uint32_t)win[i]);
        if (task_size >= avg) {
          tasks[task_id] = p + 1u;
          task_size = 0u;
          task_id += 1u;
        }
      }
    }
  }
  if (threadIdx.x == 0)
    for (uint32_t t = task_id; t <= grid; ++t) tasks[t] = F;
}

// ---- partition bounds ----------------------------------------------------
__device__ __forceinline__ void part_bounds(const uint64_t *off, uint64_t len,
                                            uint32_t pad, uint32_t F,
                                            uint32_t p, uint64_t &b,
                                            uint64_t &e) {
  b = off[p];
  e = (p + 1 < F) ? off[p + 1] - pad : len;
  if (e < b) e = b;
}

// ---- item planning -------------------------------------------------------
__device__ __forceinline__ uint64_t plan_load(const uint64_t *p) {
  uint64_t v;
  asm volatile("ld.acquire.gpu.global.u64 %0, [%1];" : "=l"(v) : "l"(p) : "memory");
  return v;
}
__device__ __forceinline__ void plan_store(uint64_t *p, uint64_t v) {
  asm volatile("st.release.gpu.global.u64 [%0], %1;" ::"l"(p), "l"(v) : "memory");
}

// item_start[p] = sum_{q<p} items(q); item_start[F] = total.
__global__ void __launch_bounds__(kPlanThreads)
    join_plan_kernel(const uint64_t *__restrict__ build_off, uint64_t build_len,
                     uint32_t build_pad, const uint64_t *__restrict__ probe_off,
                     uint64_t probe_len, uint32_t probe_pad, uint32_t F,
                     uint32_t width, uint32_t *__restrict__ item_start,
                     uint64_t *tile_state, uint32_t *tile_counter,
                     int *status) {
  __shared__ uint32_t tile_s, prefix_s;
  __shared__ uint32_t warp_tmp[33];
  __shared__ uint32_t vals[kPlanThreads];
  if (threadIdx.x == 0) tile_s = atomicAdd(tile_counter, 1u);
  __syncthreads();
  const uint32_t t = tile_s;
  const uint32_t p = t * kPlanThreads + threadIdx.x;
  uint32_t items = 0;
  if (p < F) {
    uint64_t bb, be, pb, pe;
    part_bounds(build_off, build_len, build_pad, F, p, bb, be);
    part_bounds(probe_off, probe_len, probe_pad, F, p, pb, pe);
    if (be > bb && pe > pb) items = (uint32_t)((pe - pb + width - 1) / width);
  }
  vals[threadIdx.x] = items;
  __syncthreads();
  const uint32_t tile_total = block_exclusive_scan_u32(vals, kPlanThreads, warp_tmp);
  if (threadIdx.x == 0) {
    // decoupled look-back over tiles (flag in the high bits)
    constexpr uint64_t kAgg = 1ull << 62, kPre = 2ull << 62,
                       kVal = (1ull << 62) - 1ull;
    uint64_t prefix = 0;
    if (t == 0) {
      plan_store(&tile_state[0], kPre | tile_total);
    } else {
      plan_store(&tile_state[t], kAgg | tile_total);
      int64_t j = (int64_t)t - 1;
      uint32_t polls = 0;
      while (j >= 0) {
        uint64_t s = plan_load(&tile_state[j]);
        uint64_t flag = s & ~kVal;
        if (flag == 0) {
          if (++polls > kSpinLimit) {
            record_error(status, kDevErrTimeout);
            break;
          }
          spin_pause(polls);
          continue;
        }
        prefix += s & kVal;
        if (flag == kPre) break;
        --j;
      }
      plan_store(&tile_state[t], kPre | (prefix + tile_total));
    }
    prefix_s = (uint32_t)prefix;
  }
  __syncthreads();
  if (p < F) item_start[p] = prefix_s + vals[threadIdx.x];
  if (p + 1 == F) item_start[F] = prefix_s + vals[threadIdx.x] + items;
}

// ---- the join -------------------------------------------------------------
template <typename K>
struct ChainTable {
  uint32_t *heads;  // [1 << kChainLog2Buckets]
  uint32_t *next;   // [cap]
  K *keys;          // [cap]
  uint32_t cap;
};

template <typename K>
__device__ __forceinline__ uint32_t chain_bucket(K key, uint32_t ignore_bits) {
  // hash of the key bits above the partition bits (radix_join.cu:275-276)
  return mult_shift_hash<K>(
      static_cast<K>(static_cast<uint64_t>(static_cast<int64_t>(key)) >>
                     ignore_bits),
      kChainLog2Buckets);
}

template <typename K>
__device__ __forceinline__ uint64_t perfect_index(K key, uint32_t ignore_bits) {
  return static_cast<uint64_t>(static_cast<int64_t>(key)) >> ignore_bits;
}

template <typename K, int kScheme>
__global__ void __launch_bounds__(1024, 1) radix_join_kernel(
    const Tuple<K> *__restrict__ build, const uint64_t *__restrict__ build_off,
    uint64_t build_len, uint32_t build_pad, const Tuple<K> *__restrict__ probe,
    const uint64_t *__restrict__ probe_off, uint64_t probe_len,
    uint32_t probe_pad, uint32_t F, uint32_t ignore_bits,
    const uint32_t *__restrict__ item_start, uint32_t *item_counter,
    uint32_t smem_bytes, int64_t *__restrict__ result_set,
    uint64_t *match_count, int *status) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  uint32_t *ctrl = reinterpret_cast<uint32_t *>(smem_raw);  // item, p, max
  unsigned char *table = smem_raw + kCtrlSmem;
  const uint32_t table_bytes = smem_bytes - kCtrlSmem;

  // table layout
  ChainTable<K> ct;
  K *pkeys = reinterpret_cast<K *>(table);
  uint32_t pcap = 0;
  if (kScheme == 2) {
    const uint32_t nb = 1u << kChainLog2Buckets;
    ct.heads = reinterpret_cast<uint32_t *>(table);
    ct.cap = (table_bytes - nb * 4u) / (uint32_t)(sizeof(K) + 4u);
    ct.keys = reinterpret_cast<K *>(table + nb * 4u);
    ct.next = reinterpret_cast<uint32_t *>(table + nb * 4u + ct.cap * sizeof(K));
  } else {
    pcap = table_bytes / (uint32_t)sizeof(K);
  }
  const uint32_t cap = (kScheme == 2) ? ct.cap : 0xffffffffu;
  if (kScheme != 2) {
    // every slot starts empty; afterwards only used slots are cleared
    for (uint32_t i = threadIdx.x; i < pcap; i += blockDim.x)
      pkeys[i] = null_key<K>();
  }

  const uint32_t total_items = item_start[F];
  int64_t sum = 0;
  uint64_t cnt = 0;
  int64_t cached_p = -1;
  uint64_t cached_used = 0;  // perfect: highest slot written + 1

  for (;;) {
    __syncthreads();
    if (threadIdx.x == 0) {
      uint32_t item = atomicAdd(item_counter, 1u);
      uint32_t p = 0;
      if (item < total_items) {
        uint32_t lo = 0, hi = F;  // last p with item_start[p] <= item
        while (hi - lo > 1) {
          uint32_t mid = (lo + hi) >> 1;
          if (item_start[mid] <= item) lo = mid; else hi = mid;
        }
        p = lo;
      }
      ctrl[0] = item;
      ctrl[1] = p;
    }
    __syncthreads();
    const uint32_t item = ctrl[0], p = ctrl[1];
    if (item >= total_items) break;
    const uint32_t k = item - item_start[p];
    const uint32_t nitems = item_start[p + 1] - item_start[p];
    uint64_t bb, be, pb, pe;
    part_bounds(build_off, build_len, build_pad, F, p, bb, be);
    part_bounds(probe_off, probe_len, probe_pad, F, p, pb, pe);
    const uint64_t per = (pe - pb + nitems - 1) / nitems;
    const uint64_t qb = pb + per * k, qe = min(pe, qb + per);
    const uint64_t bsize = be - bb;

    for (uint64_t r0 = 0; r0 < bsize; r0 += cap) {
      const uint64_t rn = min((uint64_t)cap, bsize - r0);
      const bool reuse = (cached_p == (int64_t)p) && bsize <= cap;
      if (!reuse) {
        // ---- build ----
        if (kScheme == 2) {
          for (uint32_t i = threadIdx.x; i < (1u << kChainLog2Buckets);
               i += blockDim.x)
            ct.heads[i] = kEnd;
          __syncthreads();
          for (uint32_t i = threadIdx.x; i < rn; i += blockDim.x) {
            const K key = load_tuple(build + bb + r0 + i).key;
            ct.keys[i] = key;
            ct.next[i] = atomicExch(&ct.heads[chain_bucket(key, ignore_bits)], i);
          }
        } else {
          // clear the slots the previous build used
          for (uint64_t i = threadIdx.x; i < cached_used; i += blockDim.x)
            pkeys[i] = null_key<K>();
          __syncthreads();
          uint32_t used = 0;
          for (uint32_t i = threadIdx.x; i < rn; i += blockDim.x) {
            const K key = load_tuple(build + bb + r0 + i).key;
            const uint64_t idx = perfect_index(key, ignore_bits);
            if (idx < pcap) {
              pkeys[idx] = key;
              used = max(used, (uint32_t)idx + 1u);
            } else {
              record_error(status, kDevErrCapacity);
            }
          }
          // block max of `used`
          __syncthreads();
          if (threadIdx.x == 0) ctrl[2] = 0;
          __syncthreads();
          atomicMax(&ctrl[2], used);
          __syncthreads();
          cached_used = ctrl[2];
        }
        __syncthreads();
        cached_p = (bsize <= cap) ? (int64_t)p : -1;
      }
      // ---- probe ----
      for (uint64_t base = qb; base < qe;
           base += (uint64_t)blockDim.x * kProbeUnroll) {
        Tuple<K> t[kProbeUnroll];
#pragma unroll
        for (uint32_t u = 0; u < kProbeUnroll; ++u) {
          const uint64_t j = base + (uint64_t)u * blockDim.x + threadIdx.x;
          if (j < qe) t[u] = load_tuple_cs(probe + j);
        }
#pragma unroll
        for (uint32_t u = 0; u < kProbeUnroll; ++u) {
          const uint64_t j = base + (uint64_t)u * blockDim.x + threadIdx.x;
          if (j >= qe) continue;
          const K key = t[u].key;
          if (kScheme == 2) {
            for (uint32_t e = ct.heads[chain_bucket(key, ignore_bits)];
                 e != kEnd; e = ct.next[e]) {
              if (ct.keys[e] == key) {
                sum += static_cast<int64_t>(t[u].value);
                cnt += 1;
              }
            }
          } else {
            const uint64_t idx = perfect_index(key, ignore_bits);
            if (idx < pcap && pkeys[idx] == key) {
              sum += static_cast<int64_t>(t[u].value);
              cnt += 1;
            }
          }
        }
      }
      if (bsize > cap) __syncthreads();  // next round rebuilds the table
    }
  }

  result_set[(uint64_t)blockIdx.x * blockDim.x + threadIdx.x] += sum;
  if (match_count != nullptr) {
    __shared__ uint64_t red_tmp[32];
    uint64_t bc = block_reduce_u64(cnt, red_tmp);
    if (threadIdx.x == 0 && bc != 0) atomicAdd((unsigned long long *)match_count,
                                               (unsigned long long)bc);
  }
}

// ---- launchers ---------------------------------------------------------------
uint32_t join_items_capacity(uint32_t fanout) { return fanout + 1; }

template <typename K>
cudaError_t launch_assign_tasks(const uint64_t *probe_offsets,
                                uint32_t probe_len, uint32_t probe_pad,
                                uint32_t radix_bits, uint32_t grid,
                                uint32_t *tasks, cudaStream_t stream) {
  assign_tasks_kernel<<<1, 1024, 0, stream>>>(
      probe_offsets, probe_len, probe_pad, 1u << radix_bits, grid, tasks);
  return cudaGetLastError();
}

template <typename K>
cudaError_t launch_radix_join(const void *build, const uint64_t *build_off,
                              uint64_t build_len, uint32_t build_pad,
                              const void *probe, const uint64_t *probe_off,
                              uint64_t probe_len, uint32_t probe_pad,
                              uint32_t fanout, uint32_t ignore_bits, int scheme,
                              uint32_t grid, uint32_t block,
                              int64_t *result_set, uint64_t *match_count,
                              JoinScratch s, uint32_t sm_count,
                              cudaStream_t stream) {
  // probe width per item: enough items to keep every CTA busy, but at least
  // 8K tuples so that table builds stay amortised
  const uint64_t probe_tuples =
      probe_len > (uint64_t)probe_pad * fanout ? probe_len - (uint64_t)probe_pad * fanout : 0;
  uint64_t width = probe_tuples / ((uint64_t)grid * 8u + 1u);
  if (width < 8192) width = 8192;
  if (width > (1u << 30)) width = 1u << 30;
  const uint32_t tiles = (fanout + kPlanThreads - 1) / kPlanThreads;
  cudaError_t e = cudaMemsetAsync(s.tile_state, 0,
                                  (size_t)(tiles + 1) * sizeof(uint64_t), stream);
  if (e != cudaSuccess) return e;
  e = cudaMemsetAsync(s.tile_counter, 0, sizeof(uint32_t), stream);
  if (e != cudaSuccess) return e;
  e = cudaMemsetAsync(s.item_counter, 0, sizeof(uint32_t), stream);
  if (e != cudaSuccess) return e;
  join_plan_kernel<<<tiles, kPlanThreads, 0, stream>>>(
      build_off, build_len, build_pad, probe_off, probe_len, probe_pad, fanout,
      (uint32_t)width, s.item_start, s.tile_state, s.tile_counter, s.status);
  e = cudaGetLastError();
  if (e != cudaSuccess) return e;

  const uint32_t smem = (uint32_t)device_max_smem_optin();
  const void *fn = scheme == 2 ? (const void *)radix_join_kernel<K, 2>
                               : (const void *)radix_join_kernel<K, 0>;
  e = cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize,
                           (int)smem);
  if (e != cudaSuccess) return e;
  if (scheme == 2)
    radix_join_kernel<K, 2><<<grid, block, smem, stream>>>(
        reinterpret_cast<const Tuple<K> *>(build), build_off, build_len,
        build_pad, reinterpret_cast<const Tuple<K> *>(probe), probe_off,
        probe_len, probe_pad, fanout, ignore_bits, s.item_start,
        s.item_counter, smem, result_set, match_count, s.status);
  else
    radix_join_kernel<K, 0><<<grid, block, smem, stream>>>(
        reinterpret_cast<const Tuple<K> *>(build), build_off, build_len,
        build_pad, reinterpret_cast<const Tuple<K> *>(probe), probe_off,
        probe_len, probe_pad, fanout, ignore_bits, s.item_start,
        s.item_counter, smem, result_set, match_count, s.status);
  (void)sm_count;
  return cudaGetLastError();
}

#define FI_INSTANTIATE_JOIN(K)                                                 \
  template cudaError_t launch_assign_tasks<K>(const uint64_t *, uint32_t,      \
                                              uint32_t, uint32_t, uint32_t,    \
                                              uint32_t *, cudaStream_t);       \
  template cudaError_t launch_radix_join<K>(                                   \
      const void *, const uint64_t *, uint64_t, uint32_t, const void *,        \
      const uint64_t *, uint64_t, uint32_t, uint32_t, uint32_t, int, uint32_t, \
      uint32_t, int64_t *, uint64_t *, JoinScratch, uint32_t, cudaStream_t);

FI_INSTANTIATE_JOIN(int32_t)
FI_INSTANTIATE_JOIN(int64_t)

}  // namespace fi
