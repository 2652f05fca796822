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
//    (W probe tuples each).  A planning kernel counts the items, scans them
//    (decoupled look-back) and writes an item -> partition table.  Persistent
//    CTAs walk the items with a grid stride, so a Zipf-skewed partition is
//    probed by many CTAs instead of one.
//  * The build side of an item's partition is loaded into shared memory: a
//    bucket-chaining table (u32 heads, u16 next links, keys) sized from the
//    average build partition, or a perfect-hash array indexed by
//    key >> ignore_bits.  With blocks of up to 512 threads two CTAs share an
//    SM (four with up to 256), so one CTA's build overlaps another's probe.
//    A CTA keeps its
//    table when its next item belongs to the same partition.  Build values
//    are not stored: the aggregate only reads s.value.
//  * A build side larger than the table is joined in rounds (each round
//    builds a slice and probes the item), so capacity is never exceeded
//    (the reference asserts instead).
//  * Probe tuples stream in with 16-byte evict-first loads, several per
//    thread in flight.  When an item starts, its CTA issues one
//    prefetch.global.L2 per 128-byte line of the item's build range (unless
//    the table is kept) and of the first kProbePrefetch tuples of its probe
//    range, so the build and probe iterations
//    after the first find their lines in L2 instead of paying a DRAM round
//    trip each: 7.49 -> 6.61 ms for the 1024M x 1024M int64 join.  Also
//    prefetching the next item's build lines when this item's probe starts
//    measured 7.33 ms: the lines of two items per CTA crowd L2.
//  * Each thread adds its sum into result_set[global thread] (the reference's
//    output convention, cuda_radix_join.rs:15-30); match counts are reduced
//    per CTA and added to one u64.
//  * Measured on B200 and left out (1024M x 1024M int64, 9+9 bits, join 7.47
//    ms with four 256-thread CTAs per SM): a TMA-fed variant (one 1024-thread
//    CTA per SM, the next item's build side bulk-copied into a staging buffer
//    while the current item probes, probe tuples in two 2048-tuple chunk
//    buffers): 9.63 ms, since 227 KB cannot keep a whole next partition in
//    flight and each item waits on its first chunks; bulk L2 prefetches of
//    the next item's build and probe ranges: 10.37 ms; eight probe loads in
//    flight per thread instead of four: 9.16 ms (register spills), or 8.20
//    ms with three 256-thread CTAs per SM to give them the registers: the
//    number of partitions an SM works on at once matters more than the
//    loads each thread keeps in flight.  u16 bucket heads (twice the
//    buckets in the same shared memory, chains half as long) with a 16-bit
//    CAS-loop exchange in the build: join 6.61 -> 8.06 ms.
#include <atomic>

#include "common.cuh"
#include "kernels.h"

namespace fi {

constexpr uint32_t kPlanThreads = 1024;
constexpr uint32_t kProbeUnroll = 4;
// Probe tuples of an item prefetched into L2 when it starts.  Prefetching
// all of a long item (a Zipf-hot partition's items hold 450K tuples, the
// Blanas data set's 64K) fills L2 with lines evicted before their use: the
// join at Zipf 1.5 took 9.19 ms with it, 7.94 ms with this cap (uniform:
// 6.61 and 6.63 ms).  A rolling window of 4096 tuples kept ahead of the
// probe loop gave 7.84 ms, but its extra code in the loop cost the uniform
// join 0.13 ms.
constexpr uint32_t kProbePrefetch = 8192;

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

// item_start[p] = sum_{q<p} items(q); item_start[F] = total.  With
// heavy_cap > 0 (bucket chaining), a partition whose build side exceeds
// heavy_cap tuples gets no items; it is appended instead to the heavy list
// that grows down from item_part[item_cap - 1] (*heavy_count entries).  The
// two fit together: every partition takes at most ceil(probe / width) >= 1
// entries, and item_cap bounds their sum.
__global__ void __launch_bounds__(kPlanThreads)
    join_plan_kernel(const uint64_t *__restrict__ build_off, uint64_t build_len,
                     uint32_t build_pad, const uint64_t *__restrict__ probe_off,
                     uint64_t probe_len, uint32_t probe_pad, uint32_t F,
                     uint32_t width, uint32_t heavy_cap, uint32_t item_cap,
                     uint32_t *__restrict__ item_start,
                     uint32_t *__restrict__ item_part, uint32_t *heavy_count,
                     uint64_t *tile_state, uint32_t *tile_counter, int *status) {
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
    if (be > bb && pe > pb) {
      if (heavy_cap != 0 && be - bb > heavy_cap)
        item_part[item_cap - 1u - atomicAdd(heavy_count, 1u)] = p;
      else
        items = (uint32_t)((pe - pb + width - 1) / width);
    }
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
  if (p < F) {
    const uint32_t first = prefix_s + vals[threadIdx.x];
    item_start[p] = first;
    for (uint32_t k = 0; k < items; ++k) item_part[first + k] = p;
  }
  if (p + 1 == F) item_start[F] = prefix_s + vals[threadIdx.x] + items;
}

// ---- the join -------------------------------------------------------------
__device__ __forceinline__ void prefetch_l2(const void *p) {
  asm volatile("prefetch.global.L2 [%0];" ::"l"(p));
}

constexpr uint32_t kLinkEnd = 0xffffu;  // u16 chain links
constexpr uint32_t kHeadEnd = 0xffffffffu;

template <typename K>
__device__ __forceinline__ uint32_t chain_bucket(K key, uint32_t ignore_bits,
                                                 uint32_t log2_buckets) {
  // hash of the key bits above the partition bits (radix_join.cu:275-276)
  return mult_shift_hash<K>(
      static_cast<K>(static_cast<uint64_t>(static_cast<int64_t>(key)) >>
                     ignore_bits),
      log2_buckets);
}

template <typename K>
__device__ __forceinline__ uint64_t perfect_index(K key, uint32_t ignore_bits) {
  return static_cast<uint64_t>(static_cast<int64_t>(key)) >> ignore_bits;
}

// Table layout in dynamic shared memory.
//   chaining: keys K[cap] | next u16[cap] | heads u32[2^log2_buckets]
//   perfect:  keys K[pcap], indexed by key >> ignore_bits
template <typename K>
struct SmemTable {
  K *keys;
  uint16_t *next;
  uint32_t *heads;
  uint32_t cap;
};

template <typename K>
__host__ __device__ inline uint32_t chain_capacity(uint32_t table_bytes,
                                                   uint32_t log2_buckets) {
  const uint32_t hb = 4u << log2_buckets;
  if (table_bytes <= hb + 64) return 0;
  uint32_t cap = (table_bytes - hb - 64) / (uint32_t)(sizeof(K) + 2);
  cap &= ~7u;
  return cap < 65528u ? cap : 65528u;
}

// Heavy partitions (bucket chaining): a partition whose build side exceeds
// the table was left out of the items and listed at the end of item_part;
// each becomes R x Q units (build round r of `cap` tuples x probe slice q of
// at most `width` tuples), numbered consecutively over the list and dealt
// round-robin to the CTAs.  A partition of tens of millions of equal build
// keys (e.g. the null keys of a selective data set) is so spread over the
// whole GPU instead of being joined round after round by one CTA.  Called
// by every thread of radix_join_kernel after its items, with the CTA's table
// in `smem`; kept out of line so that the item loop's code is the same with
// and without it (inlined, the kernel's register allocation changed and the
// join of 1024M x 1024M int64 became 4% slower).
struct HeavyResult {
  int64_t sum;
  uint64_t cnt;
};

template <typename K>
__device__ __noinline__ HeavyResult join_heavy_units(
    unsigned char *smem, const Tuple<K> *__restrict__ build,
    const uint64_t *__restrict__ build_off, uint64_t build_len, uint32_t build_pad,
    const Tuple<K> *__restrict__ probe, const uint64_t *__restrict__ probe_off,
    uint64_t probe_len, uint32_t probe_pad, uint32_t F, uint32_t ignore_bits,
    const uint32_t *__restrict__ item_part, uint32_t item_cap, uint32_t H,
    uint32_t width, uint32_t table_bytes, uint32_t log2_buckets) {
  const uint32_t tid = threadIdx.x, nt = blockDim.x;
  const uint32_t cap = chain_capacity<K>(table_bytes, log2_buckets);
  K *tkeys = reinterpret_cast<K *>(smem);
  uint16_t *tnext = reinterpret_cast<uint16_t *>(tkeys + cap);
  uint32_t *heads =
      reinterpret_cast<uint32_t *>(smem + ((cap * (sizeof(K) + 2) + 15) & ~15u));
  const uint32_t nbuckets = 1u << log2_buckets;
  HeavyResult res{0, 0};
  int64_t cached_p = -1, cached_r = -1;
  uint64_t g0 = 0;
  for (uint32_t h = 0; h < H; ++h) {
    const uint32_t hp = item_part[item_cap - 1u - h];
    uint64_t bb, be, pb, pe;
    part_bounds(build_off, build_len, build_pad, F, hp, bb, be);
    part_bounds(probe_off, probe_len, probe_pad, F, hp, pb, pe);
    const uint64_t bsize = be - bb, psize = pe - pb;
    const uint64_t R = (bsize + cap - 1) / cap;
    const uint64_t Q = (psize + width - 1) / width;
    const uint64_t per = (psize + Q - 1) / Q;
    const uint64_t U = R * Q;
    uint64_t g = g0 + (blockIdx.x + gridDim.x - g0 % gridDim.x) % gridDim.x;
    for (; g < g0 + U; g += gridDim.x) {
      const uint64_t u = g - g0, r = u / Q, qi = u % Q;
      if (!(cached_p == (int64_t)hp && cached_r == (int64_t)r)) {
        const uint64_t r0 = r * cap;
        const uint32_t rn = (uint32_t)min((uint64_t)cap, bsize - r0);
        __syncthreads();  // the previous unit's probe is done with the table
        for (uint32_t i = tid; i < nbuckets; i += nt) heads[i] = kHeadEnd;
        __syncthreads();
        for (uint32_t i = tid; i < rn; i += nt) {
          const K key = build[bb + r0 + i].key;
          tkeys[i] = key;
          const uint32_t old =
              atomicExch(&heads[chain_bucket(key, ignore_bits, log2_buckets)], i);
          tnext[i] = (uint16_t)(old == kHeadEnd ? kLinkEnd : old);
        }
        __syncthreads();
        cached_p = hp;
        cached_r = (int64_t)r;
      }
      const uint64_t qb = min(pe, pb + per * qi), qe = min(pe, qb + per);
      for (uint64_t j = qb + tid; j < qe; j += nt) {
        const Tuple<K> t = load_tuple_cs(probe + j);
        uint32_t e = heads[chain_bucket(t.key, ignore_bits, log2_buckets)];
        if (e == kHeadEnd) continue;
        for (;;) {
          if (tkeys[e] == t.key) {
            res.sum += static_cast<int64_t>(t.value);
            res.cnt += 1;
          }
          const uint32_t nx = tnext[e];
          if (nx == kLinkEnd) break;
          e = nx;
        }
      }
    }
    g0 += U;
  }
  return res;
}

// Persistent join: CTA b takes items b, b + grid, b + 2*grid, ...  Items
// are near-equal in probe work (at most `width` probe tuples each), so the
// grid stride balances skewed inputs while avoiding a global work counter;
// the partition of the next item is prefetched.  With bucket chaining the
// planner gives no items to partitions whose build side exceeds the table;
// join_heavy_units joins those after the items.
template <typename K, int kScheme, int kMaxThreads, int kMinBlocks>
__global__ void __launch_bounds__(kMaxThreads, kMinBlocks) radix_join_kernel(
    const Tuple<K> *__restrict__ build, const uint64_t *__restrict__ build_off,
    uint64_t build_len, uint32_t build_pad, const Tuple<K> *__restrict__ probe,
    const uint64_t *__restrict__ probe_off, uint64_t probe_len,
    uint32_t probe_pad, uint32_t F, uint32_t ignore_bits,
    const uint32_t *__restrict__ item_start,
    const uint32_t *__restrict__ item_part, uint32_t table_bytes,
    uint32_t log2_buckets, int64_t *__restrict__ result_set,
    uint64_t *match_count, int *status, uint32_t item_cap,
    const uint32_t *__restrict__ heavy_count, uint32_t width) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  __shared__ uint32_t s_used;
  __shared__ uint64_t red_tmp[32];
  const uint32_t tid = threadIdx.x, nt = blockDim.x;

  SmemTable<K> tb;
  tb.keys = reinterpret_cast<K *>(smem_raw);
  uint32_t cap, pcap = 0;
  if (kScheme == 2) {
    cap = chain_capacity<K>(table_bytes, log2_buckets);
    tb.next = reinterpret_cast<uint16_t *>(tb.keys + cap);
    tb.heads = reinterpret_cast<uint32_t *>(smem_raw +
                                            ((cap * (sizeof(K) + 2) + 15) & ~15u));
  } else {
    pcap = table_bytes / (uint32_t)sizeof(K);
    cap = 0xffffffffu;
    // every slot starts empty; afterwards only the used prefix is cleared
    for (uint32_t i = tid; i < pcap; i += nt) tb.keys[i] = null_key<K>();
  }
  const uint32_t nbuckets = 1u << log2_buckets;

  const uint32_t total_items = item_start[F];
  int64_t sum = 0;
  uint64_t cnt = 0;
  int64_t cached_p = -1;
  uint32_t cached_used = 0;  // perfect: highest slot written + 1

  uint32_t item = blockIdx.x;
  uint32_t p = item < total_items ? item_part[item] : 0u;
  for (; item < total_items; item += gridDim.x) {
    const uint32_t nitem = item + gridDim.x;
    const uint32_t np = nitem < total_items ? item_part[nitem] : 0u;  // prefetch
    const uint32_t k = item - item_start[p];
    const uint32_t nitems = item_start[p + 1] - item_start[p];
    uint64_t bb, be, pb, pe;
    part_bounds(build_off, build_len, build_pad, F, p, bb, be);
    part_bounds(probe_off, probe_len, probe_pad, F, p, pb, pe);
    const uint64_t per = (pe - pb + nitems - 1) / nitems;
    const uint64_t qb = pb + per * k, qe = min(pe, qb + per);
    const uint64_t bsize = be - bb;
    {  // the item's lines into L2 now, so that its loop iterations hit L2
      constexpr uint32_t kLine = 128 / sizeof(Tuple<K>);
      const uint32_t bn = (cached_p == (int64_t)p && bsize <= cap)
                              ? 0u : (uint32_t)min(bsize, (uint64_t)cap);
      const uint32_t qn = (uint32_t)min(qe - qb, (uint64_t)kProbePrefetch);
      for (uint32_t i = tid * kLine; i < bn; i += nt * kLine) prefetch_l2(build + bb + i);
      for (uint32_t i = tid * kLine; i < qn; i += nt * kLine) prefetch_l2(probe + qb + i);
    }

    for (uint64_t r0 = 0; r0 < bsize; r0 += cap) {
      const uint32_t rn = (uint32_t)min((uint64_t)cap, bsize - r0);
      const bool reuse = (cached_p == (int64_t)p) && bsize <= cap;
      if (!reuse) {
        __syncthreads();  // the previous item's probe is done with the table
        if (kScheme == 2) {
          for (uint32_t i = tid; i < nbuckets; i += nt) tb.heads[i] = kHeadEnd;
          __syncthreads();
          for (uint32_t i0 = 0; i0 < rn; i0 += nt * 4u) {
            K kk[4];
#pragma unroll
            for (uint32_t u = 0; u < 4; ++u) {
              const uint32_t i = i0 + u * nt + tid;
              if (i < rn) kk[u] = build[bb + r0 + i].key;
            }
#pragma unroll
            for (uint32_t u = 0; u < 4; ++u) {
              const uint32_t i = i0 + u * nt + tid;
              if (i < rn) {
                tb.keys[i] = kk[u];
                const uint32_t old = atomicExch(
                    &tb.heads[chain_bucket(kk[u], ignore_bits, log2_buckets)], i);
                tb.next[i] = (uint16_t)(old == kHeadEnd ? kLinkEnd : old);
              }
            }
          }
        } else {
          for (uint32_t i = tid; i < cached_used; i += nt) tb.keys[i] = null_key<K>();
          if (tid == 0) s_used = 0;
          __syncthreads();
          uint32_t used = 0;
          for (uint32_t i = tid; i < rn; i += nt) {
            const K key = build[bb + r0 + i].key;
            const uint64_t idx = perfect_index(key, ignore_bits);
            if (idx < pcap) {
              tb.keys[idx] = key;
              used = max(used, (uint32_t)idx + 1u);
            } else {
              record_error(status, kDevErrCapacity);
            }
          }
          if (used) atomicMax(&s_used, used);
        }
        __syncthreads();
        if (kScheme != 2) cached_used = s_used;
        cached_p = (bsize <= cap) ? (int64_t)p : -1;
      }
      // ---- probe ----
      for (uint64_t base = qb; base < qe; base += (uint64_t)nt * kProbeUnroll) {
        Tuple<K> t[kProbeUnroll];
#pragma unroll
        for (uint32_t u = 0; u < kProbeUnroll; ++u) {
          const uint64_t j = base + (uint64_t)u * nt + tid;
          if (j < qe) t[u] = load_tuple_cs(probe + j);
        }
#pragma unroll
        for (uint32_t u = 0; u < kProbeUnroll; ++u) {
          const uint64_t j = base + (uint64_t)u * nt + tid;
          if (j >= qe) continue;
          const K key = t[u].key;
          if (kScheme == 2) {
            uint32_t e = tb.heads[chain_bucket(key, ignore_bits, log2_buckets)];
            if (e != kHeadEnd) {
              for (;;) {
                if (tb.keys[e] == key) {
                  sum += static_cast<int64_t>(t[u].value);
                  cnt += 1;
                }
                const uint32_t nx = tb.next[e];
                if (nx == kLinkEnd) break;
                e = nx;
              }
            }
          } else {
            const uint64_t idx = perfect_index(key, ignore_bits);
            if (idx < pcap && tb.keys[idx] == key) {
              sum += static_cast<int64_t>(t[u].value);
              cnt += 1;
            }
          }
        }
      }
    }
    p = np;
  }
  if (kScheme == 2 && heavy_count != nullptr) {
    const uint32_t H = *heavy_count;
    if (H) {
      const HeavyResult hr = join_heavy_units<K>(
          smem_raw, build, build_off, build_len, build_pad, probe, probe_off,
          probe_len, probe_pad, F, ignore_bits, item_part, item_cap, H, width,
          table_bytes, log2_buckets);
      sum += hr.sum;
      cnt += hr.cnt;
    }
  }

  result_set[(uint64_t)blockIdx.x * nt + tid] += sum;
  if (match_count != nullptr) {
    const uint64_t bc = block_reduce_u64(cnt, red_tmp);
    if (tid == 0 && bc != 0)
      atomicAdd((unsigned long long *)match_count, (unsigned long long)bc);
  }
}

// ---- launchers ---------------------------------------------------------------
constexpr uint64_t kMinItemWidth = 8192;

uint32_t join_items_capacity(uint32_t fanout, uint64_t probe_len) {
  return (uint32_t)(fanout + probe_len / kMinItemWidth + 2);
}

template <typename K>
cudaError_t launch_assign_tasks(const uint64_t *probe_offsets,
                                uint32_t probe_len, uint32_t probe_pad,
                                uint32_t radix_bits, uint32_t grid,
                                uint32_t *tasks, cudaStream_t stream) {
  assign_tasks_kernel<<<1, 1024, 0, stream>>>(
      probe_offsets, probe_len, probe_pad, 1u << radix_bits, grid, tasks);
  return cudaGetLastError();
}

template <typename K, int kScheme>
static const void *join_kernel_ptr(uint32_t ctas_per_sm) {
  return ctas_per_sm == 4   ? (const void *)radix_join_kernel<K, kScheme, 256, 4>
         : ctas_per_sm == 2 ? (const void *)radix_join_kernel<K, kScheme, 512, 2>
                            : (const void *)radix_join_kernel<K, kScheme, 1024, 1>;
}

uint32_t join_ctas_per_sm(uint32_t block) {
  return block <= 256 ? 4u : block <= 512 ? 2u : 1u;
}

template <typename K, int kScheme>
static uint32_t join_dyn_smem_query(uint32_t ctas);

// Dynamic shared memory of one join CTA when `ctas` share an SM (queried
// once per kernel and shape; every device of a process is taken to be a B200).
template <typename K, int kScheme>
static uint32_t join_dyn_smem(uint32_t ctas) {
  static std::atomic<uint32_t> cached[3];
  const int slot = ctas == 4 ? 0 : ctas == 2 ? 1 : 2;
  const uint32_t c = cached[slot].load(std::memory_order_relaxed);
  if (c) return c;
  const uint32_t v = join_dyn_smem_query<K, kScheme>(ctas);
  cached[slot].store(v, std::memory_order_relaxed);
  return v;
}

template <typename K, int kScheme>
static uint32_t join_dyn_smem_query(uint32_t ctas) {
  cudaFuncAttributes attr;
  if (cudaFuncGetAttributes(&attr, join_kernel_ptr<K, kScheme>(ctas)) != cudaSuccess) {
    cudaGetLastError();
    return 0;
  }
  int dev = 0, per_sm = 0, reserved = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&per_sm, cudaDevAttrMaxSharedMemoryPerMultiprocessor, dev);
  cudaDeviceGetAttribute(&reserved, cudaDevAttrReservedSharedMemoryPerBlock, dev);
  uint32_t dyn = (uint32_t)device_max_smem_optin() - (uint32_t)attr.sharedSizeBytes;
  if (ctas > 1) {
    const int share = per_sm / (int)ctas - reserved - (int)attr.sharedSizeBytes;
    if (share > 0 && (uint32_t)share < dyn) dyn = (uint32_t)share;
  }
  return dyn & ~127u;
}

// Bucket count of the chaining table for an average build partition `avg`:
// the next power of two above it, then fewer only while the table would not
// hold it with 1/8 headroom.
template <typename K>
static uint32_t join_log2_buckets(uint32_t dyn, uint64_t avg) {
  uint32_t lb = 8;
  while (lb < 14 && (1ull << lb) < avg) ++lb;
  while (lb > 8 && chain_capacity<K>(dyn, lb) < avg + avg / 8) --lb;
  return lb;
}

// A shape fits when its table holds an average partition with 1/8 headroom
// and at most about two keys per bucket (2^(floor(log2 avg) - 1) buckets or
// more): fewer buckets make chains that cost more than the extra CTAs win.
template <typename K>
uint32_t join_auto_block(uint64_t build_tuples, uint32_t fanout) {
  const uint64_t avg = build_tuples / (fanout ? fanout : 1) + 1;
  uint32_t lb_min = 0;
  while ((2ull << lb_min) <= avg) ++lb_min;  // floor(log2 avg)
  lb_min = lb_min > 9 ? lb_min - 1 : 8;
  if (lb_min > 14) lb_min = 14;
  for (uint32_t block : {256u, 512u}) {
    const uint32_t dyn = join_dyn_smem<K, 2>(join_ctas_per_sm(block));
    if (dyn && chain_capacity<K>(dyn, lb_min) >= avg + avg / 8) return block;
  }
  return 1024;
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
  (void)sm_count;
  // Several CTAs per SM (an equal share of the shared memory each) when the
  // block allows it, so that one CTA's table build overlaps another's probe:
  // 4 CTAs of <= 256 threads, 2 of <= 512, else one of 1024.
  const uint32_t ctas = join_ctas_per_sm(block);
  const void *fn = scheme == 2 ? join_kernel_ptr<K, 2>(ctas) : join_kernel_ptr<K, 0>(ctas);
  const uint32_t dyn =
      scheme == 2 ? join_dyn_smem<K, 2>(ctas) : join_dyn_smem<K, 0>(ctas);
  if (dyn == 0) return cudaErrorInvalidValue;
  cudaError_t e =
      cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)dyn);
  if (e != cudaSuccess) return e;

  // buckets (join_log2_buckets): a larger build side is joined in rounds;
  // asking for twice the average instead cut 8K-tuple partitions down to
  // 256 buckets, and the 32-entry chains made the join of 2^28 x 2^30 int64
  // tuples 7x slower (36.7 ms against 4.4-5.5 ms with short chains,
  // measured on B200).
  const uint64_t build_tuples =
      build_len > (uint64_t)build_pad * fanout ? build_len - (uint64_t)build_pad * fanout : 0;
  const uint64_t avg = build_tuples / fanout + 1;
  const uint32_t lb = join_log2_buckets<K>(dyn, avg);
  const uint32_t cap = chain_capacity<K>(dyn, lb);
  if (scheme == 2 && cap == 0) return cudaErrorInvalidValue;

  // probe width per item: about four items per CTA for the bulk, never below
  // kMinItemWidth tuples so that table builds stay amortised
  const uint64_t probe_tuples =
      probe_len > (uint64_t)probe_pad * fanout ? probe_len - (uint64_t)probe_pad * fanout : 0;
  uint64_t width = probe_tuples / ((uint64_t)grid * 4u + 1u);
  if (width < kMinItemWidth) width = kMinItemWidth;
  if (width > (1u << 30)) width = 1u << 30;
  const uint32_t item_cap = join_items_capacity(fanout, probe_len);
  uint32_t *heavy_count = s.tile_counter + 1;
  const uint32_t tiles = (fanout + kPlanThreads - 1) / kPlanThreads;
  e = cudaMemsetAsync(s.tile_state, 0, (size_t)(tiles + 1) * sizeof(uint64_t), stream);
  if (e != cudaSuccess) return e;
  e = cudaMemsetAsync(s.tile_counter, 0, 2 * sizeof(uint32_t), stream);
  if (e != cudaSuccess) return e;
  join_plan_kernel<<<tiles, kPlanThreads, 0, stream>>>(
      build_off, build_len, build_pad, probe_off, probe_len, probe_pad, fanout,
      (uint32_t)width, scheme == 2 ? cap : 0u, item_cap, s.item_start,
      s.item_part, heavy_count, s.tile_state, s.tile_counter, s.status);
  e = cudaGetLastError();
  if (e != cudaSuccess) return e;

  const auto *b = reinterpret_cast<const Tuple<K> *>(build);
  const auto *pr = reinterpret_cast<const Tuple<K> *>(probe);
#define FI_JOIN_LAUNCH(S, T, M)                                                \
  radix_join_kernel<K, S, T, M><<<grid, block, dyn, stream>>>(                 \
      b, build_off, build_len, build_pad, pr, probe_off, probe_len, probe_pad, \
      fanout, ignore_bits, s.item_start, s.item_part, dyn, lb, result_set,     \
      match_count, s.status, item_cap, heavy_count, (uint32_t)width)
  if (scheme == 2) {
    if (ctas == 4) FI_JOIN_LAUNCH(2, 256, 4);
    else if (ctas == 2) FI_JOIN_LAUNCH(2, 512, 2);
    else FI_JOIN_LAUNCH(2, 1024, 1);
  } else {
    if (ctas == 4) FI_JOIN_LAUNCH(0, 256, 4);
    else if (ctas == 2) FI_JOIN_LAUNCH(0, 512, 2);
    else FI_JOIN_LAUNCH(0, 1024, 1);
  }
#undef FI_JOIN_LAUNCH
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
template uint32_t join_auto_block<int32_t>(uint64_t, uint32_t);
template uint32_t join_auto_block<int64_t>(uint64_t, uint32_t);

}  // namespace fi
