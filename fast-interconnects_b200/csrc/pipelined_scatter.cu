// Pipelined two-level radix scatter for high fanouts, 12..18 bits (sm_100a).
//
// Replaces, above 11 radix bits, the reference's first-pass scatters for
// large fanouts (HSSWWCv4 / SSWWCv2, sql-ops/cudautils/radix_partition.cu:
// 689-1477); the per-(chunk, partition) tuple multisets are the same as every
// other scatter's.
//
// Why two levels: a tile of a few thousand tuples holds one or two tuples per
// partition at these fanouts, so a one-level scatter stores (and, sharing
// cursors, claims) tuple by tuple.  Measured on B200 over 512M int64 tuples,
// such per-tuple global requests run at about 40 G/s: 12-16 ms at 12-14 bits.
// Splitting the bits in halves keeps every run long: level 1 sorts a tile by
// the high half (64..512 buckets) and level 2 sorts a bucket by the low half.
//
// Why pipelined: level 1's output is written and read once more.  Done as two
// passes over the whole relation that costs 32 extra bytes of HBM traffic per
// tuple.  Here one persistent kernel takes work items from a queue in the
// order L1(chunk 0), L2(chunk 0), L1(chunk 1), L2(chunk 1), ...: the level-1
// tiles of chunk c scatter into c's scratch range, and the level-2 items of
// chunk c, one per bucket, run right after and read that range while it is
// still in L2 (one chunk of scratch, e.g. 58 MB for 512M int64 tuples over
// 148 chunks), then discard its lines from L2 so that they are never written
// back.  HBM sees the input once and the output once.
//
// Work items and waits: a level-1 item never waits.  A level-2 item of chunk
// c waits (bounded, kSpinLimit polls) until all level-1 items of c are done
// (a per-chunk counter, release/acquire); those items were handed out before
// it and are running or done, so the wait always ends.  A wait that gives up
// records kDevErrTimeout and skips its bucket.
//
// Scratch layout (chunks C, buckets FH = 2^hi, `work`):
//   tmp_start[C * FH] u64  first scratch slot of bucket (c, h)
//   bucket_len[C * FH] u32 tuples of bucket (c, h)
//   l1_cursor[C * FH] u32  slots claimed so far in bucket (c, h)
//   done[C] u32            finished level-1 tiles of chunk c
//   ticket u32             next work item
// `tmp` holds len tuples: bucket (c, h) at [c * clen + sum_{h' < h}
// bucket_len(c, h'), ...), so a chunk's buckets fill its input range.
#include <algorithm>

#include "common.cuh"
#include "kernels.h"
#include "tile_scatter.cuh"

namespace fi {

namespace {

template <typename K>
using PtlShape = TileWide<K>;

uint32_t ptl_hi_bits(uint32_t radix_bits) { return (radix_bits + 1) / 2; }

struct PtlWork {
  uint64_t *tmp_start;
  uint32_t *bucket_len;
  uint32_t *l1_cursor;
  uint32_t *done;
  uint32_t *ticket;
};

PtlWork ptl_work(void *work, uint32_t chunks, uint32_t hi) {
  const size_t n = (size_t)chunks << hi;
  char *p = static_cast<char *>(work);
  PtlWork w;
  w.tmp_start = reinterpret_cast<uint64_t *>(p);
  w.bucket_len = reinterpret_cast<uint32_t *>(p + n * 8);
  w.l1_cursor = w.bucket_len + n;
  w.done = w.l1_cursor + n;
  w.ticket = w.done + chunks;
  return w;
}

// Tuples of final region (c, p) under the cursor layout: Chunked offsets
// (region (c, p) ends where (c, p+1) starts minus padding, the chunk's last
// region where chunk c+1's first starts minus padding, the relation's last at
// its padded length), or Contiguous per-block cursors (block c's share of
// partition p ends where block c+1's share starts; the last block's where
// partition p+1 starts minus padding).
__device__ __forceinline__ uint64_t region_len(const uint64_t *cur, uint32_t c,
                                               uint32_t p, uint32_t chunks,
                                               uint32_t F, uint32_t pad,
                                               bool contiguous,
                                               uint64_t padded_len) {
  const uint64_t i = (uint64_t)c * F + p;
  uint64_t next;
  if (contiguous) {
    if (c + 1 < chunks)
      next = cur[i + F];
    else
      next = (p + 1 < F) ? cur[p + 1] - pad : padded_len;
  } else {
    if (p + 1 < F)
      next = cur[i + 1] - pad;
    else
      next = (c + 1 < chunks) ? cur[i + 1] - pad : padded_len;
  }
  return next - cur[i];
}

// One CTA per chunk: bucket lengths, their scratch starts, zeroed level-1
// cursors and counters.
__global__ void ptl_init_kernel(const uint64_t *__restrict__ cursors,
                                uint32_t chunks, uint32_t radix_bits,
                                uint32_t hi, uint32_t pad, bool contiguous,
                                uint64_t padded_len, uint64_t clen,
                                PtlWork w) {
  __shared__ uint64_t tmp[33];
  const uint32_t c = blockIdx.x, F = 1u << radix_bits, FH = 1u << hi;
  const uint32_t FL = F >> hi;
  uint64_t run = (uint64_t)c * clen;
  for (uint32_t h0 = 0; h0 < FH; h0 += blockDim.x) {
    const uint32_t h = h0 + threadIdx.x;
    uint64_t n = 0;
    if (h < FH)
      for (uint32_t l = 0; l < FL; ++l)
        n += region_len(cursors, c, h * FL + l, chunks, F, pad, contiguous,
                        padded_len);
    uint64_t total;
    const uint64_t ex = block_exclusive_scan_u64(n, tmp, &total);
    if (h < FH) {
      const uint64_t i = (uint64_t)c * FH + h;
      w.tmp_start[i] = run + ex;
      w.bucket_len[i] = (uint32_t)n;
      w.l1_cursor[i] = 0;
    }
    run += total;
  }
  if (threadIdx.x == 0) {
    w.done[c] = 0;
    if (c == 0) *w.ticket = 0;
  }
}

// Work item t -> (level 2?, chunk, index in the chunk's items).  Items:
// L1(0) [A], L2(0) [B], L1(1) [A], ..., L1(C-1) [Z], L2(C-1) [B], where A
// tiles make a full chunk, Z the last one, and B = FH buckets.
__device__ __forceinline__ bool ptl_decode(uint64_t t, uint32_t C, uint64_t A,
                                           uint64_t Z, uint64_t B, bool *l2,
                                           uint32_t *c, uint64_t *i) {
  const uint64_t AB = A + B, full = (uint64_t)(C - 1) * AB;
  if (t < full) {
    *c = (uint32_t)(t / AB);
    const uint64_t r = t % AB;
    *l2 = r >= A;
    *i = *l2 ? r - A : r;
    return true;
  }
  uint64_t v = t - full;
  *c = C - 1;
  if (v < Z) {
    *l2 = false;
    *i = v;
    return true;
  }
  v -= Z;
  *l2 = true;
  *i = v;
  return v < B;
}

__device__ __forceinline__ uint32_t ld_acquire_u32(const uint32_t *p) {
  uint32_t v;
  asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}

// Tuples of the scratch range, read at L2 (other SMs wrote them; this SM's L1
// may hold lines of an earlier use of the buffer).
template <typename K>
struct ScratchSource {
  const Tuple<K> *__restrict__ tuples;
  __device__ __forceinline__ void load(uint64_t i, K &k, K &v) {
    const Tuple<K> *p = tuples + i;
    if constexpr (sizeof(K) == 8) {
      longlong2 x = __ldcg(reinterpret_cast<const longlong2 *>(p));
      k = (K)x.x;
      v = (K)x.y;
    } else {
      int2 x = __ldcg(reinterpret_cast<const int2 *>(p));
      k = (K)x.x;
      v = (K)x.y;
    }
  }
};

// Drops the scratch lines that lie wholly inside [begin, end) (bytes) from L2
// without writing them back: their tuples have been consumed.
__device__ __forceinline__ void discard_lines(const void *begin, const void *end) {
  const uintptr_t b = (reinterpret_cast<uintptr_t>(begin) + 127u) & ~(uintptr_t)127u;
  const uintptr_t e = reinterpret_cast<uintptr_t>(end) & ~(uintptr_t)127u;
  for (uintptr_t a = b + (uintptr_t)threadIdx.x * 128u; a < e;
       a += (uintptr_t)blockDim.x * 128u)
    asm volatile("discard.global.L2 [%0], 128;" ::"l"(a) : "memory");
}

// Shared memory: staged tuples [kTile] | gbase [2^hi] u64 |
// toff [2^max(hi, lo) + 1] u32 | cur [2^lo] u32 | scan_tmp [33] u32.
template <typename K>
size_t ptl_smem(uint32_t hi, uint32_t lo) {
  using S = PtlShape<K>;
  const size_t f = (size_t)1 << std::max(hi, lo);
  return (size_t)S::kTile * sizeof(Tuple<K>) +
         ((size_t)1 << hi) * sizeof(uint64_t) +
         (f + 1 + ((size_t)1 << lo) + 33) * sizeof(uint32_t);
}

template <typename K>
__global__ void __launch_bounds__(PtlShape<K>::kThreads, PtlShape<K>::kMinBlocks)
    ptl_scatter_kernel(const K *__restrict__ keys, const K *__restrict__ pays,
                       uint64_t len, uint64_t clen, uint32_t chunks,
                       uint32_t hi, uint32_t lo, uint32_t ignore_bits,
                       const uint64_t *__restrict__ cursors,
                       Tuple<K> *__restrict__ out, uint64_t out_len,
                       Tuple<K> *__restrict__ tmp, PtlWork w, int *status) {
  using S = PtlShape<K>;
  constexpr uint32_t T = S::kThreads, I = S::kItems, kTile = S::kTile;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const uint32_t FH = 1u << hi, FL = 1u << lo, F = FH * FL;
  Tuple<K> *staged = reinterpret_cast<Tuple<K> *>(smem_raw);
  uint64_t *gbase = reinterpret_cast<uint64_t *>(staged + kTile);
  uint32_t *toff = reinterpret_cast<uint32_t *>(gbase + FH);
  uint32_t *cur = toff + (max(FH, FL) + 1);
  uint32_t *scan_tmp = cur + FL;
  __shared__ uint32_t s_ticket;
  __shared__ int s_ok;

  const uint64_t mask_hi = (uint64_t)(FH - 1u) << (ignore_bits + lo);
  const uint64_t mask_lo = (uint64_t)(FL - 1u) << ignore_bits;
  const uint64_t A = clen ? (clen + kTile - 1) / kTile : 0;
  const uint64_t last_len = len - clen * (chunks - 1);
  const uint64_t Z = (last_len + kTile - 1) / kTile;
  const uint32_t tid = threadIdx.x;

  for (uint32_t p = tid; p <= max(FH, FL); p += T) toff[p] = 0;
  for (;;) {
    __syncthreads();
    if (tid == 0) s_ticket = atomicAdd(w.ticket, 1u);
    __syncthreads();
    bool level2;
    uint32_t c;
    uint64_t idx;
    if (!ptl_decode(s_ticket, chunks, A, Z, FH, &level2, &c, &idx)) break;
    const uint64_t cbegin = (uint64_t)c * clen;
    const uint64_t cend = (c + 1 < chunks) ? cbegin + clen : len;
    if (!level2) {
      // ---- level 1: one tile of chunk c, sorted by bucket into scratch ----
      const uint64_t t0 = cbegin + idx * kTile;
      const uint32_t n = (uint32_t)min((uint64_t)kTile, cend - t0);
      K ck[I], cv[I];
      uint32_t hh[I], rk[I];
#pragma unroll
      for (uint32_t u = 0; u < I; ++u) {
        const uint32_t j = u * T + tid;
        const bool act = j < n;
        if (act) {
          ck[u] = load_cs(keys + t0 + j);
          cv[u] = load_cs(pays + t0 + j);
        }
        hh[u] = act ? key_to_partition(ck[u], mask_hi, ignore_bits + lo) : 0u;
        rk[u] = warp_aggregated_rank(toff, hh[u], act);
      }
      __syncthreads();
      block_exclusive_scan_u32(toff, FH, scan_tmp);
      if (tid == 0) toff[FH] = n;
      __syncthreads();
      // claim each bucket's run in the chunk's scratch range
      for (uint32_t h = tid; h < FH; h += T) {
        const uint32_t cnt = toff[h + 1] - toff[h];
        if (cnt) {
          const uint64_t b = (uint64_t)c * FH + h;
          gbase[h] = w.tmp_start[b] + atomicAdd(&w.l1_cursor[b], cnt);
        }
      }
#pragma unroll
      for (uint32_t u = 0; u < I; ++u)
        if (u * T + tid < n) staged[toff[hh[u]] + rk[u]] = Tuple<K>{ck[u], cv[u]};
      __syncthreads();
      for (uint32_t j = tid; j < n; j += T) {
        const Tuple<K> t = staged[j];
        const uint32_t h = key_to_partition(t.key, mask_hi, ignore_bits + lo);
        const uint64_t dst = gbase[h] + (j - toff[h]);
        if (dst < len)
          store_tuple(tmp + dst, t);
        else
          record_error(status, kDevErrCapacity);
      }
      __syncthreads();
      for (uint32_t p = tid; p <= FH; p += T) toff[p] = 0;
      if (tid == 0) {
        __threadfence();  // this tile's scratch stores before the count
        atomicAdd(&w.done[c], 1u);
      }
    } else {
      // ---- level 2: bucket (c, idx), once chunk c's level 1 is done ----
      const uint32_t h = (uint32_t)idx;
      const uint64_t b = (uint64_t)c * FH + h;
      const uint32_t need = (uint32_t)((cend - cbegin + kTile - 1) / kTile);
      if (tid == 0) {
        int ok = 0;
        for (uint32_t it = 0; it < kSpinLimit; ++it) {
          if (ld_acquire_u32(&w.done[c]) >= need) {
            ok = 1;
            break;
          }
          spin_pause(it);
        }
        if (!ok) record_error(status, kDevErrTimeout);
        s_ok = ok;
      }
      __syncthreads();
      const uint32_t n = w.bucket_len[b];
      if (!s_ok || n == 0) continue;
      const uint64_t ts = w.tmp_start[b];
      const uint64_t *cp = cursors + (uint64_t)c * F + (uint64_t)h * FL;
      const uint64_t base = cp[0];
      for (uint32_t l = tid; l < FL; l += T) cur[l] = (uint32_t)(cp[l] - base);
      __syncthreads();
      ScratchSource<K> src{tmp};
      tile_scatter_range<K, S>(src, ts, ts + n, FL, mask_lo, ignore_bits, cur,
                               toff, scan_tmp, staged, out, base, out_len,
                               status);
      discard_lines(tmp + ts, tmp + ts + n);
    }
  }
}

}  // namespace

size_t pipelined_scatter_work_bytes(uint32_t chunks, uint32_t radix_bits) {
  const size_t n = (size_t)chunks << ptl_hi_bits(radix_bits);
  return n * 8 + n * 4 + n * 4 + (size_t)chunks * 4 + 16;
}

template <typename K>
cudaError_t launch_partition_pipelined(
    const K *keys, const K *pays, uint64_t len, uint32_t chunks,
    uint32_t radix_bits, uint32_t ignore_bits, const uint64_t *cursors,
    bool contiguous, uint64_t padded_len, void *out, uint64_t out_len,
    void *tmp, void *work, int *status, uint32_t sm_count, cudaStream_t stream) {
  using S = PtlShape<K>;
  constexpr uint64_t kAlignMask = ~((uint64_t)(kAlignBytes / sizeof(K)) - 1ull);
  const uint64_t clen = ((len + chunks - 1) / chunks) & kAlignMask;
  const uint32_t hi = ptl_hi_bits(radix_bits), lo = radix_bits - hi;
  const PtlWork w = ptl_work(work, chunks, hi);
  const uint32_t pad = (uint32_t)(kPaddingBytes / sizeof(Tuple<K>));
  ptl_init_kernel<<<chunks, 256, 0, stream>>>(cursors, chunks, radix_bits, hi, pad,
                                              contiguous, padded_len, clen, w);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return e;
  const size_t sm = ptl_smem<K>(hi, lo);
  e = cudaFuncSetAttribute((const void *)ptl_scatter_kernel<K>,
                           cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
  if (e != cudaSuccess) return e;
  int per_sm = 0;
  e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(
      &per_sm, (const void *)ptl_scatter_kernel<K>, (int)S::kThreads, sm);
  if (e != cudaSuccess) return e;
  const uint32_t grid = (uint32_t)std::max(per_sm, 1) * sm_count;
  ptl_scatter_kernel<K><<<grid, S::kThreads, sm, stream>>>(
      keys, pays, len, clen, chunks, hi, lo, ignore_bits, cursors,
      reinterpret_cast<Tuple<K> *>(out), out_len, reinterpret_cast<Tuple<K> *>(tmp),
      w, status);
  return cudaGetLastError();
}

#define FI_INSTANTIATE_PIPELINED(K)                                              \
  template cudaError_t launch_partition_pipelined<K>(                            \
      const K *, const K *, uint64_t, uint32_t, uint32_t, uint32_t,              \
      const uint64_t *, bool, uint64_t, void *, uint64_t, void *, void *, int *, \
      uint32_t, cudaStream_t);

FI_INSTANTIATE_PIPELINED(int32_t)
FI_INSTANTIATE_PIPELINED(int64_t)

}  // namespace fi
