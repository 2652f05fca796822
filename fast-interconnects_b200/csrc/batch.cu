// Batched small radix joins on one B200 (no reference counterpart: the
// reference runs one join per gpu_radix_join call,
// radix-join/src/execution_methods/gpu_radix_join.rs:90-565, and its
// nearest piece to a work queue is the greedy task assignment of
// sql-ops/cudautils/radix_join.cu:58-98).
//
// A join below a few million tuples cannot fill 148 SMs, and through the
// plain engine it pays about twenty launches and their latencies.  The batch
// path runs up to hundreds of such joins at once, as four kernels over the
// whole batch:
//
//   1. histogram: grid-stride over 4096-tuple tiles of all jobs' R and S;
//      a shared-memory histogram per tile, flushed with global atomics
//      into the job's counters;
//   2. scan: one CTA per (job, relation) turns the counters into partition
//      offsets and claim cursors inside the job's arena region;
//   3. scatter: per tile, shared-memory counting sort by partition, one
//      global atomic claim per (tile, partition) run, then stores of whole
//      tuples into the arena (AoS, no padding);
//   4. join: persistent CTAs take (job, partition) items from a device work
//      queue, build a bucket-chaining table of the build partition in
//      shared memory (in rounds when it exceeds the table) and probe the
//      probe partition, adding matches and payload sums to the job's result.
//
// Results are per job: the wrapping sum of the matched probe payloads and
// the match count, the same as the engine and the CPU radix join.
#include <algorithm>
#include <cstring>

#include "../../include/fi_sqlops.h"
#include "api_internal.h"
#include "batch.h"
#include "common.cuh"
#include "kernels.h"

namespace fi {

constexpr uint32_t kBatchThreads = 512;
constexpr uint32_t kBatchItems = kBatchTile / kBatchThreads;  // per thread

// Shared-memory join table per key type: capacity (build tuples per round)
// and buckets.  Two CTAs per SM.
template <typename K>
struct BatchTable;
template <>
struct BatchTable<int64_t> {
  static constexpr uint32_t kCap = 6144, kLogBuckets = 12;
};
template <>
struct BatchTable<int32_t> {
  static constexpr uint32_t kCap = 8192, kLogBuckets = 12;
};
template <typename K>
constexpr size_t batch_join_smem() {
  return (size_t)BatchTable<K>::kCap * (sizeof(K) + 4) +
         ((size_t)4 << BatchTable<K>::kLogBuckets);
}

uint32_t batch_bits(uint64_t build_len) {
  uint32_t b = 0;
  while (b < kBatchMaxBits && (build_len >> b) > 3072) ++b;
  return b;
}

// Job j and relation (0 = R, 1 = S) of global tile t, and the tile's tuple
// range.  tile_r/tile_s are staged in shared memory.
__device__ __forceinline__ void batch_locate_tile(
    uint32_t t, uint32_t jobs, const uint32_t *tile_r, const uint32_t *tile_s,
    const BatchJobDesc *desc, uint32_t &j, uint32_t &rel, uint64_t &begin,
    uint64_t &end) {
  uint32_t lo = 0, hi = jobs;  // last job with tile_r[j] <= t
  while (hi - lo > 1) {
    const uint32_t mid = (lo + hi) >> 1;
    if (tile_r[mid] <= t) lo = mid; else hi = mid;
  }
  j = lo;
  rel = t >= tile_s[j] ? 1u : 0u;
  const uint64_t local = (uint64_t)(t - (rel ? tile_s[j] : tile_r[j])) * kBatchTile;
  const uint64_t n = rel ? desc[j].sn : desc[j].rn;
  begin = local;
  end = min(n, local + kBatchTile);
}

__device__ __forceinline__ void batch_stage_tables(const BatchHeader *head,
                                                   const BatchJobDesc *desc,
                                                   uint32_t *tile_r,
                                                   uint32_t *tile_s) {
  const uint32_t jobs = head->jobs;
  for (uint32_t j = threadIdx.x; j < jobs; j += blockDim.x) {
    tile_r[j] = desc[j].tile_r;
    tile_s[j] = desc[j].tile_s;
  }
  __syncthreads();
}

template <typename K>
__global__ void __launch_bounds__(kBatchThreads)
    batch_hist_kernel(const BatchHeader *__restrict__ head,
                      const BatchJobDesc *__restrict__ desc,
                      uint32_t *__restrict__ counts) {
  __shared__ uint32_t tile_r[kBatchMaxJobs], tile_s[kBatchMaxJobs];
  __shared__ uint32_t hist[1u << kBatchMaxBits];
  batch_stage_tables(head, desc, tile_r, tile_s);
  const uint32_t jobs = head->jobs, tiles = head->tiles;
  for (uint32_t t = blockIdx.x; t < tiles; t += gridDim.x) {
    uint32_t j, rel;
    uint64_t b, e;
    batch_locate_tile(t, jobs, tile_r, tile_s, desc, j, rel, b, e);
    const uint32_t F = 1u << desc[j].bits;
    const K *keys = reinterpret_cast<const K *>(rel ? desc[j].sk : desc[j].rk);
    for (uint32_t p = threadIdx.x; p < F; p += blockDim.x) hist[p] = 0;
    __syncthreads();
    const uint64_t mask = (uint64_t)F - 1u;
    for (uint64_t i = b + threadIdx.x; i < e; i += blockDim.x)
      atomicAdd(&hist[key_to_partition(keys[i], mask, 0)], 1u);
    __syncthreads();
    uint32_t *dst = counts + desc[j].cnt_base + rel * F;
    for (uint32_t p = threadIdx.x; p < F; p += blockDim.x)
      if (hist[p]) atomicAdd(&dst[p], hist[p]);
    __syncthreads();
  }
}

// One CTA per (job, relation): exclusive scan of the counters.
__global__ void __launch_bounds__(1024)
    batch_scan_kernel(const BatchHeader *__restrict__ head,
                      const BatchJobDesc *__restrict__ desc,
                      const uint32_t *__restrict__ counts,
                      uint32_t *__restrict__ offs, uint32_t *__restrict__ curs) {
  __shared__ uint32_t cnt[(1u << kBatchMaxBits) + 33];
  const uint32_t j = blockIdx.x >> 1, rel = blockIdx.x & 1u;
  if (j >= head->jobs) return;
  const uint32_t F = 1u << desc[j].bits;
  const uint32_t base = desc[j].cnt_base + rel * F;
  for (uint32_t p = threadIdx.x; p < F; p += blockDim.x) cnt[p] = counts[base + p];
  __syncthreads();
  block_exclusive_scan_u32(cnt, F, cnt + (1u << kBatchMaxBits));
  for (uint32_t p = threadIdx.x; p < F; p += blockDim.x) {
    offs[base + p] = cnt[p];
    curs[base + p] = cnt[p];
  }
}

}  // namespace fi

namespace fi {

template <typename K>
__global__ void __launch_bounds__(kBatchThreads)
    batch_scatter_kernel(const BatchHeader *__restrict__ head,
                         const BatchJobDesc *__restrict__ desc,
                         uint32_t *__restrict__ curs,
                         Tuple<K> *__restrict__ arena) {
  __shared__ uint32_t tile_r[kBatchMaxJobs], tile_s[kBatchMaxJobs];
  __shared__ uint32_t cnt[1u << kBatchMaxBits];
  batch_stage_tables(head, desc, tile_r, tile_s);
  const uint32_t jobs = head->jobs, tiles = head->tiles;
  for (uint32_t t = blockIdx.x; t < tiles; t += gridDim.x) {
    uint32_t j, rel;
    uint64_t b, e;
    batch_locate_tile(t, jobs, tile_r, tile_s, desc, j, rel, b, e);
    const uint32_t F = 1u << desc[j].bits;
    const uint64_t mask = (uint64_t)F - 1u;
    const K *keys = reinterpret_cast<const K *>(rel ? desc[j].sk : desc[j].rk);
    const K *pays = reinterpret_cast<const K *>(rel ? desc[j].sp : desc[j].rp);
    for (uint32_t p = threadIdx.x; p < F; p += blockDim.x) cnt[p] = 0;
    __syncthreads();
    K k[kBatchItems], v[kBatchItems];
    uint32_t part[kBatchItems], rank[kBatchItems];
#pragma unroll
    for (uint32_t u = 0; u < kBatchItems; ++u) {
      const uint64_t i = b + (uint64_t)u * blockDim.x + threadIdx.x;
      if (i < e) {
        k[u] = keys[i];
        v[u] = pays[i];
        part[u] = key_to_partition(k[u], mask, 0);
        rank[u] = atomicAdd(&cnt[part[u]], 1u);
      }
    }
    __syncthreads();
    // claim one run per partition of this tile; cnt becomes the run's start
    uint32_t *cur = curs + desc[j].cnt_base + rel * F;
    for (uint32_t p = threadIdx.x; p < F; p += blockDim.x)
      if (cnt[p]) cnt[p] = atomicAdd(&cur[p], cnt[p]);
    __syncthreads();
    Tuple<K> *out = arena + (rel ? desc[j].out_s : desc[j].out_r);
#pragma unroll
    for (uint32_t u = 0; u < kBatchItems; ++u) {
      const uint64_t i = b + (uint64_t)u * blockDim.x + threadIdx.x;
      if (i < e) store_tuple(out + cnt[part[u]] + rank[u], Tuple<K>{k[u], v[u]});
    }
    __syncthreads();
  }
}

// Persistent join over (job, partition) items taken from a work queue.
template <typename K>
__global__ void __launch_bounds__(kBatchThreads, 2)
    batch_join_kernel(const BatchHeader *__restrict__ head,
                      const BatchJobDesc *__restrict__ desc,
                      const uint32_t *__restrict__ offs,
                      const Tuple<K> *__restrict__ arena,
                      uint32_t *__restrict__ queue,
                      BatchJobResult *__restrict__ res) {
  using T = BatchTable<K>;
  constexpr uint32_t kBuckets = 1u << T::kLogBuckets;
  constexpr uint32_t kEmpty = 0xffffffffu;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  K *tkeys = reinterpret_cast<K *>(smem_raw);
  uint32_t *tnext = reinterpret_cast<uint32_t *>(tkeys + T::kCap);
  uint32_t *heads = tnext + T::kCap;
  __shared__ uint32_t item_base[kBatchMaxJobs];
  __shared__ uint32_t item_s;
  __shared__ uint64_t red[32];
  const uint32_t jobs = head->jobs, items = head->items;
  for (uint32_t j = threadIdx.x; j < jobs; j += blockDim.x)
    item_base[j] = desc[j].item_base;
  for (;;) {
    __syncthreads();
    if (threadIdx.x == 0) item_s = atomicAdd(queue, 1u);
    __syncthreads();
    const uint32_t it = item_s;
    if (it >= items) break;
    uint32_t lo = 0, hi = jobs;  // last job with item_base[j] <= it
    while (hi - lo > 1) {
      const uint32_t mid = (lo + hi) >> 1;
      if (item_base[mid] <= it) lo = mid; else hi = mid;
    }
    const uint32_t j = lo, p = it - item_base[j];
    const uint32_t bits = desc[j].bits, F = 1u << bits;
    const uint32_t cb = desc[j].cnt_base;
    const uint64_t rb = offs[cb + p];
    const uint64_t re = p + 1 < F ? offs[cb + p + 1] : desc[j].rn;
    const uint64_t sb = offs[cb + F + p];
    const uint64_t se = p + 1 < F ? offs[cb + F + p + 1] : desc[j].sn;
    const Tuple<K> *R = arena + desc[j].out_r;
    const Tuple<K> *S = arena + desc[j].out_s;
    uint64_t sum = 0, cnt = 0;
    if (re > rb && se > sb) {
      for (uint64_t r0 = rb; r0 < re; r0 += T::kCap) {
        const uint32_t m = (uint32_t)min((uint64_t)T::kCap, re - r0);
        for (uint32_t i = threadIdx.x; i < kBuckets; i += blockDim.x) heads[i] = kEmpty;
        __syncthreads();
        for (uint32_t i = threadIdx.x; i < m; i += blockDim.x) {
          const K key = R[r0 + i].key;
          const uint32_t h =
              (uint32_t)(((uint64_t)(int64_t)key >> bits) & (kBuckets - 1u));
          tkeys[i] = key;
          tnext[i] = atomicExch(&heads[h], i);
        }
        __syncthreads();
        // every chain ends in kEmpty: each slot was linked in exactly once
        for (uint64_t i = sb + threadIdx.x; i < se; i += blockDim.x) {
          const Tuple<K> s = load_tuple(S + i);
          const uint32_t h =
              (uint32_t)(((uint64_t)(int64_t)s.key >> bits) & (kBuckets - 1u));
          for (uint32_t x = heads[h]; x != kEmpty; x = tnext[x]) {
            if (tkeys[x] == s.key) {
              sum += (uint64_t)(int64_t)s.value;
              ++cnt;
            }
          }
        }
        __syncthreads();
      }
    }
    sum = block_reduce_u64(sum, red);
    cnt = block_reduce_u64(cnt, red);
    if (threadIdx.x == 0 && cnt) {
      atomicAdd((unsigned long long *)&res[j].sum, (unsigned long long)sum);
      atomicAdd((unsigned long long *)&res[j].count, (unsigned long long)cnt);
    }
  }
}

}  // namespace fi

// ---- runner -------------------------------------------------------------------
namespace fi {

namespace {
uint64_t ceil_div(uint64_t a, uint64_t b) { return (a + b - 1) / b; }
}  // namespace

#define FI_BCK(expr)                          \
  do {                                        \
    cudaError_t e_ = (expr);                  \
    if (e_ != cudaSuccess) {                  \
      cudaGetLastError();                     \
      return cuda_error(e_, "batch runner");  \
    }                                         \
  } while (0)

static size_t desc_bytes(uint32_t max_jobs) {
  return 64 + (size_t)max_jobs * sizeof(BatchJobDesc);
}

int BatchRunner::init(uint32_t key_bytes, uint32_t max_jobs,
                      uint64_t max_tuples, uint32_t sm_count, int priority) {
  if (key_bytes != 4 && key_bytes != 8)
    return set_error(FI_ERR_INVALID_ARGUMENT, "key_bytes must be 4 or 8");
  if (max_jobs == 0 || max_jobs > kBatchMaxJobs)
    return set_error(FI_ERR_INVALID_ARGUMENT, "max_jobs must lie in [1, %u]",
                     kBatchMaxJobs);
  if (max_tuples == 0 || max_tuples >= (1ull << 32))
    return set_error(FI_ERR_INVALID_ARGUMENT, "max_tuples must lie in [1, 2^32)");
  release();
  key_bytes_ = key_bytes;
  max_jobs_ = max_jobs;
  max_tuples_ = max_tuples;
  sm_count_ = sm_count;
  max_counters_ = (uint64_t)max_jobs * 2u << kBatchMaxBits;
  const size_t db = desc_bytes(max_jobs);
  FI_BCK(cudaStreamCreateWithPriority(&stream_, cudaStreamNonBlocking, priority));
  FI_BCK(cudaEventCreateWithFlags(&done_, cudaEventDisableTiming));
  void *p = nullptr;
  FI_BCK(cudaMalloc(&p, db));
  d_head_ = (BatchHeader *)p;
  d_desc_ = (BatchJobDesc *)((unsigned char *)p + 64);
  FI_BCK(cudaMalloc((void **)&d_counts_, max_counters_ * 4));
  FI_BCK(cudaMalloc((void **)&d_offs_, max_counters_ * 4));
  FI_BCK(cudaMalloc((void **)&d_curs_, max_counters_ * 4));
  FI_BCK(cudaMalloc((void **)&d_queue_, 16));
  FI_BCK(cudaMalloc(&d_arena_, max_tuples * 2 * key_bytes));
  FI_BCK(cudaMalloc((void **)&d_res_, (size_t)max_jobs * sizeof(BatchJobResult)));
  FI_BCK(cudaHostAlloc((void **)&host_desc_, db, cudaHostAllocDefault));
  FI_BCK(cudaHostAlloc((void **)&host_res_,
                       (size_t)max_jobs * sizeof(BatchJobResult),
                       cudaHostAllocDefault));
  std::memset(host_desc_, 0, db);
  bytes_ = db + 3 * max_counters_ * 4 + 16 + max_tuples * 2 * key_bytes +
           (uint64_t)max_jobs * sizeof(BatchJobResult);
  return capture();
}

template <typename K>
static void batch_enqueue(cudaStream_t st, uint32_t max_jobs, uint32_t sm,
                          BatchHeader *head, BatchJobDesc *desc,
                          uint32_t *counts, uint32_t *offs, uint32_t *curs,
                          void *arena, uint32_t *queue, BatchJobResult *res) {
  batch_hist_kernel<K><<<sm * 4, kBatchThreads, 0, st>>>(head, desc, counts);
  batch_scan_kernel<<<max_jobs * 2, 1024, 0, st>>>(head, desc, counts, offs, curs);
  batch_scatter_kernel<K><<<sm * 4, kBatchThreads, 0, st>>>(
      head, desc, curs, reinterpret_cast<Tuple<K> *>(arena));
  batch_join_kernel<K><<<sm * 2, kBatchThreads, batch_join_smem<K>(), st>>>(
      head, desc, offs, reinterpret_cast<const Tuple<K> *>(arena), queue, res);
}

int BatchRunner::capture() {
  if (key_bytes_ == 8)
    FI_BCK(cudaFuncSetAttribute((const void *)batch_join_kernel<int64_t>,
                                cudaFuncAttributeMaxDynamicSharedMemorySize,
                                (int)batch_join_smem<int64_t>()));
  else
    FI_BCK(cudaFuncSetAttribute((const void *)batch_join_kernel<int32_t>,
                                cudaFuncAttributeMaxDynamicSharedMemorySize,
                                (int)batch_join_smem<int32_t>()));
  cudaGraph_t graph = nullptr;
  FI_BCK(cudaStreamBeginCapture(stream_, cudaStreamCaptureModeThreadLocal));
  cudaMemcpyAsync(d_head_, host_desc_, desc_bytes(max_jobs_),
                  cudaMemcpyHostToDevice, stream_);
  cudaMemsetAsync(d_counts_, 0, max_counters_ * 4, stream_);
  cudaMemsetAsync(d_res_, 0, (size_t)max_jobs_ * sizeof(BatchJobResult), stream_);
  cudaMemsetAsync(d_queue_, 0, 16, stream_);
  if (key_bytes_ == 8)
    batch_enqueue<int64_t>(stream_, max_jobs_, sm_count_, d_head_, d_desc_,
                           d_counts_, d_offs_, d_curs_, d_arena_, d_queue_, d_res_);
  else
    batch_enqueue<int32_t>(stream_, max_jobs_, sm_count_, d_head_, d_desc_,
                           d_counts_, d_offs_, d_curs_, d_arena_, d_queue_, d_res_);
  cudaMemcpyAsync(host_res_, d_res_, (size_t)max_jobs_ * sizeof(BatchJobResult),
                  cudaMemcpyDeviceToHost, stream_);
  cudaError_t ce = cudaStreamEndCapture(stream_, &graph);
  if (ce != cudaSuccess) {
    if (graph) cudaGraphDestroy(graph);
    return cuda_error(ce, "batch graph capture");
  }
  ce = cudaGraphInstantiate(&exec_, graph, 0);
  cudaGraphDestroy(graph);
  if (ce != cudaSuccess) return cuda_error(ce, "batch graph instantiate");
  return FI_OK;
}

bool BatchRunner::fits(const BatchJob *jobs, uint32_t n) const {
  if (n > max_jobs_) return false;
  uint64_t tuples = 0;
  for (uint32_t i = 0; i < n; ++i) {
    if (jobs[i].bits > kBatchMaxBits) return false;
    tuples += jobs[i].rn + jobs[i].sn;
  }
  return tuples <= max_tuples_;
}

int BatchRunner::launch(const BatchJob *jobs, uint32_t n) {
  if (!exec_) return set_error(FI_ERR_RUNTIME, "batch runner not initialised");
  if (!fits(jobs, n))
    return set_error(FI_ERR_CAPACITY, "jobs exceed the batch's capacity");
  auto *head = reinterpret_cast<BatchHeader *>(host_desc_);
  auto *desc = reinterpret_cast<BatchJobDesc *>(host_desc_ + 64);
  uint64_t tuples = 0;
  uint32_t counters = 0, tiles = 0, items = 0;
  for (uint32_t i = 0; i < n; ++i) {
    const BatchJob &b = jobs[i];
    BatchJobDesc &d = desc[i];
    d.rk = b.rk; d.rp = b.rp; d.sk = b.sk; d.sp = b.sp;
    d.rn = b.rn; d.sn = b.sn;
    d.bits = b.bits;
    d.out_r = tuples;
    d.out_s = tuples + b.rn;
    tuples += b.rn + b.sn;
    d.cnt_base = counters;
    counters += 2u << b.bits;
    d.tile_r = tiles;
    d.tile_s = tiles + (uint32_t)ceil_div(b.rn, kBatchTile);
    tiles = d.tile_s + (uint32_t)ceil_div(b.sn, kBatchTile);
    d.item_base = items;
    items += 1u << b.bits;
    d.pad_ = 0;
  }
  head->jobs = n;
  head->tiles = tiles;
  head->items = items;
  head->counters = counters;
  FI_BCK(cudaGraphLaunch(exec_, stream_));
  FI_BCK(cudaEventRecord(done_, stream_));
  return FI_OK;
}

void BatchRunner::release() {
  if (exec_) cudaGraphExecDestroy(exec_);
  if (d_head_) cudaFree(d_head_);
  if (d_counts_) cudaFree(d_counts_);
  if (d_offs_) cudaFree(d_offs_);
  if (d_curs_) cudaFree(d_curs_);
  if (d_queue_) cudaFree(d_queue_);
  if (d_arena_) cudaFree(d_arena_);
  if (d_res_) cudaFree(d_res_);
  if (host_desc_) cudaFreeHost(host_desc_);
  if (host_res_) cudaFreeHost(host_res_);
  if (done_) cudaEventDestroy(done_);
  if (stream_) cudaStreamDestroy(stream_);
  exec_ = nullptr;
  d_head_ = nullptr; d_desc_ = nullptr; d_counts_ = d_offs_ = d_curs_ = nullptr;
  d_queue_ = nullptr; d_arena_ = nullptr; d_res_ = nullptr;
  host_desc_ = nullptr; host_res_ = nullptr; done_ = nullptr; stream_ = nullptr;
  bytes_ = 0;
  busy_ = false;
}

}  // namespace fi

// ---- C ABI ----------------------------------------------------------------------
struct fi_join_batch {
  fi::BatchRunner runner;
};

extern "C" int fi_join_batch_new(uint32_t tuple_bytes, uint32_t max_jobs,
                                 uint64_t max_tuples, fi_join_batch **out) {
  using namespace fi;
  if (!out) return set_error(FI_ERR_INVALID_ARGUMENT, "null output handle");
  *out = nullptr;
  if (tuple_bytes != 8 && tuple_bytes != 16)
    return set_error(FI_ERR_INVALID_ARGUMENT, "tuple_bytes must be 8 or 16");
  auto *b = new fi_join_batch();
  int rc = b->runner.init(tuple_bytes / 2, max_jobs, max_tuples,
                          (uint32_t)device_sm_count());
  if (rc) {
    delete b;
    return rc;
  }
  *out = b;
  return FI_OK;
}

extern "C" void fi_join_batch_free(fi_join_batch *b) { delete b; }

extern "C" uint64_t fi_join_batch_device_bytes(const fi_join_batch *b) {
  return b ? b->runner.device_bytes() : 0;
}

extern "C" int fi_join_batch_run(fi_join_batch *b, const fi_batch_job *jobs,
                                 uint32_t n_jobs, fi_join_result *results) {
  using namespace fi;
  if (!b || (n_jobs && (!jobs || !results)))
    return set_error(FI_ERR_INVALID_ARGUMENT, "null argument");
  std::vector<BatchJob> js(n_jobs);
  for (uint32_t i = 0; i < n_jobs; ++i) {
    const fi_batch_job &j = jobs[i];
    if ((j.build_len && (!j.build_key || !j.build_pay)) ||
        (j.probe_len && (!j.probe_key || !j.probe_pay)))
      return set_error(FI_ERR_INVALID_ARGUMENT, "job %u has a null column", i);
    if (j.radix_bits > (int32_t)kBatchMaxBits)
      return set_error(FI_ERR_UNSUPPORTED, "batched joins use at most %u radix bits",
                       kBatchMaxBits);
    js[i] = BatchJob{j.build_key, j.build_pay, j.probe_key, j.probe_pay,
                     j.build_len, j.probe_len,
                     j.radix_bits < 0 ? batch_bits(j.build_len) : (uint32_t)j.radix_bits};
  }
  if (!b->runner.fits(js.data(), n_jobs))
    return set_error(FI_ERR_CAPACITY,
                     "the jobs exceed the batch (at most %u jobs and %llu tuples)",
                     b->runner.max_jobs(),
                     (unsigned long long)b->runner.max_tuples());
  int rc = b->runner.launch(js.data(), n_jobs);
  if (rc) return rc;
  cudaError_t ce = cudaEventSynchronize(b->runner.done());
  if (ce != cudaSuccess) return cuda_error(ce, "batch");
  for (uint32_t i = 0; i < n_jobs; ++i) {
    results[i].sum = (int64_t)b->runner.results()[i].sum;
    results[i].count = b->runner.results()[i].count;
  }
  return FI_OK;
}
