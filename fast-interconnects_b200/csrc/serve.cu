// Join server: continuous batching of radix joins on one B200.
//
// No reference counterpart: the reference's execution method runs one join
// per call with two reused StreamStates (gpu_radix_join.rs:51-68,321-396).
// The server admits requests of uneven sizes as they arrive and keeps the
// GPU busy with several of them at once:
//
//  * memory: the engines and batch arenas are allocated at start; the rest
//    of the budget is one device slab for the relations the server holds,
//    handed out by a host-side first-fit allocator, so admitting a request
//    calls no CUDA allocator and frees nothing that the GPU still reads.
//  * admission: a request is admitted when its relations (when the server
//    holds them) get a block of the slab.  Requests are admitted in arrival
//    order within two queues, small joins first, so that they need not wait
//    behind a large one that waits for memory; one larger than the whole
//    slab fails with FI_ERR_CAPACITY.
//  * loading: server-held relations (host or synthetic sources) are copied
//    or generated: those of small joins at admission on a high-priority load
//    stream (an event marks them ready), those of large joins on their
//    worker's stream just before the join.
//  * small joins (|R| + |S| below small_tuples) queue for a batch runner of
//    their key type.  A free runner takes the queue (up to its capacity)
//    when the other runner of the type is idle, the queue holds a quarter
//    of a batch, or its oldest job has waited batch_wait_us, and replays its
//    captured graph.  Two runners per key type alternate, so a batch forms
//    while the previous one runs.
//  * large joins run on a worker: a resident engine on its own stream,
//    planned by the autotuner, built once and probed in slices of
//    probe_slice tuples.  A free worker takes the shortest admitted large
//    join (or one that has waited over 0.5 s); a worker keeps two joins
//    enqueued on its stream, so the next starts without a host round trip,
//    and the one after is loaded on a load stream while they run.  Workers
//    overlap with each other and with batches.  By default two workers (one
//    when two engines would take over half the budget): their large joins
//    fill each other's idle phases (launch gaps, short kernels, tails).
//  * completion: the scheduler thread polls the done events, releases the
//    reservation and the relations, and hands responses to waiters.
#include <algorithm>
#include <chrono>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <map>
#include <mutex>
#include <thread>
#include <unordered_map>
#include <vector>

#include "../../include/fi_sqlops.h"
#include "api_internal.h"
#include "batch.h"
#include "kernels.h"

namespace fi {

// The autotuner's model plan (autotune.cu).
void autotune_model(uint64_t build_len, fi_tuned_plan *out);

namespace {

using Clock = std::chrono::steady_clock;

double us_between(Clock::time_point a, Clock::time_point b) {
  return std::chrono::duration<double, std::micro>(b - a).count();
}

struct Request {
  fi_join_request req{};
  fi_tuned_plan plan{};
  uint64_t reserve = 0;        // bytes of the budget this request holds
  void *block = nullptr;       // its block of the relation arena
  void *owned[4] = {};         // server-held relation columns (in block)
  const void *cols[4] = {};    // columns the join reads (device)
  cudaEvent_t ready = nullptr; // relations loaded
  cudaStream_t load = nullptr; // stream that loaded (and frees) them
  bool small = false;
  bool loaded = false;         // its load is enqueued
  Clock::time_point t_submit, t_admit;
  fi_join_response resp{};
  bool done = false;
};

constexpr uint32_t kMaxSlices = 64;

// One large join enqueued on a worker: its timing events and result
// buffers.
struct Slot {
  cudaEvent_t start = nullptr, done = nullptr;
  fi_join_result *d_res = nullptr;  // [kMaxSlices]
  fi_join_result *h_res = nullptr;  // pinned [kMaxSlices + 1]; the engine's
                                    // error word after the last slice
  uint32_t slices = 0;
  Request *req = nullptr;
};

// A worker keeps up to kWorkerSlots large joins enqueued on its stream: the
// next one waits on the stream behind the running one (stream order keeps
// the shared engine safe), so the GPU does not idle while the host notices
// a completion and enqueues the next join.
constexpr uint32_t kWorkerSlots = 2;

struct Worker {
  fi_radix_join_engine *engine = nullptr;
  cudaStream_t stream = nullptr;
  Slot slot[kWorkerSlots];
  uint32_t head = 0;   // oldest enqueued slot
  uint32_t count = 0;  // slots enqueued
};

// Host-side first-fit allocator over one device slab that holds the
// relations of admitted requests: admission never calls the CUDA allocator,
// and a block is only handed out again after the host has seen the work of
// its previous owner complete.
class Arena {
 public:
  static constexpr uint64_t kAlign = 256;
  void init(void *base, uint64_t size) {
    base_ = (unsigned char *)base;
    free_.clear();
    if (size) free_[0] = size;
  }
  void *alloc(uint64_t bytes) {
    bytes = round(bytes);
    for (auto it = free_.begin(); it != free_.end(); ++it) {
      if (it->second < bytes) continue;
      const uint64_t off = it->first, left = it->second - bytes;
      free_.erase(it);
      if (left) free_[off + bytes] = left;
      return base_ + off;
    }
    return nullptr;
  }
  void release(void *p, uint64_t bytes) {
    uint64_t off = (uint64_t)((unsigned char *)p - base_), len = round(bytes);
    auto next = free_.lower_bound(off);
    if (next != free_.end() && off + len == next->first) {  // merge right
      len += next->second;
      next = free_.erase(next);
    }
    if (next != free_.begin()) {  // merge left
      auto prev = std::prev(next);
      if (prev->first + prev->second == off) {
        prev->second += len;
        return;
      }
    }
    free_[off] = len;
  }

 private:
  static uint64_t round(uint64_t b) { return (b + kAlign - 1) / kAlign * kAlign; }
  unsigned char *base_ = nullptr;
  std::map<uint64_t, uint64_t> free_;  // offset -> length of free blocks
};

struct Runner {
  BatchRunner batch;
  std::vector<Request *> jobs;
  cudaEvent_t start = nullptr, end = nullptr;  // timing events of a batch
};

}  // namespace
}  // namespace fi

using namespace fi;

struct fi_join_server {
  fi_join_server_config cfg{};
  int device = 0;
  // relations of small joins load on a high-priority stream, so that they
  // do not queue behind the generation or copy of a large one
  cudaStream_t load_small = nullptr;
  std::vector<Worker> workers;
  std::vector<Runner> runners;  // [0,1]: int32 keys, [2,3]: int64 keys
  uint64_t fixed = 0, reserved = 0, peak = 0;
  void *slab = nullptr;         // relation arena (budget - fixed, or less)
  uint64_t slab_bytes = 0;
  Arena arena;

  std::mutex mu;
  std::condition_variable cv_work, cv_done;
  bool stop = false;
  std::thread sched;
  uint64_t next_ticket = 1;
  std::deque<Request *> pending;               // not yet admitted (large)
  std::deque<Request *> pending_small;         // not yet admitted (small)
  std::deque<Request *> small_q[2];            // admitted small, per key type
  std::deque<Request *> large_q;               // admitted large
  std::unordered_map<uint64_t, Request *> all; // every uncollected request
  fi_join_server_stats stats{};
  int fatal = 0;                               // sticky CUDA error

  void loop();
  bool admit(Request *r);
  void load(Request *r, cudaStream_t stream);
  void release(Request *r);
  bool dispatch_batches(Clock::time_point now);
  bool dispatch_large();
  std::deque<Request *>::iterator next_large(Clock::time_point now);
  Request *prefetched = nullptr;  // last large join loaded ahead of its run
  cudaStream_t load_large = nullptr;
  bool complete();
  void finish(Request *r, int status);
  void teardown();
};

namespace {

uint64_t key_bytes_of(const fi_join_request &q) { return q.tuple_bytes / 2; }

int type_index(const fi_join_request &q) { return q.tuple_bytes == 16 ? 1 : 0; }

// Device bytes of a request's relations when the server holds them.
uint64_t relation_bytes(const fi_join_request &q) {
  const uint64_t kb = key_bytes_of(q);
  switch (q.source) {
    case FI_SOURCE_HOST:
      return 2 * kb * (q.build_len + q.probe_len);
    case FI_SOURCE_SYNTHETIC:  // payload = key: one column per relation
      return kb * (q.build_len + q.probe_len);
    default:
      return 0;
  }
}

template <typename K>
void generate(Request *r, cudaStream_t st) {
  const fi_join_request &q = r->req;
  launch_gen_primary_keys<K>((K *)r->owned[0], q.build_len, q.seed, (K)1, st);
  if (q.zipf_s > 0)
    launch_gen_zipf_fk<K>((K *)r->owned[1], q.probe_len, q.build_len, q.zipf_s,
                          q.seed + 1, q.seed, (K)1, st);
  else
    launch_gen_uniform_fk<K>((K *)r->owned[1], q.probe_len, q.build_len,
                             q.seed + 1, (K)1, st);
}

}  // namespace

void fi_join_server::release(Request *r) {
  if (r->block) arena.release(r->block, r->reserve);
  r->block = nullptr;
  for (void *&p : r->owned) p = nullptr;
  if (r->ready) {
    cudaEventDestroy(r->ready);
    r->ready = nullptr;
  }
  reserved -= r->reserve;
  r->reserve = 0;
}

void fi_join_server::finish(Request *r, int status) {
  if (prefetched == r) prefetched = nullptr;
  release(r);
  r->resp.status = status;
  r->resp.latency_us = us_between(r->t_submit, Clock::now());
  r->done = true;
  ++stats.completed;
  cv_done.notify_all();
}

void fi_join_server::load(Request *r, cudaStream_t stream) {
  const fi_join_request &q = r->req;
  const uint64_t kb = key_bytes_of(q);
  if (q.source == FI_SOURCE_DEVICE) {
    r->cols[0] = q.build_key; r->cols[1] = q.build_pay;
    r->cols[2] = q.probe_key; r->cols[3] = q.probe_pay;
    return;
  }
  const uint64_t lens[4] = {q.build_len, q.build_len, q.probe_len, q.probe_len};
  const bool host = q.source == FI_SOURCE_HOST;
  cudaStream_t load_stream = stream;
  r->loaded = true;
  r->load = load_stream;
  const int ncols = host ? 4 : 2;
  unsigned char *at = (unsigned char *)r->block;
  for (int i = 0; i < ncols; ++i) {
    const uint64_t n = host ? lens[i] : lens[2 * i];
    r->owned[i] = at;
    at += (n * kb + Arena::kAlign - 1) / Arena::kAlign * Arena::kAlign;
  }
  if (host) {
    const void *src[4] = {q.build_key, q.build_pay, q.probe_key, q.probe_pay};
    for (int i = 0; i < 4; ++i) {
      if (lens[i])
        cudaMemcpyAsync(r->owned[i], src[i], lens[i] * kb, cudaMemcpyHostToDevice,
                        load_stream);
      r->cols[i] = r->owned[i];
    }
  } else {
    if (kb == 8)
      generate<int64_t>(r, load_stream);
    else
      generate<int32_t>(r, load_stream);
    r->cols[0] = r->cols[1] = r->owned[0];
    r->cols[2] = r->cols[3] = r->owned[1];
  }
  cudaEventCreateWithFlags(&r->ready, cudaEventDisableTiming);
  cudaEventRecord(r->ready, load_stream);
}

bool fi_join_server::admit(Request *r) {
  const fi_join_request &q = r->req;
  // columns rounded to the arena's alignment, at most four of them
  const uint64_t need = relation_bytes(q) ? relation_bytes(q) + 4 * Arena::kAlign : 0;
  if (need > slab_bytes) {
    finish(r, set_error(FI_ERR_CAPACITY,
                        "request needs %llu bytes, more than the free budget",
                        (unsigned long long)need));
    return true;
  }
  if (need) {
    r->block = arena.alloc(need);
    if (!r->block) return false;  // wait for memory to be released
  }
  reserved += need;
  peak = std::max(peak, reserved);
  r->reserve = need;
  r->t_admit = Clock::now();
  r->resp.queue_us = us_between(r->t_submit, r->t_admit);
  fi_autotune_plan(q.tuple_bytes, q.build_len, q.probe_len, q.zipf_s > 0 ? 1 : 0,
                   cfg.small_tuples, &r->plan);
  r->small = r->plan.batched != 0 && q.build_len + q.probe_len <= cfg.batch_tuples;
  if (!r->small) {
    fi_tuned_plan &p = r->plan;
    // within the workers' engines (12 + 10 bits); perfect hashing needs
    // dense unique build keys, which only the synthetic source guarantees
    if (p.batched || p.radix_bits.pass_bits[0] > 12 || p.radix_bits.pass_bits[1] > 10)
      autotune_model(q.build_len, &p);
    if (p.hashing_scheme == FI_HASHING_PERFECT && q.source != FI_SOURCE_SYNTHETIC)
      p.hashing_scheme = FI_HASHING_BUCKET_CHAINING;
  }
  // small joins load now, on the high-priority stream, to be ready for the
  // next batch; large ones load on their worker's stream when they run
  if (r->small) {
    load(r, load_small);
    small_q[type_index(q)].push_back(r);
  } else {
    large_q.push_back(r);
  }
  return true;
}

bool fi_join_server::dispatch_batches(Clock::time_point now) {
  bool progress = false;
  for (int t = 0; t < 2; ++t) {
    std::deque<Request *> &q = small_q[t];
    for (int i = 0; i < 2 && !q.empty(); ++i) {
      Runner &run = runners[2 * t + i];
      if (run.batch.busy()) continue;
      const bool other_busy = runners[2 * t + (1 - i)].batch.busy();
      const bool full = q.size() >= std::max<uint32_t>(1, run.batch.max_jobs() / 4);
      const bool old = us_between(q.front()->t_admit, now) >= cfg.batch_wait_us;
      if (other_busy && !full && !old) continue;
      std::vector<BatchJob> jobs;
      run.jobs.clear();
      uint64_t tuples = 0;
      while (!q.empty() && jobs.size() < run.batch.max_jobs()) {
        Request *r = q.front();
        const uint64_t n = r->req.build_len + r->req.probe_len;
        if (tuples + n > run.batch.max_tuples()) break;
        tuples += n;
        jobs.push_back(BatchJob{r->cols[0], r->cols[1], r->cols[2], r->cols[3],
                                r->req.build_len, r->req.probe_len,
                                (uint32_t)r->plan.radix_bits.pass_bits[0]});
        run.jobs.push_back(r);
        q.pop_front();
        if (r->ready) cudaStreamWaitEvent(run.batch.stream(), r->ready, 0);
      }
      cudaEventRecord(run.start, run.batch.stream());
      const int rc = run.batch.launch(jobs.data(), (uint32_t)jobs.size());
      cudaEventRecord(run.end, run.batch.stream());
      if (rc) {
        for (Request *r : run.jobs) finish(r, rc);
        run.jobs.clear();
        continue;
      }
      run.batch.set_busy(true);
      ++stats.batches;
      stats.batched_jobs += jobs.size();
      progress = true;
    }
  }
  return progress;
}

static int run_large(Worker &w, Slot &sl, Request *r, uint64_t slice) {
  const fi_join_request &q = r->req;
  const fi_tuned_plan &p = r->plan;
  if (r->ready) {
    cudaError_t ce = cudaStreamWaitEvent(w.stream, r->ready, 0);
    if (ce != cudaSuccess) return cuda_error(ce, "stream wait");
  }
  cudaEventRecord(sl.start, w.stream);
  fi_join_plan jp{p.radix_bits, p.hashing_scheme, p.join_block, p.scatter};
  int rc = fi_radix_join_engine_set_plan(w.engine, &jp);
  if (rc) return rc;
  const uint64_t sn = q.probe_len;
  if (sn > slice * kMaxSlices)
    return set_error(FI_ERR_CAPACITY, "probe relation needs more than %u slices",
                     kMaxSlices);
  sl.slices = sn ? (uint32_t)((sn + slice - 1) / slice) : 0;
  fi_stream_t st = (fi_stream_t)w.stream;
  if (q.tuple_bytes == 16) {
    rc = fi_radix_join_engine_build_int64(w.engine, (const int64_t *)r->cols[0],
                                          (const int64_t *)r->cols[1], q.build_len, st);
    for (uint32_t s = 0; !rc && s < sl.slices; ++s) {
      const uint64_t o = (uint64_t)s * slice, n = std::min(slice, sn - o);
      rc = fi_radix_join_engine_probe_int64(
          w.engine, (const int64_t *)r->cols[2] + o, (const int64_t *)r->cols[3] + o,
          n, sl.d_res + s, st);
    }
  } else {
    rc = fi_radix_join_engine_build_int32(w.engine, (const int32_t *)r->cols[0],
                                          (const int32_t *)r->cols[1], q.build_len, st);
    for (uint32_t s = 0; !rc && s < sl.slices; ++s) {
      const uint64_t o = (uint64_t)s * slice, n = std::min(slice, sn - o);
      rc = fi_radix_join_engine_probe_int32(
          w.engine, (const int32_t *)r->cols[2] + o, (const int32_t *)r->cols[3] + o,
          n, sl.d_res + s, st);
    }
  }
  if (rc) return rc;
  if (sl.slices) {
    cudaError_t ce = cudaMemcpyAsync(sl.h_res, sl.d_res, sl.slices * sizeof(fi_join_result),
                                     cudaMemcpyDeviceToHost, w.stream);
    if (ce != cudaSuccess) return cuda_error(ce, "result copy");
  }
  // the engine's error word, without a device-wide synchronisation
  rc = fi_radix_join_engine_status_async(w.engine, (int *)(sl.h_res + kMaxSlices), st);
  if (rc) return rc;
  cudaError_t ce = cudaEventRecord(sl.done, w.stream);
  if (ce != cudaSuccess) return cuda_error(ce, "event record");
  return FI_OK;
}

bool fi_join_server::dispatch_large() {
  bool progress = false;
  for (Worker &w : workers) {
    while (w.count < kWorkerSlots && !large_q.empty() && !fatal) {
      auto pick = next_large(Clock::now());
      Request *r = *pick;
      large_q.erase(pick);
      progress = true;
      if (r->req.build_len > cfg.max_build) {
        finish(r, set_error(FI_ERR_CAPACITY,
                            "build relation above the server's max_build"));
        continue;
      }
      Slot &sl = w.slot[(w.head + w.count) % kWorkerSlots];
      if (!r->loaded) load(r, w.stream);
      const int rc = run_large(w, sl, r, cfg.probe_slice);
      if (rc) {
        // the engine may hold work of this request: wait for it before the
        // relations are released
        cudaStreamSynchronize(w.stream);
        finish(r, rc);
      } else {
        sl.req = r;
        ++w.count;
        ++stats.engine_runs;
      }
    }
  }
  // prefetch: load the next large join while the workers run, so that its
  // generation or copy overlaps the current join
  if (!large_q.empty() && !fatal &&
      (!prefetched || cudaEventQuery(prefetched->ready) != cudaErrorNotReady)) {
    auto nx = next_large(Clock::now());
    if (!(*nx)->loaded && (*nx)->req.build_len <= cfg.max_build) {
      load(*nx, load_large);
      prefetched = *nx;
      progress = true;
    }
  }
  return progress;
}

std::deque<Request *>::iterator fi_join_server::next_large(Clock::time_point now) {
  // shortest job first, so that a long join does not hold up the many
  // shorter ones behind it; a join that has waited longer than
  // kMaxLargeWaitUs goes first, which bounds how long the longest wait
  constexpr double kMaxLargeWaitUs = 500e3;
  auto pick = large_q.begin();
  for (auto it = large_q.begin(); it != large_q.end(); ++it) {
    if (us_between((*it)->t_admit, now) > kMaxLargeWaitUs) return it;
    if ((*it)->req.build_len + (*it)->req.probe_len <
        (*pick)->req.build_len + (*pick)->req.probe_len)
      pick = it;
  }
  return pick;
}

bool fi_join_server::complete() {
  bool progress = false;
  for (Worker &w : workers) {
    // a worker's joins finish in the order they were enqueued
    while (w.count > 0) {
      Slot &sl = w.slot[w.head];
      const cudaError_t ce = cudaEventQuery(sl.done);
      if (ce == cudaErrorNotReady) break;
      Request *r = sl.req;
      sl.req = nullptr;
      w.head = (w.head + 1) % kWorkerSlots;
      --w.count;
      progress = true;
      if (ce != cudaSuccess) {
        fatal = cuda_error(ce, "large join");
        finish(r, fatal);
        continue;
      }
      uint64_t sum = 0, count = 0;
      for (uint32_t s = 0; s < sl.slices; ++s) {
        sum += (uint64_t)sl.h_res[s].sum;
        count += sl.h_res[s].count;
      }
      r->resp.result.sum = (int64_t)sum;
      r->resp.result.count = count;
      const int dev = *(const int *)(sl.h_res + kMaxSlices);
      float ms = 0.f;
      if (cudaEventElapsedTime(&ms, sl.start, sl.done) == cudaSuccess)
        stats.engine_busy_us += 1e3 * ms;
      finish(r, dev == 0 ? FI_OK
                         : set_error(dev == FI_ERR_TIMEOUT ? FI_ERR_TIMEOUT
                                                           : FI_ERR_RUNTIME,
                                     "device-side error %d in a large join", dev));
    }
  }
  for (Runner &run : runners) {
    if (!run.batch.busy()) continue;
    const cudaError_t ce = cudaEventQuery(run.batch.done());
    if (ce == cudaErrorNotReady) continue;
    run.batch.set_busy(false);
    progress = true;
    float ms = 0.f;
    if (ce == cudaSuccess && cudaEventElapsedTime(&ms, run.start, run.end) == cudaSuccess)
      stats.batch_busy_us += 1e3 * ms;
    const uint32_t n = (uint32_t)run.jobs.size();
    const int st = ce == cudaSuccess ? FI_OK : (fatal = cuda_error(ce, "batch"));
    for (uint32_t i = 0; i < n; ++i) {
      Request *r = run.jobs[i];
      r->resp.batched = 1;
      r->resp.batch_jobs = n;
      if (st == FI_OK) {
        r->resp.result.sum = (int64_t)run.batch.results()[i].sum;
        r->resp.result.count = run.batch.results()[i].count;
      }
      finish(r, st);
    }
    run.jobs.clear();
  }
  return progress;
}

void fi_join_server::loop() {
  cudaSetDevice(device);
  std::unique_lock<std::mutex> lk(mu);
  for (;;) {
    bool progress = false;
    const Clock::time_point t0 = Clock::now();
    // Admission in arrival order within two queues: small joins (a few MB
    // each, below small_tuples) and the rest.  Small joins are admitted
    // first, each as soon as its block fits, so that they do not wait
    // behind a large request that waits for arena memory; large requests
    // keep their arrival order.
    for (std::deque<Request *> *q : {&pending_small, &pending}) {
      while (!q->empty() && !fatal) {
        if (!admit(q->front())) break;
        q->pop_front();
        progress = true;
      }
    }
    progress |= complete();
    if (!fatal) {
      progress |= dispatch_batches(Clock::now());
      progress |= dispatch_large();
    }
    if (progress) stats.enqueue_us += us_between(t0, Clock::now());
    if (fatal) {
      // a CUDA error is sticky: fail everything that has not started
      for (std::deque<Request *> *q :
           {&pending_small, &pending, &small_q[0], &small_q[1], &large_q})
        while (!q->empty()) {
          finish(q->front(), fatal);
          q->pop_front();
        }
    }
    bool busy = false;
    for (Worker &w : workers) busy |= w.count > 0;
    for (Runner &r : runners) busy |= r.batch.busy();
    const bool queued = !pending.empty() || !pending_small.empty() || !small_q[0].empty() ||
                        !small_q[1].empty() || !large_q.empty();
    if (stop && !busy && !queued) break;
    if (!progress) {
      // in-flight work is polled every 20 us; an idle server sleeps until a
      // submit wakes it
      if (busy || queued)
        cv_work.wait_for(lk, std::chrono::microseconds(20));
      else
        cv_work.wait(lk);
    }
  }
}

void fi_join_server::teardown() {
  for (Worker &w : workers) {
    if (w.stream) cudaStreamSynchronize(w.stream);
    if (w.engine) fi_radix_join_engine_free(w.engine);
    for (Slot &sl : w.slot) {
      if (sl.d_res) cudaFree(sl.d_res);
      if (sl.h_res) cudaFreeHost(sl.h_res);
      if (sl.done) cudaEventDestroy(sl.done);
      if (sl.start) cudaEventDestroy(sl.start);
    }
    if (w.stream) cudaStreamDestroy(w.stream);
  }
  workers.clear();
  for (Runner &r : runners) {
    r.batch.release();
    if (r.start) cudaEventDestroy(r.start);
    if (r.end) cudaEventDestroy(r.end);
  }
  runners.clear();
  for (cudaStream_t *ls : {&load_small, &load_large})
    if (*ls) {
      cudaStreamSynchronize(*ls);
      cudaStreamDestroy(*ls);
      *ls = nullptr;
    }
  for (auto &kv : all) delete kv.second;
  all.clear();
  if (slab) cudaFree(slab);
  slab = nullptr;
  slab_bytes = 0;
}

// ---- C ABI ----------------------------------------------------------------------
extern "C" int fi_join_server_new(const fi_join_server_config *cfg,
                                  fi_join_server **out) {
  if (!out) return set_error(FI_ERR_INVALID_ARGUMENT, "null output handle");
  *out = nullptr;
  auto *s = new fi_join_server();
  if (cfg) s->cfg = *cfg;
  fi_join_server_config &c = s->cfg;
  if (!c.hbm_budget_bytes) c.hbm_budget_bytes = 150000000000ull;
  // 0: two workers when their engines take at most half the budget, else
  // one (measured on the 10,000-request stream: two workers serve 7% more at
  // 1.2x the plain path's capacity and cut p99 at 0.8x, 727 -> 500 ms)
  const bool auto_workers = c.workers == 0;
  if (auto_workers) c.workers = 2;
  if (!c.small_tuples) c.small_tuples = 4ull << 20;
  if (!c.max_batch_jobs) c.max_batch_jobs = 256;
  if (!c.batch_tuples) c.batch_tuples = 1ull << 25;
  if (!c.batch_wait_us) c.batch_wait_us = 200;
  if (!c.max_build) c.max_build = 1ull << 28;
  if (!c.probe_slice) c.probe_slice = 1ull << 28;
  if (c.max_batch_jobs > kBatchMaxJobs || c.workers > 16) {
    delete s;
    return set_error(FI_ERR_INVALID_ARGUMENT,
                     "at most %u jobs per batch and 16 workers", kBatchMaxJobs);
  }
  cudaGetDevice(&s->device);
  int rc = FI_OK;
  int prio_low = 0, prio_high = 0;  // numerically: least, greatest priority
  cudaDeviceGetStreamPriorityRange(&prio_low, &prio_high);
  cudaError_t ce = cudaStreamCreateWithPriority(&s->load_small,
                                                cudaStreamNonBlocking, prio_high);
  if (ce == cudaSuccess)
    ce = cudaStreamCreateWithFlags(&s->load_large, cudaStreamNonBlocking);
  if (ce != cudaSuccess) rc = cuda_error(ce, "stream create");
  s->workers.resize(rc ? 0 : c.workers);
  uint64_t first_engine_bytes = 0;
  for (size_t wi = 0; wi < s->workers.size(); ++wi) {
    if (rc) break;
    if (auto_workers && wi == 1 && 2 * first_engine_bytes > c.hbm_budget_bytes / 2) {
      c.workers = 1;  // worker 1 was never set up
      s->workers.resize(1);
      break;
    }
    Worker &w = s->workers[wi];
    fi_radix_bits caps{{12, 10, -1}};
    rc = fi_radix_join_engine_new(c.max_build, c.probe_slice, 16, caps,
                                  FI_HASHING_BUCKET_CHAINING, &w.engine);
    if (rc) break;
    const uint64_t engine_bytes = fi_radix_join_engine_workspace_bytes(w.engine);
    if (wi == 0) first_engine_bytes = engine_bytes;
    s->fixed += engine_bytes;
    if ((ce = cudaStreamCreateWithFlags(&w.stream, cudaStreamNonBlocking)) != cudaSuccess)
      rc = cuda_error(ce, "worker set-up");
    for (Slot &sl : w.slot) {
      if (rc) break;
      if ((ce = cudaEventCreate(&sl.done)) || (ce = cudaEventCreate(&sl.start)) ||
          (ce = cudaMalloc((void **)&sl.d_res, kMaxSlices * sizeof(fi_join_result))) ||
          (ce = cudaHostAlloc((void **)&sl.h_res,
                              (kMaxSlices + 1) * sizeof(fi_join_result),
                              cudaHostAllocDefault)))
        rc = cuda_error(ce, "worker set-up");
    }
  }
  if (!rc) {
    s->runners = std::vector<Runner>(4);
    const uint32_t sm = (uint32_t)device_sm_count();
    for (int i = 0; i < 4 && !rc; ++i) {
      rc = s->runners[i].batch.init(i < 2 ? 4 : 8, c.max_batch_jobs, c.batch_tuples, sm,
                                    prio_high);
      if (!rc && ((ce = cudaEventCreate(&s->runners[i].start)) ||
                  (ce = cudaEventCreate(&s->runners[i].end))))
        rc = cuda_error(ce, "event create");
      s->fixed += s->runners[i].batch.device_bytes();
    }
  }
  if (!rc && s->fixed > c.hbm_budget_bytes)
    rc = set_error(FI_ERR_CAPACITY, "the engines and batch arenas (%llu bytes) "
                   "exceed the budget", (unsigned long long)s->fixed);
  if (!rc) {
    // the relation arena: the rest of the budget, or what the device has
    // free (less 1 GiB of headroom), whichever is smaller
    size_t dev_free = 0, dev_total = 0;
    cudaMemGetInfo(&dev_free, &dev_total);
    uint64_t want = c.hbm_budget_bytes - s->fixed;
    const uint64_t headroom = 1ull << 30;
    if (dev_free > headroom && want > dev_free - headroom) want = dev_free - headroom;
    want &= ~(Arena::kAlign - 1);
    if (want && (ce = cudaMalloc(&s->slab, want)) != cudaSuccess)
      rc = cuda_error(ce, "relation arena");
    else {
      s->slab_bytes = want;
      s->arena.init(s->slab, want);
    }
  }
  if (rc) {
    s->teardown();
    delete s;
    return rc;
  }
  s->stats.fixed_bytes = s->fixed;
  s->stats.arena_bytes = s->slab_bytes;
  s->sched = std::thread([s] { s->loop(); });
  *out = s;
  return FI_OK;
}

extern "C" void fi_join_server_free(fi_join_server *s) {
  if (!s) return;
  {
    std::lock_guard<std::mutex> lk(s->mu);
    s->stop = true;
  }
  s->cv_work.notify_all();
  if (s->sched.joinable()) s->sched.join();
  s->teardown();
  delete s;
}

extern "C" int fi_join_server_submit(fi_join_server *s, const fi_join_request *req,
                                     uint64_t *ticket) {
  if (!s || !req || !ticket) return set_error(FI_ERR_INVALID_ARGUMENT, "null argument");
  if (req->tuple_bytes != 8 && req->tuple_bytes != 16)
    return set_error(FI_ERR_INVALID_ARGUMENT, "tuple_bytes must be 8 or 16");
  if (req->source > FI_SOURCE_SYNTHETIC)
    return set_error(FI_ERR_INVALID_ARGUMENT, "unknown source");
  if (req->source != FI_SOURCE_SYNTHETIC &&
      ((req->build_len && (!req->build_key || !req->build_pay)) ||
       (req->probe_len && (!req->probe_key || !req->probe_pay))))
    return set_error(FI_ERR_INVALID_ARGUMENT, "null column");
  auto *r = new Request();
  r->req = *req;
  r->t_submit = Clock::now();
  {
    std::lock_guard<std::mutex> lk(s->mu);
    if (s->fatal) {
      delete r;
      return s->fatal;
    }
    *ticket = s->next_ticket++;
    s->all[*ticket] = r;
    (r->req.build_len + r->req.probe_len <= s->cfg.small_tuples ? s->pending_small
                                                                 : s->pending)
        .push_back(r);
    ++s->stats.submitted;
  }
  s->cv_work.notify_one();
  return FI_OK;
}

static int collect(fi_join_server *s, uint64_t ticket, fi_join_response *resp,
                   bool block, int *done) {
  std::unique_lock<std::mutex> lk(s->mu);
  auto it = s->all.find(ticket);
  if (it == s->all.end()) return set_error(FI_ERR_INVALID_ARGUMENT, "unknown ticket");
  Request *r = it->second;
  if (block) s->cv_done.wait(lk, [r] { return r->done; });
  if (done) *done = r->done ? 1 : 0;
  if (!r->done) return FI_OK;
  *resp = r->resp;
  s->all.erase(it);
  delete r;
  return FI_OK;
}

extern "C" int fi_join_server_wait(fi_join_server *s, uint64_t ticket,
                                   fi_join_response *resp) {
  if (!s || !resp) return set_error(FI_ERR_INVALID_ARGUMENT, "null argument");
  return collect(s, ticket, resp, true, nullptr);
}

extern "C" int fi_join_server_poll(fi_join_server *s, uint64_t ticket, int *done,
                                   fi_join_response *resp) {
  if (!s || !resp || !done) return set_error(FI_ERR_INVALID_ARGUMENT, "null argument");
  return collect(s, ticket, resp, false, done);
}

extern "C" int fi_join_server_stats_get(fi_join_server *s, fi_join_server_stats *out) {
  if (!s || !out) return set_error(FI_ERR_INVALID_ARGUMENT, "null argument");
  std::lock_guard<std::mutex> lk(s->mu);
  *out = s->stats;
  out->reserved_bytes = s->reserved;
  out->peak_reserved_bytes = s->peak;
  out->workers = s->workers.size();
  return FI_OK;
}
