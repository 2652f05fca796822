// Batched execution of many small radix joins (internal C++ interface used by
// the join server and by the fi_join_batch_* entry points).
//
// A batch holds up to max_jobs joins of one key type whose build and probe
// relations together fit the batch's partition arena.  Every job is joined
// with one radix pass of its own bits; the whole batch runs as one CUDA graph
// (descriptor copy, counter reset, histogram, scan, scatter, join, result
// copy), the same graph for every batch of this runner: the kernels read the
// batch's shape from the descriptor table in device memory and walk it with
// grid-stride loops and a device work queue, so the grids are fixed and the
// graph is captured once.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <vector>

namespace fi {

// Descriptor of one job in device memory.
struct BatchJobDesc {
  const void *rk, *rp, *sk, *sp;  // build and probe columns (device)
  uint64_t rn, sn;                // build and probe lengths
  uint64_t out_r, out_s;          // first arena tuple of the job's R and S
  uint32_t bits;                  // radix bits of the job's single pass
  uint32_t cnt_base;              // counters: R at cnt_base, S at cnt_base + F
  uint32_t tile_r, tile_s;        // first global tile of R and of S
  uint32_t item_base;             // first join item (one per partition)
  uint32_t pad_;
};

struct BatchHeader {
  uint32_t jobs, tiles, items, counters;
};

struct BatchJobResult {
  uint64_t sum;    // wrapping sum of the matched probe payloads
  uint64_t count;  // matches
};

// One small join as the host submits it.
struct BatchJob {
  const void *rk, *rp, *sk, *sp;
  uint64_t rn, sn;
  uint32_t bits;  // radix bits; batch_bits() gives the default
};

constexpr uint32_t kBatchTile = 4096;    // tuples per histogram/scatter tile
constexpr uint32_t kBatchMaxBits = 12;   // largest fanout of a batched job
constexpr uint32_t kBatchMaxJobs = 1024; // job tables staged in shared memory

// Radix bits of a batched join: partitions of about 3K build tuples, so
// that most build partitions fit one shared-memory table.
uint32_t batch_bits(uint64_t build_len);

class BatchRunner {
 public:
  // key_bytes 4 or 8; allocates the arena and captures the graph.  The
  // runner's stream gets `priority` (cudaStreamCreateWithPriority; lower is
  // more urgent, 0 the default).
  int init(uint32_t key_bytes, uint32_t max_jobs, uint64_t max_tuples,
           uint32_t sm_count, int priority = 0);
  void release();
  ~BatchRunner() { release(); }

  // Whether `jobs` fit one batch of this runner.
  bool fits(const BatchJob *jobs, uint32_t n) const;
  uint64_t device_bytes() const { return bytes_; }
  uint32_t key_bytes() const { return key_bytes_; }
  uint32_t max_jobs() const { return max_jobs_; }
  uint64_t max_tuples() const { return max_tuples_; }

  // Writes the descriptors and replays the graph on the runner's stream;
  // `done` is recorded after the results are back in host memory.  The
  // runner must not be busy (its pinned descriptor buffer is rewritten).
  int launch(const BatchJob *jobs, uint32_t n);
  cudaEvent_t done() const { return done_; }
  cudaStream_t stream() const { return stream_; }
  bool busy() const { return busy_; }
  void set_busy(bool b) { busy_ = b; }
  // Results of the last launch (valid once `done` has completed).
  const BatchJobResult *results() const { return host_res_; }

 private:
  uint32_t key_bytes_ = 0, max_jobs_ = 0, sm_count_ = 0;
  uint64_t max_tuples_ = 0, max_counters_ = 0, bytes_ = 0;
  bool busy_ = false;
  cudaStream_t stream_ = nullptr;
  cudaEvent_t done_ = nullptr;
  cudaGraphExec_t exec_ = nullptr;
  // device
  BatchHeader *d_head_ = nullptr;
  BatchJobDesc *d_desc_ = nullptr;
  uint32_t *d_counts_ = nullptr, *d_offs_ = nullptr, *d_curs_ = nullptr;
  uint32_t *d_queue_ = nullptr;
  void *d_arena_ = nullptr;
  BatchJobResult *d_res_ = nullptr;
  // pinned host
  unsigned char *host_desc_ = nullptr;  // header (64 bytes) + descriptors
  BatchJobResult *host_res_ = nullptr;
  int capture();
};

}  // namespace fi
