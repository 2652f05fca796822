// Internal helpers shared by the C-ABI translation units.
#pragma once

#include <cuda_runtime.h>
#include <stddef.h>
#include <stdint.h>

namespace fi {

// Largest fanout of one prefix sum (u32 counters; above 2^15 bins the
// histogram is split into bin ranges of 2^15 counters each).
constexpr uint32_t kMaxHistBits = 18;
// Largest fanout of the single-level tile scatter.
constexpr uint32_t kMaxTileBits = 14;
// The partitioner switches to the hierarchical two-level scatter above this
// many bits.  Measured on B200 (512M int64 tuples, 148 chunks): one level
// moves 5.2 / 4.9 / 3.6 TB/s at 6 / 8 / 10 bits but 1.5 and 0.7 TB/s at 12
// and 14 bits, where a 4096-8192-tuple tile leaves runs of one or two tuples
// per partition and 148 chunks x 2^bits half-written 128-byte lines overflow
// L2; two levels of 2^(bits/2) partitions each keep their runs long at
// twice the traffic.
constexpr uint32_t kSingleLevelBits = 11;
// Largest fanout of one pass overall.
constexpr uint32_t kMaxRadixBits = 18;
// Largest number of source chunks of prefix_sum_and_transform.
constexpr uint32_t kMaxTransformChunks = 8192;

// An owned, growable device allocation.
struct DevBuf {
  void *ptr = nullptr;
  size_t size = 0;
  int reserve(size_t bytes, bool zero);
  void release();
};

int set_error(int code, const char *fmt, ...);
int cuda_error(cudaError_t e, const char *what);
int read_and_clear_status(DevBuf &status);
uint32_t padding_len(uint32_t tuple_bytes);

}  // namespace fi
