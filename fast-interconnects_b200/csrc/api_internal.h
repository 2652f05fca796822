// Internal helpers shared by the C-ABI translation units.
#pragma once

#include <cuda_runtime.h>
#include <stddef.h>
#include <stdint.h>

namespace fi {

// Largest fanout of one pass with a shared-memory histogram (u32 counters).
constexpr uint32_t kMaxHistBits = 15;
// Largest fanout of the single-level tile scatter; larger fanouts use the
// hierarchical two-level scatter.
constexpr uint32_t kMaxTileBits = 14;
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
