// Chunked prefix sum that allocates no device memory.
//
// Some callers cannot allocate device memory: code running under an
// allocator or a memory budget it does not own (a database engine that hands
// out all device memory from its own pool, a plugin host that forbids
// cudaMalloc on its threads), or code that must not trigger the implicit
// synchronisation a cudaMalloc/cudaFree can cause in the middle of a stream.
// For them this entry point computes the same offsets as
// fi_gpu_prefix_sum_int64 on a Chunked partitioner, but keeps its scratch
// counters in a fixed array compiled into the library instead of in a buffer
// owned by a partitioner handle.
//
// The array (kNoAllocScratchBytes, 2 MiB) lives in device memory of every
// GPU that loads the library, until the process exits.  All calls share it:
// calls whose kernels overlap on the GPU (different streams, or different
// host threads) race on it and produce wrong offsets; serialise them.  The
// counters a call needs are cleared by the call itself (cudaMemsetAsync on
// the stream), so the contents left by a previous call do not matter.
//
// Host code cannot use the array's symbol as a device address: the symbol
// is a host-side stand-in.  The device address is looked up with
// cudaGetSymbolAddress, with that device current, by the first call on that
// device; make that first call before capturing the stream into a CUDA
// graph.  Calls made while the stream is not being captured look the address
// up again, so a cudaDeviceReset (which unloads the module and may place the
// array elsewhere when it is loaded again) between calls is harmless.
#include <cuda_runtime.h>

#include <mutex>

#include "../../include/fi_sqlops.h"
#include "api_internal.h"
#include "common.cuh"
#include "kernels.h"

namespace {

constexpr size_t kNoAllocScratchBytes = 2u << 20;
constexpr uint64_t kNoAllocCounters = kNoAllocScratchBytes / sizeof(uint32_t);
constexpr int kMaxDevices = 64;

static __device__ __align__(256) uint32_t g_noalloc_counters[kNoAllocCounters];

std::mutex g_noalloc_mutex;
uint32_t *g_noalloc_addr[kMaxDevices] = {};

// Device address of g_noalloc_counters on the current device.  Looked up on
// the first call on the device, and again on every call whose stream is not
// being captured (a capture keeps the address recorded before it).
int noalloc_scratch(cudaStream_t stream, uint32_t **out) {
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return fi::cuda_error(e, "cudaGetDevice");
  if (dev < 0 || dev >= kMaxDevices)
    return fi::set_error(FI_ERR_UNSUPPORTED, "device ordinal %d out of range", dev);
  cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
  const bool capturing = cudaStreamIsCapturing(stream, &cap) != cudaSuccess ||
                         cap != cudaStreamCaptureStatusNone;
  cudaGetLastError();  // a failed query leaves no sticky error behind
  std::lock_guard<std::mutex> lock(g_noalloc_mutex);
  if (g_noalloc_addr[dev] == nullptr || !capturing) {
    void *p = nullptr;
    e = cudaGetSymbolAddress(&p, g_noalloc_counters);
    if (e != cudaSuccess || p == nullptr)
      return fi::cuda_error(e == cudaSuccess ? cudaErrorInvalidSymbol : e,
                            "cudaGetSymbolAddress of the fixed scratch array");
    g_noalloc_addr[dev] = static_cast<uint32_t *>(p);
  }
  *out = g_noalloc_addr[dev];
  return FI_OK;
}

}  // namespace

extern "C" int fi_gpu_chunked_prefix_sum_noalloc_int64(
    const int64_t *partition_attr, uint64_t len, uint32_t num_chunks,
    uint32_t radix_bits, uint32_t ignore_bits, uint64_t *offsets,
    fi_stream_t stream) {
  using namespace fi;
  if (num_chunks == 0)
    return set_error(FI_ERR_INVALID_ARGUMENT, "num_chunks must be at least 1");
  if (radix_bits > kMaxHistBits)
    return set_error(FI_ERR_UNSUPPORTED,
                     "prefix sums support at most %u radix bits per pass",
                     kMaxHistBits);
  if (ignore_bits + radix_bits > 64)
    return set_error(FI_ERR_INVALID_ARGUMENT, "ignore_bits + radix_bits > 64");
  if (!offsets || (len > 0 && !partition_attr))
    return set_error(FI_ERR_INVALID_ARGUMENT, "null pointer argument");
  const uint64_t counters = (uint64_t)num_chunks << radix_bits;
  if (counters > kNoAllocCounters)
    return set_error(FI_ERR_INVALID_ARGUMENT,
                     "num_chunks * 2^radix_bits = %llu counters exceeds the "
                     "fixed scratch array of %llu counters (2 MiB); use fewer "
                     "chunks or radix bits, or fi_gpu_prefix_sum_int64",
                     (unsigned long long)counters,
                     (unsigned long long)kNoAllocCounters);
  if ((len + num_chunks - 1) / num_chunks >= 0xffffffffull)
    return set_error(FI_ERR_INTEGER_OVERFLOW,
                     "Relation is too large and causes an integer overflow. Try "
                     "using more chunks by setting a higher CUDA grid size");
  uint32_t *scratch = nullptr;
  int rc = noalloc_scratch((cudaStream_t)stream, &scratch);
  if (rc) return rc;
  HistScratch s{scratch, nullptr, nullptr, nullptr};
  cudaError_t e = launch_chunked_prefix_sum<int64_t>(
      partition_attr, len, num_chunks, radix_bits, ignore_bits,
      padding_len(2 * sizeof(int64_t)), offsets, s,
      (uint32_t)device_sm_count(), (cudaStream_t)stream);
  if (e != cudaSuccess) return cuda_error(e, "prefix sum launch");
  return FI_OK;
}
