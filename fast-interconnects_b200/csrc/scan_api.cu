// Exclusive prefix sums of u64 arrays: the counterparts of the reference's
// scan test exports host_block_exclusive_prefix_sum_uint64 and
// host_device_exclusive_prefix_sum[_initialize]_uint64
// (sql-ops/include/prefix_scan.h:55-122,213-384) and of
// GpuPrefixSum::state_len (sql-ops/src/prefix_scan/gpu_prefix_scan.rs:40-51).
//
// Same results: with T threads, thread t owns the contiguous items
// [t*ti, (t+1)*ti) (ti = ceil(n / T)) and every item becomes the exclusive
// sum of the items before it plus (t+1) * padding.  The block version scans
// `size / grid` items per block independently; the device version scans
// the whole array across the grid.
//
// B200 design of the device-wide scan: tiles are claimed in order through
// a counter (dynamic tile ids), so a tile only ever waits for tiles whose
// blocks are already running; each tile publishes its aggregate, then its
// inclusive prefix, in the caller's state array and looks back over its
// predecessors (decoupled look-back, Merrill & Garland 2016) with a bounded
// spin.  The state holds the tile counter in its first entry and the tile
// slots from entry 32 on; state_len entries of 32 bytes are always enough.
#include "../../include/fi_sqlops.h"
#include "api_internal.h"
#include "common.cuh"

namespace fi {
namespace {

constexpr uint64_t kFlagAgg = 1, kFlagPre = 2;

struct ScanSlot {  // 32 bytes, the size of the reference's ScanState<u64>
  uint64_t status, aggregate, prefix, pad;
};

__device__ __forceinline__ uint64_t ld_acquire(const uint64_t *p) {
  uint64_t v;
  asm volatile("ld.acquire.gpu.global.u64 %0, [%1];" : "=l"(v) : "l"(p) : "memory");
  return v;
}
__device__ __forceinline__ void st_release(uint64_t *p, uint64_t v) {
  asm volatile("st.release.gpu.global.u64 [%0], %1;" ::"l"(p), "l"(v) : "memory");
}

// Block b scans its own size/grid items: thread t owns [t*ti, (t+1)*ti)
// of them (clamped to the slice) and adds (t+1) * padding.
__global__ void block_scan_kernel(uint64_t *data, uint64_t size, uint64_t padding) {
  __shared__ uint64_t tmp[33];
  const uint64_t bsize = size / gridDim.x;
  uint64_t *d = data + bsize * blockIdx.x;
  const uint64_t ti = (bsize + blockDim.x - 1) / blockDim.x;
  const uint64_t t = threadIdx.x;
  const uint64_t b = min(bsize, t * ti), e = min(bsize, b + ti);
  uint64_t local = 0;
  for (uint64_t i = b; i < e; ++i) local += d[i];
  uint64_t total;
  uint64_t run = block_exclusive_scan_u64(local, tmp, &total);
  for (uint64_t i = b; i < e; ++i) {
    const uint64_t v = d[i];
    d[i] = run + (t + 1) * padding;
    run += v;
  }
}

__global__ void device_scan_init_kernel(ScanSlot *state, uint64_t len) {
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < len;
       i += (uint64_t)gridDim.x * blockDim.x)
    state[i] = ScanSlot{0, 0, 0, 0};
}

__global__ void device_scan_kernel(uint64_t *data, uint64_t size, uint64_t padding,
                                   ScanSlot *state, int *status) {
  __shared__ uint64_t tmp[33];
  __shared__ uint64_t tile_s, carry_s;
  if (threadIdx.x == 0) tile_s = atomicAdd((unsigned long long *)&state[0].status, 1ull);
  __syncthreads();
  const uint64_t tile = tile_s;
  const uint64_t T = (uint64_t)gridDim.x * blockDim.x;
  const uint64_t ti = (size + T - 1) / T;
  const uint64_t first = tile * blockDim.x * ti;  // tile's first item
  const uint64_t n = first < size ? min(size - first, (uint64_t)blockDim.x * ti) : 0;
  uint64_t *d = data + (first < size ? first : size);
  // 1. tile total
  const uint64_t t = threadIdx.x;
  const uint64_t b = min(n, t * ti), e = min(n, b + ti);
  uint64_t local = 0;
  for (uint64_t i = b; i < e; ++i) local += d[i];
  uint64_t total;
  const uint64_t ex = block_exclusive_scan_u64(local, tmp, &total);
  // 2. publish the aggregate, look back for the exclusive prefix
  if (threadIdx.x == 0) {
    ScanSlot *me = &state[32 + tile];
    uint64_t prefix = 0;
    if (tile == 0) {
      me->prefix = total;
      st_release(&me->status, kFlagPre);
    } else {
      me->aggregate = total;
      st_release(&me->status, kFlagAgg);
      int64_t j = (int64_t)tile - 1;
      uint32_t polls = 0;
      while (j >= 0) {
        ScanSlot *s = &state[32 + j];
        const uint64_t f = ld_acquire(&s->status);
        if (f == 0) {
          if (++polls > kSpinLimit) {
            record_error(status, kDevErrTimeout);
            break;
          }
          spin_pause(polls);
          continue;
        }
        if (f == kFlagPre) {
          prefix += s->prefix;
          break;
        }
        prefix += s->aggregate;
        --j;
      }
      me->prefix = prefix + total;
      st_release(&me->status, kFlagPre);
    }
    carry_s = prefix;
  }
  __syncthreads();
  // 3. write the exclusive sums
  uint64_t run = carry_s + ex;
  const uint64_t gthread = tile * blockDim.x + t;
  for (uint64_t i = b; i < e; ++i) {
    const uint64_t v = d[i];
    d[i] = run + (gthread + 1) * padding;
    run += v;
  }
}

}  // namespace
}  // namespace fi

using namespace fi;

extern "C" uint64_t fi_gpu_prefix_sum_state_len(uint32_t grid_size, uint32_t block_size) {
  return (uint64_t)grid_size * block_size / 32 + 32;
}

extern "C" int fi_block_exclusive_prefix_sum_uint64(uint64_t *data, uint64_t size,
                                                    uint64_t padding, uint32_t grid_size,
                                                    uint32_t block_size,
                                                    fi_stream_t stream) {
  if (!data && size) return set_error(FI_ERR_INVALID_ARGUMENT, "null data");
  if (grid_size == 0 || block_size == 0 || block_size > 1024 || block_size % 32)
    return set_error(FI_ERR_INVALID_ARGUMENT,
                     "grid must be positive, block a multiple of 32 up to 1024");
  block_scan_kernel<<<grid_size, block_size, 0, (cudaStream_t)stream>>>(data, size,
                                                                         padding);
  const cudaError_t e = cudaGetLastError();
  return e == cudaSuccess ? FI_OK : cuda_error(e, "block prefix sum launch");
}

extern "C" int fi_device_exclusive_prefix_sum_initialize_uint64(
    void *state, uint32_t grid_size, uint32_t block_size, fi_stream_t stream) {
  if (!state) return set_error(FI_ERR_INVALID_ARGUMENT, "null state");
  const uint64_t len = fi_gpu_prefix_sum_state_len(grid_size, block_size);
  device_scan_init_kernel<<<(uint32_t)((len + 255) / 256), 256, 0,
                            (cudaStream_t)stream>>>(static_cast<ScanSlot *>(state), len);
  const cudaError_t e = cudaGetLastError();
  return e == cudaSuccess ? FI_OK : cuda_error(e, "prefix sum state launch");
}

extern "C" int fi_device_exclusive_prefix_sum_uint64(uint64_t *data, uint64_t size,
                                                     uint64_t padding, void *state,
                                                     uint32_t grid_size,
                                                     uint32_t block_size,
                                                     int *status, fi_stream_t stream) {
  if ((!data && size) || !state)
    return set_error(FI_ERR_INVALID_ARGUMENT, "null argument");
  if (grid_size == 0 || block_size == 0 || block_size > 1024 || block_size % 32)
    return set_error(FI_ERR_INVALID_ARGUMENT,
                     "grid must be positive, block a multiple of 32 up to 1024");
  // the tile slots must fit the state the caller sized with state_len
  if ((uint64_t)grid_size + 32 > fi_gpu_prefix_sum_state_len(grid_size, block_size))
    return set_error(FI_ERR_INVALID_ARGUMENT, "block too small for the state layout");
  device_scan_kernel<<<grid_size, block_size, 0, (cudaStream_t)stream>>>(
      data, size, padding, static_cast<ScanSlot *>(state), status);
  const cudaError_t e = cudaGetLastError();
  return e == cudaSuccess ? FI_OK : cuda_error(e, "device prefix sum launch");
}
