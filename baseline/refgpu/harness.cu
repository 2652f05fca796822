// Launch harness for the reference's own GPU kernels, compiled from the
// reference tree where it lies (baseline/refgpu/Makefile) and linked with this
// file into baseline/refgpu/_build/libref_gpu.so.
//
// Benchmark and test infrastructure only: the library under
// fast-interconnects_b200/ neither links nor calls it.  It lets the same B200
// run the reference kernels beside this repository's on identical inputs, as
// the Rust host code of the reference would launch them
// (sql-ops/src/partition/gpu_radix_partition.rs:561-1239,
// sql-ops/src/join/cuda_radix_join.rs:172-276): same argument structs, grid,
// block and dynamic shared memory.
//
// Kernels covered; none of them waits on another thread, block or grid:
//   gpu_chunked_prefix_sum_int{32,64}              radix_partition.cu:40-96
//   gpu_chunked_radix_partition_*  (NC)            radix_partition.cu:472-525
//   gpu_chunked_laswwc_radix_partition_*           radix_partition.cu:528-683
//   gpu_radix_join_assign_tasks                    radix_join.cu:58-98
//   gpu_join_aggregate_smem_{perfect,chaining}_*   radix_join.cu:103-311
// Left out: the SSWWCv2 / SSWWCv2G / HSSWWCv4 scatters, whose warps spin on
// buffer slots without a bound (radix_partition.cu:837,1058,1318), and the
// cooperative Contiguous prefix sums.
//
// The reference kernels check capacities with device asserts and index shared
// memory without bounds checks.  Every launch here is therefore split in a
// synchronous *_prepare call, which checks on the host that no assert can
// fire and no index can leave its array, and the launch itself, which runs
// only with exactly the arguments its prepare call accepted.
#include <cuda_runtime.h>

#include <cstdarg>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <vector>

namespace {

// Argument structs, laid out as the reference's #[repr(C)] structs
// (gpu_radix_partition.rs:41-58 and :123-141, cuda_radix_join.rs:77-95) and
// their C++ counterparts (include/gpu_radix_partition.h:37-119,
// cudautils/radix_join.cu:35-49).
struct RgPrefixSumArgs {
  const void *partition_attr;
  size_t data_len;
  size_t canonical_chunk_len;
  uint32_t padding_len;
  uint32_t radix_bits;
  uint32_t ignore_bits;
  void *prefix_scan_state;
  unsigned long long *tmp_partition_offsets;
  unsigned long long *partition_offsets;
};
static_assert(sizeof(RgPrefixSumArgs) == 64, "PrefixSumArgs layout");

struct RgRadixPartitionArgs {
  const void *partition_attr_data;
  const void *payload_attr_data;
  size_t data_len;
  uint32_t padding_len;
  uint32_t radix_bits;
  uint32_t ignore_bits;
  const unsigned long long *partition_offsets;
  const uint32_t *tmp_partition_offsets;
  const char *l2_cache_buffers;
  const char *device_memory_buffers;
  uint64_t device_memory_buffer_bytes;
  void *partitioned_relation;
};
static_assert(sizeof(RgRadixPartitionArgs) == 88, "RadixPartitionArgs layout");

struct RgJoinAggregateArgs {
  const void *build_rel;
  const uint64_t *build_rel_partition_offsets;
  const void *probe_rel;
  const uint64_t *probe_rel_partition_offsets;
  int64_t *aggregation_result;
  uint32_t *task_assignments;
  uint32_t build_rel_len;
  uint32_t probe_rel_len;
  uint32_t build_rel_padding_len;
  uint32_t probe_rel_padding_len;
  uint32_t radix_bits;
  uint32_t ignore_bits;
  uint32_t ht_entries;
};
static_assert(sizeof(RgJoinAggregateArgs) == 80, "JoinAggregateArgs layout");

// sql-ops/build.rs:47-72
constexpr uint32_t kAlignBytes = 128;
constexpr uint32_t kPaddingBytes = 128;
constexpr uint32_t kLog2NumBanks = 5;
constexpr uint32_t kLaswwcTuplesPerThread = 5;
constexpr uint32_t kChainingBuckets = 2048;

char g_err[512];

int fail(int code, const char *fmt, ...) {
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(g_err, sizeof(g_err), fmt, ap);
  va_end(ap);
  return code;
}

int cuda_fail(cudaError_t e, const char *what) {
  return fail(-3, "%s: %s", what, cudaGetErrorString(e));
}

int max_smem_optin(uint32_t *out) {
  int dev = 0, v = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return cuda_fail(e, "cudaGetDevice");
  e = cudaDeviceGetAttribute(&v, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
  if (e != cudaSuccess) return cuda_fail(e, "cudaDeviceGetAttribute");
  *out = (uint32_t)v;
  return 0;
}

bool pow2(uint32_t x) { return x && !(x & (x - 1)); }

// Arguments a prepare call accepted; the launch must repeat them exactly.
struct Token {
  std::vector<unsigned char> bytes;
  bool valid = false;
};
Token g_partition_token, g_join_token;

template <typename... A>
std::vector<unsigned char> pack(const A &...a) {
  std::vector<unsigned char> v;
  auto put = [&v](const void *p, size_t n) {
    const unsigned char *c = static_cast<const unsigned char *>(p);
    v.insert(v.end(), c, c + n);
  };
  (put(&a, sizeof(a)), ...);
  return v;
}

// Largest (u64(key) >> shift) over the tuples of every partition range
// [begin[p], end[p]) of an AoS relation; keys are sign-extended to 64 bits
// first, as the reference's key_to_partition does.
template <typename K>
__global__ void max_shifted_key_kernel(const K *rel, const uint64_t *begin,
                                       const uint64_t *end, uint32_t parts,
                                       uint32_t shift,
                                       unsigned long long *out) {
  unsigned long long m = 0;
  for (uint32_t p = blockIdx.x; p < parts; p += gridDim.x)
    for (uint64_t i = begin[p] + threadIdx.x; i < end[p]; i += blockDim.x) {
      const unsigned long long k =
          (unsigned long long)(long long)rel[2 * i] >> shift;
      m = k > m ? k : m;
    }
  if (m) atomicMax(out, m);
}

}  // namespace

// The reference kernels (defined in the reference's radix_partition.cu and
// radix_join.cu; the names are C symbols, so these declarations bind to them).
extern "C" __global__ void gpu_chunked_prefix_sum_int32(RgPrefixSumArgs);
extern "C" __global__ void gpu_chunked_prefix_sum_int64(RgPrefixSumArgs);
extern "C" __global__ void gpu_chunked_radix_partition_int32_int32(RgRadixPartitionArgs);
extern "C" __global__ void gpu_chunked_radix_partition_int64_int64(RgRadixPartitionArgs);
extern "C" __global__ void gpu_chunked_laswwc_radix_partition_int32_int32(
    RgRadixPartitionArgs, uint32_t);
extern "C" __global__ void gpu_chunked_laswwc_radix_partition_int64_int64(
    RgRadixPartitionArgs, uint32_t);
extern "C" __global__ void gpu_radix_join_assign_tasks(RgJoinAggregateArgs);
extern "C" __global__ void gpu_join_aggregate_smem_perfect_i32_i32_i32(RgJoinAggregateArgs);
extern "C" __global__ void gpu_join_aggregate_smem_perfect_i64_i64_i64(RgJoinAggregateArgs);
extern "C" __global__ void gpu_join_aggregate_smem_chaining_i32_i32_i32(
    RgJoinAggregateArgs, uint32_t);
extern "C" __global__ void gpu_join_aggregate_smem_chaining_i64_i64_i64(
    RgJoinAggregateArgs, uint32_t);

extern "C" const char *rg_last_error() { return g_err; }

// Padding tuples in front of every partition (partitioned_relation.rs:27-29).
extern "C" uint32_t rg_padding_len(int key_bytes) {
  return kPaddingBytes / (2u * (uint32_t)key_bytes);
}

// ---------------------------------------------------------------------------
// Chunked prefix sum: grid = chunks, shared memory = (block + block/32 +
// fanout) u32 (gpu_radix_partition.rs:655-679).  offsets: chunks * 2^bits u64.
// ---------------------------------------------------------------------------
static int check_prefix_sum(int key_bytes, const void *keys, uint64_t len,
                            uint32_t chunks, uint32_t radix_bits,
                            uint32_t ignore_bits, const uint64_t *offsets,
                            uint32_t block, uint32_t *smem) {
  if (key_bytes != 4 && key_bytes != 8) return fail(-1, "key_bytes must be 4 or 8");
  if (chunks == 0) return fail(-1, "chunks must be at least 1");
  if (!pow2(block) || block < 32 || block > 1024)
    return fail(-1, "block must be a power of two in [32, 1024]");
  if (radix_bits > 20 || ignore_bits + radix_bits > 64)
    return fail(-1, "radix_bits/ignore_bits out of range");
  if (!offsets || (len && !keys)) return fail(-1, "null pointer");
  if ((len + chunks - 1) / chunks >= 0xffffffffull)
    return fail(-2, "chunk length overflows u32");
  uint32_t max_smem = 0;
  int rc = max_smem_optin(&max_smem);
  if (rc) return rc;
  *smem = (block + (block >> kLog2NumBanks) + (1u << radix_bits)) * 4u;
  if (*smem > max_smem) return fail(-1, "prefix sum needs %u B of shared memory", *smem);
  return 0;
}

static int launch_prefix_sum(int key_bytes, const void *keys, uint64_t len,
                             uint32_t chunks, uint32_t radix_bits,
                             uint32_t ignore_bits, uint64_t *offsets,
                             uint32_t block, uint32_t smem, cudaStream_t s) {
  const uint64_t align = kAlignBytes / (uint64_t)key_bytes;
  RgPrefixSumArgs a{keys,
                    (size_t)len,
                    (size_t)(((len + chunks - 1) / chunks) & ~(align - 1)),
                    rg_padding_len(key_bytes),
                    radix_bits,
                    ignore_bits,
                    nullptr,
                    nullptr,
                    reinterpret_cast<unsigned long long *>(offsets)};
  const void *fn = key_bytes == 4 ? (const void *)gpu_chunked_prefix_sum_int32
                                  : (const void *)gpu_chunked_prefix_sum_int64;
  cudaError_t e = cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       (int)smem);
  if (e != cudaSuccess) return cuda_fail(e, "cudaFuncSetAttribute");
  void *args[] = {&a};
  e = cudaLaunchKernel(fn, dim3(chunks), dim3(block), args, smem, s);
  return e == cudaSuccess ? 0 : cuda_fail(e, "prefix sum launch");
}

extern "C" int rg_chunked_prefix_sum(int key_bytes, const void *keys,
                                     uint64_t len, uint32_t chunks,
                                     uint32_t radix_bits, uint32_t ignore_bits,
                                     uint64_t *offsets, uint32_t block,
                                     void *stream) {
  uint32_t smem = 0;
  int rc = check_prefix_sum(key_bytes, keys, len, chunks, radix_bits,
                            ignore_bits, offsets, block, &smem);
  if (rc) return rc;
  return launch_prefix_sum(key_bytes, keys, len, chunks, radix_bits,
                           ignore_bits, offsets, block, smem,
                           (cudaStream_t)stream);
}

// ---------------------------------------------------------------------------
// Chunked scatter, variant 0 = NC (shared memory: fanout u32), 1 = LASWWC
// (all opt-in shared memory, gpu_radix_partition.rs:1139-1175).
//
// rg_partition_prepare recomputes the reference prefix sum of the keys and
// requires the caller's offsets to equal it, so every tuple lands inside its
// region; it also requires the relation to hold len + chunks * fanout * pad
// tuples, 16-byte aligned columns and relation, and LASWWC's buffers to fit
// shared memory (its asserts, radix_partition.cu:558-569).
// ---------------------------------------------------------------------------
extern "C" int rg_partition_prepare(int variant, int key_bytes, const void *keys,
                                    const void *pays, uint64_t len,
                                    uint32_t chunks, uint32_t radix_bits,
                                    uint32_t ignore_bits, const uint64_t *offsets,
                                    void *relation, uint64_t relation_len,
                                    uint32_t block) {
  g_partition_token.valid = false;
  if (variant != 0 && variant != 1) return fail(-1, "variant must be 0 (NC) or 1 (LASWWC)");
  uint32_t psmem = 0;
  int rc = check_prefix_sum(key_bytes, keys, len, chunks, radix_bits,
                            ignore_bits, offsets, block, &psmem);
  if (rc) return rc;
  if (!relation || (len && !pays)) return fail(-1, "null pointer");
  if ((uintptr_t)keys % kAlignBytes || (uintptr_t)pays % kAlignBytes ||
      (uintptr_t)relation % 16)
    return fail(-1, "columns must be 128-byte and the relation 16-byte aligned");
  const uint64_t F = 1ull << radix_bits;
  const uint64_t pad = rg_padding_len(key_bytes);
  if (relation_len < len + chunks * F * pad)
    return fail(-1, "relation holds %llu tuples, needs %llu",
                (unsigned long long)relation_len,
                (unsigned long long)(len + chunks * F * pad));
  uint32_t max_smem = 0;
  rc = max_smem_optin(&max_smem);
  if (rc) return rc;
  if (variant == 0 && F * 4 > max_smem) return fail(-1, "NC: fanout too large");
  if (variant == 1 &&
      (uint64_t)block * kLaswwcTuplesPerThread * 2u * (uint64_t)key_bytes +
              2u * F * 4u > max_smem)
    return fail(-1, "LASWWC: buffers exceed shared memory");
  // the caller's offsets must be the reference prefix sum of these keys
  uint64_t *tmp = nullptr;
  cudaError_t e = cudaMalloc(&tmp, chunks * F * sizeof(uint64_t));
  if (e != cudaSuccess) return cuda_fail(e, "cudaMalloc");
  rc = launch_prefix_sum(key_bytes, keys, len, chunks, radix_bits, ignore_bits,
                         tmp, block, psmem, 0);
  std::vector<uint64_t> a(chunks * F), b(chunks * F);
  if (!rc) {
    e = cudaMemcpy(a.data(), tmp, a.size() * 8, cudaMemcpyDeviceToHost);
    if (e == cudaSuccess)
      e = cudaMemcpy(b.data(), offsets, b.size() * 8, cudaMemcpyDeviceToHost);
    if (e != cudaSuccess) rc = cuda_fail(e, "offset copy");
  }
  cudaFree(tmp);
  if (rc) return rc;
  if (a != b) return fail(-1, "offsets differ from the reference prefix sum of the keys");
  g_partition_token.bytes = pack(variant, key_bytes, keys, pays, len, chunks,
                                 radix_bits, ignore_bits, offsets, relation,
                                 relation_len, block);
  g_partition_token.valid = true;
  return 0;
}

extern "C" int rg_partition(int variant, int key_bytes, const void *keys,
                            const void *pays, uint64_t len, uint32_t chunks,
                            uint32_t radix_bits, uint32_t ignore_bits,
                            const uint64_t *offsets, void *relation,
                            uint64_t relation_len, uint32_t block,
                            void *stream) {
  if (!g_partition_token.valid ||
      g_partition_token.bytes != pack(variant, key_bytes, keys, pays, len, chunks,
                                      radix_bits, ignore_bits, offsets, relation,
                                      relation_len, block))
    return fail(-1, "rg_partition: arguments were not checked by rg_partition_prepare");
  uint32_t max_smem = 0;
  int rc = max_smem_optin(&max_smem);
  if (rc) return rc;
  RgRadixPartitionArgs a{keys,
                         pays,
                         (size_t)len,
                         rg_padding_len(key_bytes),
                         radix_bits,
                         ignore_bits,
                         reinterpret_cast<const unsigned long long *>(offsets),
                         nullptr,
                         nullptr,
                         nullptr,
                         0,
                         relation};
  const void *fn;
  uint32_t smem;
  if (variant == 0) {
    fn = key_bytes == 4 ? (const void *)gpu_chunked_radix_partition_int32_int32
                        : (const void *)gpu_chunked_radix_partition_int64_int64;
    smem = (1u << radix_bits) * 4u;
  } else {
    fn = key_bytes == 4 ? (const void *)gpu_chunked_laswwc_radix_partition_int32_int32
                        : (const void *)gpu_chunked_laswwc_radix_partition_int64_int64;
    smem = max_smem;
  }
  cudaError_t e = cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       (int)smem);
  if (e != cudaSuccess) return cuda_fail(e, "cudaFuncSetAttribute");
  void *args[] = {&a, &smem};
  e = cudaLaunchKernel(fn, dim3(chunks), dim3(block), args, smem,
                       (cudaStream_t)stream);
  return e == cudaSuccess ? 0 : cuda_fail(e, "partition launch");
}

// ---------------------------------------------------------------------------
// Radix join: assign_tasks<<<grid, 1>>>, then the join with all opt-in shared
// memory (cuda_radix_join.rs:209-272).  scheme 0 = perfect (ht_entries =
// smem / sizeof(HtEntry) - 1), 1 = bucket chaining (2048 buckets).
// Relations are contiguous (one chunk); lengths are the relations' padded
// lengths.
//
// rg_join_prepare checks every partition range, that each build partition
// fits the table (the asserts at radix_join.cu:131,161,251), and for perfect
// hashing that every build and probe key indexes inside the table (the
// kernel indexes shared memory with key >> ignore_bits unchecked).
// ---------------------------------------------------------------------------
static uint32_t join_ht_entries(int scheme, int key_bytes, uint32_t max_smem) {
  if (scheme == 0) return max_smem / (2u * (uint32_t)key_bytes) - 1u;
  // entries of the chaining table (radix_join.cu:206-216)
  return (max_smem - kChainingBuckets * 4u) / (2u + 2u * (uint32_t)key_bytes);
}

static int check_ranges(const uint64_t *d_off, uint64_t len, uint32_t pad,
                        uint32_t F, std::vector<uint64_t> &begin,
                        std::vector<uint64_t> &end, uint64_t *largest) {
  std::vector<uint64_t> off(F);
  cudaError_t e = cudaMemcpy(off.data(), d_off, F * 8ull, cudaMemcpyDeviceToHost);
  if (e != cudaSuccess) return cuda_fail(e, "offset copy");
  begin.resize(F);
  end.resize(F);
  *largest = 0;
  for (uint32_t p = 0; p < F; ++p) {
    if (p + 1 < F && off[p + 1] < pad) return fail(-1, "offsets below padding");
    const uint64_t up = (p + 1 < F) ? off[p + 1] - pad : len;
    if (off[p] > up || up > len) return fail(-1, "partition %u range invalid", p);
    begin[p] = off[p];
    end[p] = up;
    if (up - off[p] > *largest) *largest = up - off[p];
  }
  return 0;
}

template <typename K>
static int max_shifted_key(const void *rel, const std::vector<uint64_t> &begin,
                           const std::vector<uint64_t> &end, uint32_t shift,
                           unsigned long long *out) {
  const uint32_t F = (uint32_t)begin.size();
  uint64_t *d = nullptr;
  cudaError_t e = cudaMalloc(&d, 2 * F * 8ull + 8);
  if (e != cudaSuccess) return cuda_fail(e, "cudaMalloc");
  unsigned long long *m = reinterpret_cast<unsigned long long *>(d + 2 * F);
  e = cudaMemcpy(d, begin.data(), F * 8ull, cudaMemcpyHostToDevice);
  if (e == cudaSuccess) e = cudaMemcpy(d + F, end.data(), F * 8ull, cudaMemcpyHostToDevice);
  if (e == cudaSuccess) e = cudaMemset(m, 0, 8);
  if (e == cudaSuccess) {
    max_shifted_key_kernel<K><<<F < 4096 ? F : 4096, 256>>>(
        static_cast<const K *>(rel), d, d + F, F, shift, m);
    e = cudaGetLastError();
  }
  if (e == cudaSuccess) e = cudaMemcpy(out, m, 8, cudaMemcpyDeviceToHost);
  cudaFree(d);
  return e == cudaSuccess ? 0 : cuda_fail(e, "key range check");
}

extern "C" int rg_join_prepare(int scheme, int key_bytes, const void *build_rel,
                               const uint64_t *build_off, uint64_t build_len,
                               const void *probe_rel, const uint64_t *probe_off,
                               uint64_t probe_len, uint32_t radix_bits,
                               uint32_t ignore_bits, uint32_t grid,
                               uint32_t block, int64_t *result,
                               uint32_t *tasks) {
  g_join_token.valid = false;
  if (scheme != 0 && scheme != 1) return fail(-1, "scheme must be 0 (perfect) or 1 (chaining)");
  if (key_bytes != 4 && key_bytes != 8) return fail(-1, "key_bytes must be 4 or 8");
  if (!build_rel || !probe_rel || !build_off || !probe_off || !result || !tasks)
    return fail(-1, "null pointer");
  if ((uintptr_t)build_rel % 16 || (uintptr_t)probe_rel % 16)
    return fail(-1, "relations must be 16-byte aligned");
  if (build_len >= 0xffffffffull || probe_len >= 0xffffffffull)
    return fail(-2, "relation lengths must fit u32");
  if (radix_bits > 20 || ignore_bits >= 32) return fail(-1, "bits out of range");
  if (grid == 0 || block == 0 || block > 1024) return fail(-1, "bad launch shape");
  uint32_t max_smem = 0;
  int rc = max_smem_optin(&max_smem);
  if (rc) return rc;
  const uint32_t F = 1u << radix_bits, pad = rg_padding_len(key_bytes);
  const uint32_t ht = join_ht_entries(scheme, key_bytes, max_smem);
  std::vector<uint64_t> bb, be, pb, pe;
  uint64_t big_b = 0, big_p = 0;
  rc = check_ranges(build_off, build_len, pad, F, bb, be, &big_b);
  if (!rc) rc = check_ranges(probe_off, probe_len, pad, F, pb, pe, &big_p);
  if (rc) return rc;
  if (big_b > ht)
    return fail(-7, "a build partition holds %llu tuples; the table %u",
                (unsigned long long)big_b, ht);
  if (scheme == 0) {
    unsigned long long mb = 0, mp = 0;
    rc = key_bytes == 4 ? max_shifted_key<int32_t>(build_rel, bb, be, ignore_bits, &mb)
                        : max_shifted_key<int64_t>(build_rel, bb, be, ignore_bits, &mb);
    if (!rc)
      rc = key_bytes == 4 ? max_shifted_key<int32_t>(probe_rel, pb, pe, ignore_bits, &mp)
                          : max_shifted_key<int64_t>(probe_rel, pb, pe, ignore_bits, &mp);
    if (rc) return rc;
    if (mb >= ht || mp >= ht)
      return fail(-7, "a key indexes slot %llu of a %u-entry perfect table",
                  mb > mp ? mb : mp, ht);
  }
  g_join_token.bytes = pack(scheme, key_bytes, build_rel, build_off, build_len,
                            probe_rel, probe_off, probe_len, radix_bits,
                            ignore_bits, grid, block, result, tasks);
  g_join_token.valid = true;
  return 0;
}

extern "C" int rg_join(int scheme, int key_bytes, const void *build_rel,
                       const uint64_t *build_off, uint64_t build_len,
                       const void *probe_rel, const uint64_t *probe_off,
                       uint64_t probe_len, uint32_t radix_bits,
                       uint32_t ignore_bits, uint32_t grid, uint32_t block,
                       int64_t *result, uint32_t *tasks, void *stream) {
  if (!g_join_token.valid ||
      g_join_token.bytes != pack(scheme, key_bytes, build_rel, build_off, build_len,
                                 probe_rel, probe_off, probe_len, radix_bits,
                                 ignore_bits, grid, block, result, tasks))
    return fail(-1, "rg_join: arguments were not checked by rg_join_prepare");
  uint32_t max_smem = 0;
  int rc = max_smem_optin(&max_smem);
  if (rc) return rc;
  const uint32_t pad = rg_padding_len(key_bytes);
  RgJoinAggregateArgs a{build_rel,
                        build_off,
                        probe_rel,
                        probe_off,
                        result,
                        tasks,
                        (uint32_t)build_len,
                        (uint32_t)probe_len,
                        pad,
                        pad,
                        radix_bits,
                        ignore_bits,
                        scheme == 0 ? join_ht_entries(0, key_bytes, max_smem)
                                    : kChainingBuckets};
  cudaStream_t s = (cudaStream_t)stream;
  void *targs[] = {&a};
  cudaError_t e = cudaLaunchKernel((const void *)gpu_radix_join_assign_tasks,
                                   dim3(grid), dim3(1), targs, 0, s);
  if (e != cudaSuccess) return cuda_fail(e, "assign_tasks launch");
  const void *fn;
  if (scheme == 0)
    fn = key_bytes == 4 ? (const void *)gpu_join_aggregate_smem_perfect_i32_i32_i32
                        : (const void *)gpu_join_aggregate_smem_perfect_i64_i64_i64;
  else
    fn = key_bytes == 4 ? (const void *)gpu_join_aggregate_smem_chaining_i32_i32_i32
                        : (const void *)gpu_join_aggregate_smem_chaining_i64_i64_i64;
  e = cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize,
                           (int)max_smem);
  if (e != cudaSuccess) return cuda_fail(e, "cudaFuncSetAttribute");
  uint32_t smem_arg = max_smem;
  void *jargs[] = {&a, &smem_arg};
  e = cudaLaunchKernel(fn, dim3(grid), dim3(block), jargs, max_smem, s);
  return e == cudaSuccess ? 0 : cuda_fail(e, "join launch");
}
