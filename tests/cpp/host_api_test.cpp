// The C++ host API (include/fi_sqlops.hpp) on one GPU, in the shape of the
// reference's own Rust tests of the path:
//  * a Chunked prefix sum + partition (sql-ops/tests/radix_partition/mod.rs):
//    offsets equal to a host recomputation of the chunked prefix sum
//    (radix_partition.cu:40-96 semantics), every stored key inside its
//    region's partition, no tuple lost or duplicated;
//  * the radix join known answer (sql-ops/tests/test_cuda_radix_join.rs:
//    179-182): keys a permutation of 0..N-1 on both sides, payload = row + 1,
//    SUM(s.value) = N (N + 1) / 2, for both hashing schemes;
//  * the no-partitioning join, grouped by table region and in input order:
//    SUM of probe payloads 1 = the number of probes, every key present;
//  * the reference's argument check: mismatching radix bits raise
//    ErrorKind::InvalidArgument with the reference's message.
// Prints "host api ok" and exits 0 when everything holds.
#include <algorithm>
#include <cstdio>
#include <cstring>
#include <numeric>
#include <random>
#include <vector>

#include "fi_sqlops.hpp"

using namespace fi_sqlops;

#define REQUIRE(cond)                                                     \
  do {                                                                    \
    if (!(cond)) {                                                        \
      std::fprintf(stderr, "%s:%d: check failed: %s\n", __FILE__, __LINE__, #cond); \
      return 1;                                                           \
    }                                                                     \
  } while (0)

template <typename T>
static DeviceBuffer<T> upload(const std::vector<T> &h) {
  DeviceBuffer<T> d(h.size());
  check_cuda(cudaMemcpy(d.data(), h.data(), h.size() * sizeof(T), cudaMemcpyHostToDevice),
             "upload");
  return d;
}

template <typename T>
static std::vector<T> download(const T *d, size_t n) {
  std::vector<T> h(n);
  check_cuda(cudaMemcpy(h.data(), d, n * sizeof(T), cudaMemcpyDeviceToHost), "download");
  return h;
}

static int partition_test() {
  const uint64_t n = 1000003;
  const uint32_t chunks = 64, bits = 8, F = 1u << bits;
  std::vector<int64_t> keys(n), pays(n);
  std::iota(keys.begin(), keys.end(), 0);
  std::shuffle(keys.begin(), keys.end(), std::mt19937_64(42));
  for (uint64_t i = 0; i < n; ++i) pays[i] = 3 * keys[i] + 1;
  auto dk = upload(keys), dp = upload(pays);
  GpuRadixPartitioner p(GpuHistogramAlgorithm::Chunked, GpuRadixPartitionAlgorithm::SSWWCv2,
                        RadixBits(bits), chunks, 1024);
  PartitionOffsets<int64_t> o(GpuHistogramAlgorithm::Chunked, chunks, bits);
  PartitionedRelation<int64_t> rel(n, GpuHistogramAlgorithm::Chunked, bits, chunks);
  p.prefix_sum(RadixPass::First, dk.data(), n, o, nullptr);
  p.partition(RadixPass::First, dk.data(), dp.data(), n, o, rel, nullptr);
  check_cuda(cudaDeviceSynchronize(), "sync");
  p.status();
  // host recomputation of the chunked offsets
  const uint32_t pad = rel.padding_len();
  const uint64_t clen = ((n + chunks - 1) / chunks) & ~uint64_t(15);
  std::vector<uint64_t> exp(chunks * F);
  for (uint32_t c = 0; c < chunks; ++c) {
    const uint64_t b = clen * c, e = (c + 1 == chunks) ? n : b + clen;
    std::vector<uint64_t> hist(F, 0);
    for (uint64_t i = b; i < e; ++i) ++hist[(uint64_t)keys[i] & (F - 1)];
    uint64_t run = 0;
    for (uint32_t q = 0; q < F; ++q) {
      exp[c * F + q] = run + (clen + pad * F) * c + (q + 1) * pad;
      run += hist[q];
    }
  }
  const auto off = download(rel.offsets(), chunks * F);
  REQUIRE(off == exp);
  const auto tuples = download(rel.relation(), rel.padded_len());
  std::vector<char> seen(n, 0);
  for (uint32_t r = 0; r < chunks * F; ++r) {
    const uint64_t b = off[r], e = (r + 1 < chunks * F) ? off[r + 1] - pad : rel.padded_len();
    for (uint64_t i = b; i < e; ++i) {
      const auto &t = tuples[i];
      REQUIRE(t.key >= 0 && (uint64_t)t.key < n);
      REQUIRE(((uint64_t)t.key & (F - 1)) == r % F);
      REQUIRE(t.value == 3 * t.key + 1);
      REQUIRE(!seen[t.key]);
      seen[t.key] = 1;
    }
  }
  REQUIRE(std::all_of(seen.begin(), seen.end(), [](char x) { return x == 1; }));
  REQUIRE(rel.partition_len(5) > 0);
  return 0;
}

static int join_test(HashingScheme scheme) {
  const uint64_t n = 4096u * 64;  // 4096 tuples per partition at 6 bits
  const uint32_t bits = 6, grid = 37, block = 256;
  std::vector<int64_t> rk(n), sk(n), pay(n);
  std::iota(rk.begin(), rk.end(), 0);
  std::iota(sk.begin(), sk.end(), 0);
  std::shuffle(rk.begin(), rk.end(), std::mt19937_64(1));
  std::shuffle(sk.begin(), sk.end(), std::mt19937_64(2));
  std::iota(pay.begin(), pay.end(), 1);
  auto drk = upload(rk), dsk = upload(sk), dpay = upload(pay);
  GpuRadixPartitioner p(GpuHistogramAlgorithm::Chunked, GpuRadixPartitionAlgorithm::NC,
                        RadixBits(bits), 1, 1024);
  PartitionedRelation<int64_t> b(n, GpuHistogramAlgorithm::Chunked, bits, 1);
  PartitionedRelation<int64_t> pr(n, GpuHistogramAlgorithm::Chunked, bits, 1);
  for (auto *side : {&b, &pr}) {
    PartitionOffsets<int64_t> o(GpuHistogramAlgorithm::Chunked, 1, bits);
    const int64_t *k = side == &b ? drk.data() : dsk.data();
    p.prefix_sum(RadixPass::First, k, n, o, nullptr);
    p.partition(RadixPass::First, k, dpay.data(), n, o, *side, nullptr);
  }
  DeviceBuffer<int64_t> result(grid * block);
  DeviceBuffer<uint32_t> tasks(grid + 1);
  check_cuda(cudaMemset(result.data(), 0, grid * block * sizeof(int64_t)), "memset");
  CudaRadixJoin j(RadixPass::First, RadixBits(bits), scheme, grid, block);
  j.join(b, pr, result.data(), grid * block, tasks.data(), grid + 1, nullptr);
  check_cuda(cudaDeviceSynchronize(), "sync");
  j.status();
  const auto r = download(result.data(), grid * block);
  uint64_t sum = 0;
  for (int64_t v : r) sum += (uint64_t)v;
  REQUIRE(sum == n * (n + 1) / 2);
  return 0;
}

// No-partitioning join (sql-ops/tests/test_no_partitioning_join.rs shape):
// unique build keys 0..N-1, every probe key among them, probe payload 1, so
// SUM = the number of probes; grouped by table region (the default; a 16 MB
// table is two 8 MB regions) and in input order.
static int hash_join_test(HashingScheme scheme) {
  const uint64_t nb = 1u << 19, np = 1u << 21;
  const uint64_t size = 1u << 20;  // 16 MB of int64 entries: two regions
  const uint32_t grid = 148, block = 256;
  std::vector<int64_t> rk(nb), sk(np), ones(np, 1);
  std::iota(rk.begin(), rk.end(), 0);
  std::shuffle(rk.begin(), rk.end(), std::mt19937_64(3));
  for (uint64_t i = 0; i < np; ++i) sk[i] = (int64_t)((i * 2654435761u) % nb);
  auto drk = upload(rk), dsk = upload(sk), dones = upload(ones);
  for (bool grouped : {true, false}) {
    HashTable<int64_t> table(size, nullptr);
    CudaHashJoin<int64_t> hj(scheme, false, table, grid, block, grid, block);
    hj.set_build_grouping(grouped);
    hj.set_probe_grouping(grouped);
    DeviceBuffer<uint64_t> result(grid * block);
    check_cuda(cudaMemset(result.data(), 0, grid * block * sizeof(uint64_t)), "memset");
    hj.build(drk.data(), drk.data(), nb, nullptr);
    hj.probe_sum(dsk.data(), dones.data(), np, result.data(), grid * block, nullptr);
    check_cuda(cudaDeviceSynchronize(), "sync");
    hj.status();
    const auto r = download(result.data(), grid * block);
    uint64_t sum = 0;
    for (uint64_t v : r) sum += v;
    REQUIRE(sum == np);
  }
  return 0;
}

static int error_test() {
  GpuRadixPartitioner p(GpuHistogramAlgorithm::Chunked, GpuRadixPartitionAlgorithm::NC,
                        RadixBits(8), 4, 1024);
  PartitionOffsets<int64_t> o(GpuHistogramAlgorithm::Chunked, 4, 7);
  DeviceBuffer<int64_t> k(16);
  try {
    p.prefix_sum(RadixPass::First, k.data(), 16, o, nullptr);
  } catch (const Error &e) {
    REQUIRE(e.kind() == ErrorKind::InvalidArgument);
    REQUIRE(std::strstr(e.what(), "mismatching radix bits") != nullptr);
    return 0;
  }
  REQUIRE(false && "the mismatch was not reported");
  return 1;
}

int main() {
  try {
    if (partition_test()) return 1;
    if (join_test(HashingScheme::BucketChaining)) return 1;
    if (join_test(HashingScheme::Perfect)) return 1;
    if (hash_join_test(HashingScheme::LinearProbing)) return 1;
    if (hash_join_test(HashingScheme::Perfect)) return 1;
    if (error_test()) return 1;
  } catch (const Error &e) {
    std::fprintf(stderr, "error %d: %s\n", e.code(), e.what());
    return 1;
  }
  std::printf("host api ok\n");
  return 0;
}
