// No-partitioning hash join on the CPU: the counterpart of the reference's
// CpuHashJoin (sql-ops/src/join/no_partitioning_join.rs:153-304, kernels in
// sql-ops/cpputils/no_partitioning_join.cpp:27-273), beside the GPU
// CudaHashJoin of hash_join.cu.
//
// Same table and rules as the reference's CPU kernels: a caller-owned array
// of {key, value} entries whose keys start as the null key (all ones; the
// values need no initial contents); linear probing inserts at
// mult_shift_hash(key) mod 2^floor(log2(size)), claims the first null key
// slot from there with a compare-and-swap of the key, then stores the value,
// and a probe adds its payload for every matching slot up to the first empty
// one; perfect hashing stores (key, value) at index key (null keys skipped
// when the join is selective) and a probe matches when that slot holds its
// key.  Keys outside [0, size) are skipped by the perfect build and probe
// (the reference indexes with them unchecked).  Builds may run concurrently
// on disjoint slices of the build relation (the reference's threads share
// one table); every probe adds into the caller's u64 result (wrapping).
#include <cstdint>
#include <cstring>
#include <new>

#include "../../include/fi_sqlops.h"
#include "api_internal.h"
#include "common.cuh"

struct fi_cpu_hash_join {
  fi_hashing_scheme scheme;
  bool selective;
  void *table;
  uint64_t mem_len, size;
};

namespace fi {
namespace {

inline uint32_t floor_log2(uint64_t x) { return 63u - (uint32_t)__builtin_clzll(x); }

inline uint64_t cpu_hash(int32_t k, uint32_t lg) {
  return lg ? (uint64_t)(((uint32_t)k * 2654435769u) >> (32u - lg)) : 0;
}
inline uint64_t cpu_hash(int64_t k, uint32_t lg) {
  return lg ? (((uint64_t)k * 11400714819323198485ull) >> (64u - lg)) : 0;
}

template <typename K>
void lp_insert(Tuple<K> *ht, uint32_t lg, K key, K pay) {
  const uint64_t n = 1ull << lg, m = n - 1;
  uint64_t idx = cpu_hash(key, lg);
  for (uint64_t i = 0; i < n; ++i, idx = (idx + 1) & m) {
    K expect = null_key<K>();
    if (__atomic_load_n(&ht[idx].key, __ATOMIC_RELAXED) == expect &&
        __atomic_compare_exchange_n(&ht[idx].key, &expect, key, false, __ATOMIC_RELAXED,
                                    __ATOMIC_RELAXED)) {
      ht[idx].value = pay;
      return;
    }
  }
}

template <typename K>
int cpu_build(fi_cpu_hash_join *hj, const K *key, const K *pay, uint64_t len) {
  if (!hj || (len && (!key || !pay)))
    return set_error(FI_ERR_INVALID_ARGUMENT, "null argument");
  if (len > hj->mem_len)
    return set_error(FI_ERR_INVALID_ARGUMENT, "Hash table is too small for the build data");
  auto *ht = static_cast<Tuple<K> *>(hj->table);
  if (hj->scheme == FI_HASHING_LINEAR_PROBING) {
    if (hj->selective)
      return set_error(FI_ERR_UNSUPPORTED, "selective linear probing builds are not supported");
    const uint32_t lg = floor_log2(hj->size);
    for (uint64_t i = 0; i < len; ++i) lp_insert(ht, lg, key[i], pay[i]);
  } else {
    for (uint64_t i = 0; i < len; ++i) {
      const K k = key[i];
      if (hj->selective && k == null_key<K>()) continue;
      const uint64_t slot = (uint64_t)(int64_t)k;
      if (slot < hj->size) ht[slot] = Tuple<K>{k, pay[i]};
    }
  }
  return FI_OK;
}

template <typename K>
int cpu_probe_sum(fi_cpu_hash_join *hj, const K *key, const K *pay, uint64_t len,
                  uint64_t *result) {
  if (!hj || !result || (len && (!key || !pay)))
    return set_error(FI_ERR_INVALID_ARGUMENT, "null argument");
  const auto *ht = static_cast<const Tuple<K> *>(hj->table);
  uint64_t sum = 0;
  if (hj->scheme == FI_HASHING_LINEAR_PROBING) {
    const uint32_t lg = floor_log2(hj->size);
    const uint64_t n = 1ull << lg, m = n - 1;
    for (uint64_t i = 0; i < len; ++i) {
      const K k = key[i];
      uint64_t idx = cpu_hash(k, lg);
      for (uint64_t s = 0; s < n; ++s, idx = (idx + 1) & m) {
        const K e = __atomic_load_n(&ht[idx].key, __ATOMIC_RELAXED);
        if (e == k)
          sum += (uint64_t)(int64_t)pay[i];
        else if (e == null_key<K>())
          break;
      }
    }
  } else {
    for (uint64_t i = 0; i < len; ++i) {
      const K k = key[i];
      const uint64_t slot = (uint64_t)(int64_t)k;
      if (slot < hj->size && ht[slot].key == k) sum += (uint64_t)(int64_t)pay[i];
    }
  }
  __atomic_fetch_add(result, sum, __ATOMIC_RELAXED);
  return FI_OK;
}

}  // namespace
}  // namespace fi

using namespace fi;

extern "C" int fi_cpu_hash_table_init_int32(void *table, uint64_t entries) {
  if (!table && entries) return set_error(FI_ERR_INVALID_ARGUMENT, "null table");
  std::memset(table, 0xff, entries * sizeof(Tuple<int32_t>));
  return FI_OK;
}
extern "C" int fi_cpu_hash_table_init_int64(void *table, uint64_t entries) {
  if (!table && entries) return set_error(FI_ERR_INVALID_ARGUMENT, "null table");
  std::memset(table, 0xff, entries * sizeof(Tuple<int64_t>));
  return FI_OK;
}

extern "C" int fi_cpu_hash_join_new(fi_hashing_scheme hashing_scheme, int is_selective,
                                    void *hash_table, uint64_t mem_len, uint64_t size,
                                    fi_cpu_hash_join **out) {
  if (!out) return set_error(FI_ERR_INVALID_ARGUMENT, "null output handle");
  *out = nullptr;
  if (hashing_scheme != FI_HASHING_LINEAR_PROBING && hashing_scheme != FI_HASHING_PERFECT)
    return set_error(FI_ERR_UNSUPPORTED,
                     "the no-partitioning join supports LinearProbing and Perfect");
  if (!hash_table || size == 0 || size > mem_len)
    return set_error(FI_ERR_INVALID_ARGUMENT,
                     "hash table size must lie in [1, the table's length]");
  auto *hj = new (std::nothrow) fi_cpu_hash_join{hashing_scheme, is_selective != 0,
                                                 hash_table, mem_len, size};
  if (!hj) return set_error(FI_ERR_OUT_OF_MEMORY, "hash join");
  *out = hj;
  return FI_OK;
}

extern "C" void fi_cpu_hash_join_free(fi_cpu_hash_join *hj) { delete hj; }

extern "C" int fi_cpu_hash_join_build_int32(fi_cpu_hash_join *hj, const int32_t *key,
                                            const int32_t *pay, uint64_t len) {
  return cpu_build<int32_t>(hj, key, pay, len);
}
extern "C" int fi_cpu_hash_join_build_int64(fi_cpu_hash_join *hj, const int64_t *key,
                                            const int64_t *pay, uint64_t len) {
  return cpu_build<int64_t>(hj, key, pay, len);
}
extern "C" int fi_cpu_hash_join_probe_sum_int32(fi_cpu_hash_join *hj, const int32_t *key,
                                                const int32_t *pay, uint64_t len,
                                                uint64_t *result) {
  return cpu_probe_sum<int32_t>(hj, key, pay, len, result);
}
extern "C" int fi_cpu_hash_join_probe_sum_int64(fi_cpu_hash_join *hj, const int64_t *key,
                                                const int64_t *pay, uint64_t len,
                                                uint64_t *result) {
  return cpu_probe_sum<int64_t>(hj, key, pay, len, result);
}
