// Autotuner: execution plan per (tuple type, |R|, |S|, skew).
//
// The reference picks its radix bits by hand per benchmark; its script
// computes the first-pass bits from the build size and the usable shared
// memory (scripts/benchmark_gpu_radix_join.py:92) and fixes the second pass
// at 9 bits (:57).  Here a plan comes from, in order:
//   1. a measured table (fi_autotune_load), written by the tuning sweep
//      (autotune.py beside the library): the nearest entry of the same tuple
//      type by |log2 |R| - e.log2r| + |log2 k - e.log2k| + 2 |skew - e.skew|,
//      if that distance is at most 1.5;
//   2. a model: final partitions of about 4K build tuples (one
//      shared-memory table each; the 1024M x 1024M int64 join runs fastest
//      with 2^30 / 2^18), one pass up to 11 bits and two balanced passes
//      above (a single pass loses its write combining above 11 bits on
//      B200), bucket chaining, the join shape chosen by partition size
//      (join_auto_block), TMA-fed scatters.
// Joins below small_tuples in total go to batches.
#include <cmath>
#include <cstdio>
#include <cstring>
#include <mutex>
#include <vector>

#include "../../include/fi_sqlops.h"
#include "api_internal.h"
#include "batch.h"

namespace fi {
namespace {

struct TableEntry {
  uint32_t tuple_bytes;
  double log2r, log2k;
  uint32_t skew;
  int32_t bits1, bits2;
  int scheme;
  uint32_t join_block, scatter;
};

std::mutex g_table_mu;
std::vector<TableEntry> g_table;

constexpr uint64_t kDefaultSmall = 4ull << 20;

uint32_t ceil_log2(uint64_t x) {
  uint32_t b = 0;
  while (b < 63 && (1ull << b) < x) ++b;
  return b;
}

}  // namespace

void autotune_model(uint64_t build_len, fi_tuned_plan *out) {
  out->batched = 0;
  const uint64_t per = 4096;  // build tuples per final partition
  uint32_t total = build_len > per ? ceil_log2((build_len + per - 1) / per) : 0;
  if (total > 20) total = 20;
  if (total <= kSingleLevelBits) {
    out->radix_bits.pass_bits[0] = (int32_t)total;
    out->radix_bits.pass_bits[1] = -1;
  } else {
    out->radix_bits.pass_bits[0] = (int32_t)((total + 1) / 2);
    out->radix_bits.pass_bits[1] = (int32_t)(total / 2);
  }
  out->radix_bits.pass_bits[2] = -1;
  out->hashing_scheme = FI_HASHING_BUCKET_CHAINING;
  out->join_block = 0;  // by partition size (join_auto_block)
  out->scatter = 0;
}

}  // namespace fi

extern "C" int fi_autotune_plan(uint32_t tuple_bytes, uint64_t build_len,
                                uint64_t probe_len, uint32_t skew,
                                uint64_t small_tuples, fi_tuned_plan *out) {
  using namespace fi;
  if (!out) return set_error(FI_ERR_INVALID_ARGUMENT, "null output");
  if (tuple_bytes != 8 && tuple_bytes != 16)
    return set_error(FI_ERR_INVALID_ARGUMENT, "tuple_bytes must be 8 or 16");
  std::memset(out, 0, sizeof *out);
  const uint64_t small = small_tuples ? small_tuples : kDefaultSmall;
  if (build_len + probe_len < small) {
    out->batched = 1;
    out->radix_bits.pass_bits[0] = (int32_t)batch_bits(build_len);
    out->radix_bits.pass_bits[1] = -1;
    out->radix_bits.pass_bits[2] = -1;
    out->hashing_scheme = FI_HASHING_BUCKET_CHAINING;
    out->join_block = 512;
    return FI_OK;
  }
  autotune_model(build_len, out);
  std::lock_guard<std::mutex> lk(g_table_mu);
  const double lr = std::log2((double)(build_len ? build_len : 1));
  const double lk2 = std::log2((double)(probe_len ? probe_len : 1) /
                               (double)(build_len ? build_len : 1));
  const TableEntry *best = nullptr;
  double best_d = 1e30;
  for (const TableEntry &e : g_table) {
    if (e.tuple_bytes != tuple_bytes) continue;
    const double d = std::fabs(lr - e.log2r) + std::fabs(lk2 - e.log2k) +
                     2.0 * std::fabs((double)skew - (double)e.skew);
    if (d < best_d) {
      best_d = d;
      best = &e;
    }
  }
  if (best && best_d <= 1.5) {
    out->radix_bits.pass_bits[0] = best->bits1;
    out->radix_bits.pass_bits[1] = best->bits2;
    out->hashing_scheme = (fi_hashing_scheme)best->scheme;
    out->join_block = best->join_block;
    out->scatter = best->scatter;
  }
  return FI_OK;
}

extern "C" int fi_autotune_load(const char *path) {
  using namespace fi;
  std::vector<TableEntry> t;
  if (path) {
    FILE *f = std::fopen(path, "r");
    if (!f) return set_error(FI_ERR_INVALID_ARGUMENT, "cannot open %s", path);
    char line[512];
    int lineno = 0;
    while (std::fgets(line, sizeof line, f)) {
      ++lineno;
      char *p = line;
      while (*p == ' ' || *p == '\t') ++p;
      if (*p == '#' || *p == '\n' || *p == 0) continue;
      TableEntry e{};
      if (std::sscanf(p, "%u %lf %lf %u %d %d %d %u %u", &e.tuple_bytes, &e.log2r,
                      &e.log2k, &e.skew, &e.bits1, &e.bits2, &e.scheme,
                      &e.join_block, &e.scatter) != 9 ||
          (e.tuple_bytes != 8 && e.tuple_bytes != 16) || e.bits1 < 0 ||
          e.bits1 > 14 || e.bits2 > 10 ||
          (e.scheme != FI_HASHING_PERFECT && e.scheme != FI_HASHING_BUCKET_CHAINING) ||
          (e.join_block != 0 && e.join_block != 256 && e.join_block != 512 &&
           e.join_block != 1024) ||
          e.scatter > 1) {
        std::fclose(f);
        return set_error(FI_ERR_INVALID_ARGUMENT, "%s:%d: malformed tuning entry",
                         path, lineno);
      }
      t.push_back(e);
    }
    std::fclose(f);
  }
  std::lock_guard<std::mutex> lk(g_table_mu);
  g_table.swap(t);
  return FI_OK;
}
