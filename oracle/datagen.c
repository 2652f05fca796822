/*
 * Seeded relation generator, CPU side.  TEST INFRASTRUCTURE ONLY.
 *
 * The reference generates its relations with unseeded `thread_rng`
 * (datagen/src/relation.rs:93,159,173), so its inputs are not reproducible.
 * Parity is therefore defined on inputs generated here with an explicit seed
 * and fed to both the CUDA path and the oracle.  The GPU library carries the
 * same generator (fast-interconnects_b200/csrc/datagen.cu); for the
 * permutation and the uniform foreign keys the two produce identical bits,
 * which tests/test_datagen.py checks.
 *
 * Shapes follow the reference's generators:
 *   - primary keys: a permutation of a dense key range
 *     (datagen/src/relation.rs:46-73 uses 0..N-1 shuffled; the benchmark
 *     configurations of this build use 1..N, so `base` is a parameter);
 *   - foreign keys: uniform over the primary-key range (relation.rs:88-151);
 *   - Zipf foreign keys: ranks 1..N with P(r) ~ r^-s, mapped to the key of
 *     primary-key row r-1 (relation.rs:228-289 maps zipf ranks to 0..N-1).
 *
 * Building blocks (published methods, restated):
 *   - SplitMix64 finaliser (Steele, Lea, Flood 2014) as the mixing function;
 *   - a 4-round balanced Feistel network over 2^(2h) >= N with cycle walking
 *     (Black & Rogaway 2002) as the seeded bijection on [0, N);
 *   - Zipf by rejection-inversion (Hoermann & Derflinger 1996).
 */
#include <math.h>
#include <stdint.h>

static inline uint64_t dg_mix64(uint64_t x) {
  uint64_t z = x + 0x9E3779B97F4A7C15ull;
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  return z ^ (z >> 31);
}

static inline uint64_t dg_mulhi(uint64_t a, uint64_t b) {
  return (uint64_t)(((unsigned __int128)a * b) >> 64);
}

typedef struct {
  uint64_t n;
  uint32_t half_bits;
  uint64_t half_mask;
  uint64_t round_key[4];
} dg_perm;

static void dg_perm_init(dg_perm *p, uint64_t n, uint64_t seed) {
  uint32_t bits = 0;
  while (bits < 64 && (1ull << bits) < n) bits++;
  uint32_t h = (bits + 1) / 2;
  if (h == 0) h = 1;
  p->n = n;
  p->half_bits = h;
  p->half_mask = (1ull << h) - 1ull;
  for (int r = 0; r < 4; ++r)
    p->round_key[r] = dg_mix64(seed * 4ull + (uint64_t)r + 0x5151ull);
}

static inline uint64_t dg_perm_apply(const dg_perm *p, uint64_t x) {
  do {
    uint64_t l = x >> p->half_bits, r = x & p->half_mask;
    for (int k = 0; k < 4; ++k) {
      uint64_t t = r;
      r = l ^ (dg_mix64(r ^ p->round_key[k]) & p->half_mask);
      l = t;
    }
    x = (l << p->half_bits) | r;
  } while (x >= p->n);
  return x;
}

/* Zipf(N, s) by rejection-inversion.  H is the integral of x^-s, written with
 * log1p/expm1 helpers so that s == 1 needs no special case. */
static inline double dg_helper1(double x) {
  return fabs(x) > 1e-8 ? log1p(x) / x : 1.0 - x * (0.5 - x * (1.0 / 3.0));
}
static inline double dg_helper2(double x) {
  return fabs(x) > 1e-8 ? expm1(x) / x : 1.0 + x * 0.5 * (1.0 + x / 3.0);
}
static inline double dg_h_int(double x, double s) {
  double lx = log(x);
  return dg_helper2((1.0 - s) * lx) * lx;
}
static inline double dg_h(double x, double s) { return exp(-s * log(x)); }
static inline double dg_h_int_inv(double x, double s) {
  double t = x * (1.0 - s);
  if (t < -1.0) t = -1.0;
  return exp(dg_helper1(t) * x);
}

static inline uint64_t dg_zipf_rank(uint64_t n, double s, uint64_t seed,
                                    uint64_t i) {
  const double hx1 = dg_h_int(1.5, s) - 1.0;
  const double hn = dg_h_int((double)n + 0.5, s);
  const double sq = 2.0 - dg_h_int_inv(dg_h_int(2.5, s) - dg_h(2.0, s), s);
  for (uint64_t attempt = 0;; ++attempt) {
    uint64_t bits = dg_mix64(seed ^ dg_mix64(i * 64ull + attempt));
    double u01 = (double)(bits >> 11) * (1.0 / 9007199254740992.0);
    double u = hn + u01 * (hx1 - hn);
    double x = dg_h_int_inv(u, s);
    double kf = floor(x + 0.5);
    if (kf < 1.0) kf = 1.0;
    if (kf > (double)n) kf = (double)n;
    if (kf - x <= sq || u >= dg_h_int(kf + 0.5, s) - dg_h(kf, s))
      return (uint64_t)kf;
    if (attempt > 1000) return (uint64_t)kf;
  }
}

/* keys[i] = base + perm(i): a seeded permutation of base..base+n-1. */
void dg_primary_keys_i64(int64_t *keys, uint64_t n, uint64_t seed,
                         int64_t base) {
  dg_perm p;
  dg_perm_init(&p, n, seed);
  for (uint64_t i = 0; i < n; ++i) keys[i] = base + (int64_t)dg_perm_apply(&p, i);
}
void dg_primary_keys_i32(int32_t *keys, uint64_t n, uint64_t seed,
                         int32_t base) {
  dg_perm p;
  dg_perm_init(&p, n, seed);
  for (uint64_t i = 0; i < n; ++i) keys[i] = base + (int32_t)dg_perm_apply(&p, i);
}

/* Uniform foreign keys over base..base+pk_n-1. */
void dg_uniform_foreign_keys_i64(int64_t *keys, uint64_t n, uint64_t pk_n,
                                 uint64_t seed, int64_t base) {
  for (uint64_t i = 0; i < n; ++i)
    keys[i] = base + (int64_t)dg_mulhi(dg_mix64(seed ^ dg_mix64(i)), pk_n);
}
void dg_uniform_foreign_keys_i32(int32_t *keys, uint64_t n, uint64_t pk_n,
                                 uint64_t seed, int32_t base) {
  for (uint64_t i = 0; i < n; ++i)
    keys[i] = base + (int32_t)dg_mulhi(dg_mix64(seed ^ dg_mix64(i)), pk_n);
}

/* Zipf foreign keys: rank r ~ Zipf(pk_n, s), key = base + perm_pk(r-1), i.e.
 * the key of primary-key row r-1 generated with pk_seed.  s == 0 gives
 * uniform ranks. */
void dg_zipf_foreign_keys_i64(int64_t *keys, uint64_t n, uint64_t pk_n,
                              double s, uint64_t seed, uint64_t pk_seed,
                              int64_t base) {
  dg_perm p;
  dg_perm_init(&p, pk_n, pk_seed);
  for (uint64_t i = 0; i < n; ++i) {
    uint64_t r = dg_zipf_rank(pk_n, s, seed, i);
    keys[i] = base + (int64_t)dg_perm_apply(&p, r - 1);
  }
}
void dg_zipf_foreign_keys_i32(int32_t *keys, uint64_t n, uint64_t pk_n,
                              double s, uint64_t seed, uint64_t pk_seed,
                              int32_t base) {
  dg_perm p;
  dg_perm_init(&p, pk_n, pk_seed);
  for (uint64_t i = 0; i < n; ++i) {
    uint64_t r = dg_zipf_rank(pk_n, s, seed, i);
    keys[i] = base + (int32_t)dg_perm_apply(&p, r - 1);
  }
}

/* Uniform 64-bit keys (the partition-only workload): keys[i] = mix(seed, i). */
void dg_uniform_u64_keys(int64_t *keys, uint64_t n, uint64_t seed) {
  for (uint64_t i = 0; i < n; ++i)
    keys[i] = (int64_t)dg_mix64(seed ^ dg_mix64(i + 0x1234567ull));
}

/* Join selectivity (datagen/src/relation.rs:85-151): a key k stays when a
 * draw from 0..100, a function of (seed, k - base), is at most selectivity;
 * otherwise it becomes the null key (all ones).  Null keys stay null. */
static inline int dg_keep_key(uint64_t seed, uint64_t off, uint32_t selectivity) {
  return dg_mix64(seed ^ dg_mix64(off + 0x6E756C6Cull)) % 101u <= selectivity;
}
void dg_null_keys_i64(int64_t *keys, uint64_t n, uint32_t selectivity,
                      uint64_t seed, int64_t base) {
  if (selectivity >= 100) return;
  for (uint64_t i = 0; i < n; ++i)
    if (keys[i] != -1 && !dg_keep_key(seed, (uint64_t)(keys[i] - base), selectivity))
      keys[i] = -1;
}
void dg_null_keys_i32(int32_t *keys, uint64_t n, uint32_t selectivity,
                      uint64_t seed, int32_t base) {
  if (selectivity >= 100) return;
  for (uint64_t i = 0; i < n; ++i)
    if (keys[i] != -1 &&
        !dg_keep_key(seed, (uint64_t)((int64_t)keys[i] - (int64_t)base), selectivity))
      keys[i] = -1;
}
