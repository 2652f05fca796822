/*
 * Multi-threaded CPU radix join: the reported CPU baseline.  TEST
 * INFRASTRUCTURE ONLY (bench.py's CPU-baseline leg and tests).
 *
 * It follows the reference's two-pass radix-join pipeline
 * (radix-join/src/execution_methods/gpu_radix_join.rs:90-565) on host cores:
 *   pass 1: per chunk, one chunk per thread, the reference's own compiled
 *           `cpu_chunked_prefix_sum_int64` and
 *           `cpu_chunked_radix_partition_swwc_int64_int64`
 *           (sql-ops/cpputils/radix_partition.cpp:228-267, 491-557), loaded
 *           with dlopen from oracle/_ref/libref_cpu.so; the threading follows
 *           radix-join/src/execution_methods/cpu_partitioned_radix_join.rs:
 *           259-287,458-474.  Without that library the oracle restatement of
 *           the same operators is used.
 *   pass 2 + join: per first-pass partition (threads take partitions from a
 *           shared counter): gather the partition from all chunks, partition
 *           it by the second-pass bits and join every sub-partition with the
 *           bucket-chaining scheme of sql-ops/cudautils/radix_join.cu:199-311
 *           (the reference runs these two steps on the GPU only, so on the
 *           CPU they are the oracle restatement).
 * Timing uses CLOCK_MONOTONIC like the reference harness
 * (guides/benchmarking.md:61-62).
 */
#define _GNU_SOURCE
#include <dlfcn.h>
#include <pthread.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#include <time.h>

typedef struct {
  int64_t key, value;
} cb_tuple;

/* Argument structs of the reference CPU operators,
 * sql-ops/cpputils/radix_partition.cpp:91-124. */
typedef struct {
  const void *partition_attr;
  size_t data_length;
  size_t canonical_chunk_length;
  uint32_t padding_length;
  uint32_t radix_bits;
  uint32_t ignore_bits;
  unsigned int *tmp_partition_offsets;
  unsigned long long *partition_offsets;
} cb_prefix_sum_args;

typedef struct {
  const void *join_attr_data;
  const void *payload_attr_data;
  size_t data_length;
  size_t padding_length;
  uint32_t radix_bits;
  uint32_t ignore_bits;
  const unsigned long long *partition_offsets;
  unsigned long long *tmp_partition_offsets;
  void *write_combine_buffer;
  void *partitioned_relation;
} cb_partition_args;

typedef void (*cb_prefix_fn)(cb_prefix_sum_args *, uint32_t, uint32_t);
typedef void (*cb_partition_fn)(cb_partition_args *);
typedef size_t (*cb_swwc_bytes_fn)(void);

/* From oracle.c */
uint64_t or_input_chunk_size(uint64_t, uint32_t, uint32_t);
void or_chunked_prefix_sum_i64(const int64_t *, uint64_t, uint32_t, uint32_t,
                               uint32_t, uint32_t, uint64_t *);
void or_chunked_radix_partition_i64(const int64_t *, const int64_t *, uint64_t,
                                    const uint64_t *, uint32_t, uint32_t,
                                    uint32_t, void *);

static double cb_now(void) {
  struct timespec ts;
  clock_gettime(CLOCK_MONOTONIC, &ts);
  return (double)ts.tv_sec + 1e-9 * (double)ts.tv_nsec;
}

typedef struct {
  /* shared */
  const int64_t *key, *pay;
  uint64_t len;
  uint32_t chunks, bits1;
  uint64_t clen;
  uint64_t *offsets; /* chunks * F1 */
  cb_tuple *out;
  cb_prefix_fn prefix;
  cb_partition_fn partition;
  size_t swwc_bytes;
  /* per thread */
  uint32_t chunk;
} cb_pass1_job;

static void *cb_pass1_prefix(void *arg) {
  cb_pass1_job *j = (cb_pass1_job *)arg;
  uint64_t F = 1ull << j->bits1;
  uint64_t begin = j->clen * j->chunk;
  uint64_t end = (j->chunk + 1 == j->chunks) ? j->len : begin + j->clen;
  unsigned int *tmp = (unsigned int *)malloc(F * sizeof(unsigned int));
  cb_prefix_sum_args a = {j->key + begin, end - begin, j->clen, 8u,
                          j->bits1,       0u,          tmp,
                          (unsigned long long *)(j->offsets + j->chunk * F)};
  j->prefix(&a, j->chunk, j->chunks);
  free(tmp);
  return NULL;
}

static void *cb_pass1_partition(void *arg) {
  cb_pass1_job *j = (cb_pass1_job *)arg;
  uint64_t F = 1ull << j->bits1;
  uint64_t begin = j->clen * j->chunk;
  uint64_t end = (j->chunk + 1 == j->chunks) ? j->len : begin + j->clen;
  const uint64_t *off = j->offsets + j->chunk * F;
  uint64_t base = off[0] - 8u; /* chunk start, radix_partition.cpp:424-425 */
  void *wc = NULL;
  if (posix_memalign(&wc, 64, F * j->swwc_bytes) != 0) return NULL;
  unsigned long long *tmp =
      (unsigned long long *)malloc(F * sizeof(unsigned long long));
  cb_partition_args a = {j->key + begin, j->pay + begin, end - begin, 8u,
                         j->bits1, 0u, (const unsigned long long *)off, tmp,
                         wc, j->out + base};
  j->partition(&a);
  free(tmp);
  free(wc);
  return NULL;
}

typedef struct {
  const cb_tuple *rel1[2]; /* pass-1 output of R and S */
  const uint64_t *off1[2];
  uint64_t padded1[2];
  uint32_t chunks, bits1, bits2;
  volatile uint32_t next; /* work counter */
  pthread_mutex_t lock;
  uint64_t sum, count;
} cb_pass2_shared;

static uint32_t cb_hash(uint64_t v) {
  return (uint32_t)((v * 11400714819323198485ull) >> (64u - 11u));
}

static void *cb_pass2_worker(void *arg) {
  cb_pass2_shared *sh = (cb_pass2_shared *)arg;
  const uint64_t F1 = 1ull << sh->bits1, F2 = 1ull << sh->bits2;
  const uint32_t ign2 = sh->bits1, ign_join = sh->bits1 + sh->bits2;
  const uint64_t mask2 = (F2 - 1) << ign2;
  uint64_t cap[2] = {0, 0};
  cb_tuple *gath[2] = {NULL, NULL}, *part[2] = {NULL, NULL};
  uint64_t *hist[2], *cur = (uint64_t *)malloc(F2 * sizeof(uint64_t));
  hist[0] = (uint64_t *)malloc((F2 + 1) * sizeof(uint64_t));
  hist[1] = (uint64_t *)malloc((F2 + 1) * sizeof(uint64_t));
  uint32_t heads[2048];
  uint32_t *links = NULL;
  uint64_t links_cap = 0;
  uint64_t sum = 0, count = 0;
  for (;;) {
    uint32_t p1 = __sync_fetch_and_add(&sh->next, 1u);
    if (p1 >= F1) break;
    uint64_t n[2];
    for (int r = 0; r < 2; ++r) {
      /* gather partition p1 of every chunk, radix_partition.cu:343-410 */
      n[r] = 0;
      for (uint32_t c = 0; c < sh->chunks; ++c) {
        uint64_t b = sh->off1[r][c * F1 + p1];
        uint64_t e = (c + 1 == sh->chunks && p1 + 1 == F1)
                         ? sh->padded1[r]
                         : sh->off1[r][c * F1 + p1 + 1] - 8u;
        n[r] += e - b;
      }
      if (n[r] > cap[r]) {
        cap[r] = n[r];
        gath[r] = (cb_tuple *)realloc(gath[r], cap[r] * sizeof(cb_tuple));
        part[r] = (cb_tuple *)realloc(part[r], cap[r] * sizeof(cb_tuple));
      }
      uint64_t k = 0;
      for (uint32_t c = 0; c < sh->chunks; ++c) {
        uint64_t b = sh->off1[r][c * F1 + p1];
        uint64_t e = (c + 1 == sh->chunks && p1 + 1 == F1)
                         ? sh->padded1[r]
                         : sh->off1[r][c * F1 + p1 + 1] - 8u;
        memcpy(gath[r] + k, sh->rel1[r] + b, (e - b) * sizeof(cb_tuple));
        k += e - b;
      }
      /* second-pass histogram + scatter (no padding needed in a private
       * buffer; partition boundaries kept in hist[r]) */
      memset(hist[r], 0, (F2 + 1) * sizeof(uint64_t));
      for (uint64_t i = 0; i < n[r]; ++i)
        hist[r][((uint64_t)gath[r][i].key & mask2) >> ign2]++;
      uint64_t run = 0;
      for (uint64_t q = 0; q < F2; ++q) {
        uint64_t v = hist[r][q];
        hist[r][q] = run;
        cur[q] = run;
        run += v;
      }
      hist[r][F2] = run;
      for (uint64_t i = 0; i < n[r]; ++i)
        part[r][cur[((uint64_t)gath[r][i].key & mask2) >> ign2]++] = gath[r][i];
    }
    /* bucket-chaining join per sub-partition, radix_join.cu:199-311 */
    for (uint64_t q = 0; q < F2; ++q) {
      uint64_t bb = hist[0][q], be = hist[0][q + 1];
      uint64_t pb = hist[1][q], pe = hist[1][q + 1];
      if (be - bb > links_cap) {
        links_cap = be - bb;
        links = (uint32_t *)realloc(links, links_cap * sizeof(uint32_t));
      }
      for (int h = 0; h < 2048; ++h) heads[h] = UINT32_MAX;
      for (uint64_t i = 0; i < be - bb; ++i) {
        uint32_t h = cb_hash((uint64_t)part[0][bb + i].key >> ign_join);
        links[i] = heads[h];
        heads[h] = (uint32_t)i;
      }
      for (uint64_t j = pb; j < pe; ++j) {
        int64_t key = part[1][j].key;
        uint32_t h = cb_hash((uint64_t)key >> ign_join);
        for (uint32_t e = heads[h]; e != UINT32_MAX; e = links[e])
          if (part[0][bb + e].key == key) {
            sum += (uint64_t)part[1][j].value;
            count += 1;
          }
      }
    }
  }
  pthread_mutex_lock(&sh->lock);
  sh->sum += sum;
  sh->count += count;
  pthread_mutex_unlock(&sh->lock);
  for (int r = 0; r < 2; ++r) {
    free(gath[r]);
    free(part[r]);
    free(hist[r]);
  }
  free(cur);
  free(links);
  return NULL;
}

/* Runs the whole join.  ref_lib_path: the compiled reference CPU library or
 * NULL for the restatement.  times[0..2] = prefix-sum, partition, pass-2+join
 * seconds.  Returns 0 on success, negative when the reference library cannot
 * be loaded. */
int cb_cpu_radix_join_i64(const int64_t *r_key, const int64_t *r_pay,
                          uint64_t r_len, const int64_t *s_key,
                          const int64_t *s_pay, uint64_t s_len, uint32_t bits1,
                          uint32_t bits2, uint32_t threads,
                          const char *ref_lib_path, int64_t *sum_out,
                          uint64_t *count_out, double *times) {
  cb_prefix_fn prefix = NULL;
  cb_partition_fn partition = NULL;
  size_t swwc_bytes = 64;
  void *lib = NULL;
  if (ref_lib_path) {
    lib = dlopen(ref_lib_path, RTLD_NOW | RTLD_LOCAL);
    if (!lib) return -1;
    prefix = (cb_prefix_fn)dlsym(lib, "cpu_chunked_prefix_sum_int64");
    partition =
        (cb_partition_fn)dlsym(lib, "cpu_chunked_radix_partition_swwc_int64_int64");
    cb_swwc_bytes_fn wcb = (cb_swwc_bytes_fn)dlsym(lib, "cpu_swwc_buffer_bytes");
    if (!prefix || !partition || !wcb) return -2;
    swwc_bytes = wcb();
  }
  const uint64_t F1 = 1ull << bits1;
  const int64_t *keys[2] = {r_key, s_key}, *pays[2] = {r_pay, s_pay};
  uint64_t lens[2] = {r_len, s_len};
  uint64_t *offs[2];
  cb_tuple *rel[2];
  uint64_t padded[2];
  for (int r = 0; r < 2; ++r) {
    offs[r] = (uint64_t *)malloc(threads * F1 * sizeof(uint64_t));
    padded[r] = lens[r] + threads * F1 * 8u;
    rel[r] = NULL;
    if (posix_memalign((void **)&rel[r], 128, padded[r] * sizeof(cb_tuple)))
      return -3;
    memset(rel[r], 0xff, padded[r] * sizeof(cb_tuple));
  }
  pthread_t *tids = (pthread_t *)malloc(threads * sizeof(pthread_t));
  cb_pass1_job *jobs = (cb_pass1_job *)malloc(2 * threads * sizeof(cb_pass1_job));
  for (int r = 0; r < 2; ++r)
    for (uint32_t t = 0; t < threads; ++t) {
      cb_pass1_job *j = &jobs[r * threads + t];
      j->key = keys[r];
      j->pay = pays[r];
      j->len = lens[r];
      j->chunks = threads;
      j->bits1 = bits1;
      j->clen = or_input_chunk_size(lens[r], threads, 8);
      j->offsets = offs[r];
      j->out = rel[r];
      j->prefix = prefix;
      j->partition = partition;
      j->swwc_bytes = swwc_bytes;
      j->chunk = t;
    }

  double t0 = cb_now();
  for (int r = 0; r < 2; ++r) {
    if (prefix) {
      for (uint32_t t = 0; t < threads; ++t)
        pthread_create(&tids[t], NULL, cb_pass1_prefix, &jobs[r * threads + t]);
      for (uint32_t t = 0; t < threads; ++t) pthread_join(tids[t], NULL);
    } else {
      or_chunked_prefix_sum_i64(keys[r], lens[r], threads, bits1, 0, 8u, offs[r]);
    }
  }
  double t1 = cb_now();
  for (int r = 0; r < 2; ++r) {
    if (partition) {
      for (uint32_t t = 0; t < threads; ++t)
        pthread_create(&tids[t], NULL, cb_pass1_partition, &jobs[r * threads + t]);
      for (uint32_t t = 0; t < threads; ++t) pthread_join(tids[t], NULL);
    } else {
      or_chunked_radix_partition_i64(keys[r], pays[r], lens[r], offs[r],
                                     threads, bits1, 0, rel[r]);
    }
  }
  double t2 = cb_now();
  cb_pass2_shared sh;
  memset(&sh, 0, sizeof(sh));
  for (int r = 0; r < 2; ++r) {
    sh.rel1[r] = rel[r];
    sh.off1[r] = offs[r];
    sh.padded1[r] = padded[r];
  }
  sh.chunks = threads;
  sh.bits1 = bits1;
  sh.bits2 = bits2;
  pthread_mutex_init(&sh.lock, NULL);
  for (uint32_t t = 0; t < threads; ++t)
    pthread_create(&tids[t], NULL, cb_pass2_worker, &sh);
  for (uint32_t t = 0; t < threads; ++t) pthread_join(tids[t], NULL);
  double t3 = cb_now();
  pthread_mutex_destroy(&sh.lock);

  if (times) {
    times[0] = t1 - t0;
    times[1] = t2 - t1;
    times[2] = t3 - t2;
  }
  *sum_out = (int64_t)sh.sum;
  *count_out = sh.count;
  for (int r = 0; r < 2; ++r) {
    free(offs[r]);
    free(rel[r]);
  }
  free(tids);
  free(jobs);
  if (lib) dlclose(lib);
  return 0;
}
