// Seeded relation generator on the GPU (counterpart of the reference's
// datagen crate, datagen/src/relation.rs, which uses unseeded thread_rng).
//
// Same integer arithmetic as the CPU generator that the tests use, so the
// permutation and the uniform foreign keys are bit-identical on both sides:
//  * SplitMix64 finaliser (Steele, Lea, Flood 2014) as the mixing function;
//  * a 4-round balanced Feistel network over 2^(2h) >= N with cycle walking
//    (Black & Rogaway 2002) as the seeded bijection on [0, N);
//  * Zipf ranks by rejection-inversion (Hoermann & Derflinger 1996) in double
//    precision (CPU and GPU results may differ in rare last-ulp cases).
#include <math.h>

#include "common.cuh"
#include "kernels.h"

namespace fi {

__host__ __device__ __forceinline__ uint64_t dg_mix64(uint64_t x) {
  uint64_t z = x + 0x9E3779B97F4A7C15ull;
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  return z ^ (z >> 31);
}

struct Perm {
  uint64_t n;
  uint32_t half_bits;
  uint64_t half_mask;
  uint64_t rk[4];
};

static Perm make_perm(uint64_t n, uint64_t seed) {
  Perm p;
  uint32_t bits = 0;
  while (bits < 64 && (1ull << bits) < n) bits++;
  uint32_t h = (bits + 1) / 2;
  if (h == 0) h = 1;
  p.n = n;
  p.half_bits = h;
  p.half_mask = (1ull << h) - 1ull;
  for (int r = 0; r < 4; ++r) p.rk[r] = dg_mix64(seed * 4ull + (uint64_t)r + 0x5151ull);
  return p;
}

__device__ __forceinline__ uint64_t perm_apply(const Perm &p, uint64_t x) {
  do {
    uint64_t l = x >> p.half_bits, r = x & p.half_mask;
#pragma unroll
    for (int k = 0; k < 4; ++k) {
      uint64_t t = r;
      r = l ^ (dg_mix64(r ^ p.rk[k]) & p.half_mask);
      l = t;
    }
    x = (l << p.half_bits) | r;
  } while (x >= p.n);
  return x;
}

__device__ __forceinline__ double dg_helper1(double x) {
  return fabs(x) > 1e-8 ? log1p(x) / x : 1.0 - x * (0.5 - x * (1.0 / 3.0));
}
__device__ __forceinline__ double dg_helper2(double x) {
  return fabs(x) > 1e-8 ? expm1(x) / x : 1.0 + x * 0.5 * (1.0 + x / 3.0);
}
__device__ __forceinline__ double dg_h_int(double x, double s) {
  double lx = log(x);
  return dg_helper2((1.0 - s) * lx) * lx;
}
__device__ __forceinline__ double dg_h(double x, double s) { return exp(-s * log(x)); }
__device__ __forceinline__ double dg_h_int_inv(double x, double s) {
  double t = x * (1.0 - s);
  if (t < -1.0) t = -1.0;
  return exp(dg_helper1(t) * x);
}

// Constants of the rejection-inversion sampler for (n, s); computed once per
// thread, outside the per-key loop.
struct ZipfConst {
  double hx1, hn, sq;
};
__device__ ZipfConst zipf_const(uint64_t n, double s) {
  ZipfConst z;
  z.hx1 = dg_h_int(1.5, s) - 1.0;
  z.hn = dg_h_int((double)n + 0.5, s);
  z.sq = 2.0 - dg_h_int_inv(dg_h_int(2.5, s) - dg_h(2.0, s), s);
  return z;
}

__device__ uint64_t zipf_rank(uint64_t n, double s, const ZipfConst &z,
                              uint64_t seed, uint64_t i) {
  const double hx1 = z.hx1, hn = z.hn, sq = z.sq;
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

template <typename K>
__global__ void gen_pk_kernel(K *keys, uint64_t n, Perm p, K base) {
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n;
       i += (uint64_t)gridDim.x * blockDim.x)
    keys[i] = base + (K)perm_apply(p, i);
}

template <typename K>
__global__ void gen_uniform_fk_kernel(K *keys, uint64_t n, uint64_t pk_n,
                                      uint64_t seed, K base) {
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n;
       i += (uint64_t)gridDim.x * blockDim.x)
    keys[i] = base + (K)__umul64hi(dg_mix64(seed ^ dg_mix64(i)), pk_n);
}

template <typename K>
__global__ void gen_zipf_fk_kernel(K *keys, uint64_t n, uint64_t pk_n, double s,
                                   uint64_t seed, Perm p, K base) {
  const ZipfConst z = zipf_const(pk_n, s);
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n;
       i += (uint64_t)gridDim.x * blockDim.x)
    keys[i] = base + (K)perm_apply(p, zipf_rank(pk_n, s, z, seed, i) - 1);
}

__global__ void gen_u64_kernel(int64_t *keys, uint64_t n, uint64_t seed) {
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n;
       i += (uint64_t)gridDim.x * blockDim.x)
    keys[i] = (int64_t)dg_mix64(seed ^ dg_mix64(i + 0x1234567ull));
}

// Join selectivity (datagen/src/relation.rs:85-151): the reference keeps a
// primary key when a uniform draw from 0..=100 is at most `selectivity` and
// otherwise stores the null key.  Here the draw is a function of (seed,
// key - base), so a caller can recompute from a key alone whether it stayed.
__host__ __device__ __forceinline__ bool dg_keep_key(uint64_t seed, uint64_t off,
                                                     uint32_t selectivity) {
  return dg_mix64(seed ^ dg_mix64(off + 0x6E756C6Cull)) % 101u <= selectivity;
}

template <typename K>
__global__ void null_keys_kernel(K *keys, uint64_t n, uint32_t selectivity,
                                 uint64_t seed, K base) {
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n;
       i += (uint64_t)gridDim.x * blockDim.x) {
    const K k = keys[i];
    if (k == null_key<K>()) continue;
    const uint64_t off = (uint64_t)((int64_t)k - (int64_t)base);
    if (!dg_keep_key(seed, off, selectivity)) keys[i] = null_key<K>();
  }
}

static uint32_t gen_grid(uint64_t n) {
  uint64_t g = (n + 255) / 256;
  return (uint32_t)(g < 148u * 64u ? (g == 0 ? 1 : g) : 148u * 64u);
}

template <typename K>
cudaError_t launch_gen_primary_keys(K *keys, uint64_t n, uint64_t seed, K base,
                                    cudaStream_t stream) {
  if (n == 0) return cudaSuccess;
  gen_pk_kernel<K><<<gen_grid(n), 256, 0, stream>>>(keys, n, make_perm(n, seed),
                                                    base);
  return cudaGetLastError();
}

template <typename K>
cudaError_t launch_gen_uniform_fk(K *keys, uint64_t n, uint64_t pk_n,
                                  uint64_t seed, K base, cudaStream_t stream) {
  if (n == 0) return cudaSuccess;
  gen_uniform_fk_kernel<K><<<gen_grid(n), 256, 0, stream>>>(keys, n, pk_n, seed,
                                                            base);
  return cudaGetLastError();
}

template <typename K>
cudaError_t launch_gen_zipf_fk(K *keys, uint64_t n, uint64_t pk_n, double s,
                               uint64_t seed, uint64_t pk_seed, K base,
                               cudaStream_t stream) {
  if (n == 0) return cudaSuccess;
  gen_zipf_fk_kernel<K><<<gen_grid(n), 256, 0, stream>>>(
      keys, n, pk_n, s, seed, make_perm(pk_n, pk_seed), base);
  return cudaGetLastError();
}

template <typename K>
cudaError_t launch_null_keys(K *keys, uint64_t n, uint32_t selectivity,
                             uint64_t seed, K base, cudaStream_t stream) {
  if (n == 0 || selectivity >= 100) return cudaSuccess;
  null_keys_kernel<K><<<gen_grid(n), 256, 0, stream>>>(keys, n, selectivity, seed,
                                                       base);
  return cudaGetLastError();
}
template cudaError_t launch_null_keys<int32_t>(int32_t *, uint64_t, uint32_t,
                                               uint64_t, int32_t, cudaStream_t);
template cudaError_t launch_null_keys<int64_t>(int64_t *, uint64_t, uint32_t,
                                               uint64_t, int64_t, cudaStream_t);

cudaError_t launch_gen_uniform_u64(int64_t *keys, uint64_t n, uint64_t seed,
                                   cudaStream_t stream) {
  if (n == 0) return cudaSuccess;
  gen_u64_kernel<<<gen_grid(n), 256, 0, stream>>>(keys, n, seed);
  return cudaGetLastError();
}

template cudaError_t launch_gen_primary_keys<int32_t>(int32_t *, uint64_t,
                                                      uint64_t, int32_t,
                                                      cudaStream_t);
template cudaError_t launch_gen_primary_keys<int64_t>(int64_t *, uint64_t,
                                                      uint64_t, int64_t,
                                                      cudaStream_t);
template cudaError_t launch_gen_uniform_fk<int32_t>(int32_t *, uint64_t,
                                                    uint64_t, uint64_t, int32_t,
                                                    cudaStream_t);
template cudaError_t launch_gen_uniform_fk<int64_t>(int64_t *, uint64_t,
                                                    uint64_t, uint64_t, int64_t,
                                                    cudaStream_t);
template cudaError_t launch_gen_zipf_fk<int32_t>(int32_t *, uint64_t, uint64_t,
                                                 double, uint64_t, uint64_t,
                                                 int32_t, cudaStream_t);
template cudaError_t launch_gen_zipf_fk<int64_t>(int64_t *, uint64_t, uint64_t,
                                                 double, uint64_t, uint64_t,
                                                 int64_t, cudaStream_t);

}  // namespace fi
