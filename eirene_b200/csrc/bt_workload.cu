// Seeded synthetic workload generators on the device (benchmark inputs only;
// not part of the tree path).  They stand in for the reference's missing
// dataset files (input_data_{23..26}.txt, {size}_{dist}/query_95_50M.txt).
// Counter-based: element i depends only on (seed, i), so any slice can be
// regenerated.  The uniform generator is integer-only and bit-identical to the
// CPU generator in the tests; the Zipf / normal / gamma generators use
// double-precision math, whose last bit can differ from a CPU libm's: such a
// key then differs by a few units in its 40th bit (Zipf tree keys are hashed
// ranks, integer only).
#include <cuda_runtime.h>

#include "../../include/eirene_b200.h"
#include "bt_common.cuh"

namespace bt {
namespace {

__device__ __forceinline__ uint64_t mix64(uint64_t z) {  // SplitMix64 output function
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  return z ^ (z >> 31);
}
__device__ __forceinline__ uint64_t rnd(uint64_t seed, uint64_t i, uint64_t j) {
  return mix64(mix64(seed) + 0x9E3779B97F4A7C15ull * (i * 16 + j + 1));
}
__device__ __forceinline__ double unit_open(uint64_t r) { return ((double)(r >> 11) + 1.0) * (1.0 / 9007199254740992.0); }

// Zipf(s) over 1..N by rejection-inversion (Hormann & Derflinger 1996)
struct Zipf {
  double s, n, hx1, hn, sq;
};
__device__ double zh(const Zipf& z, double x) { return exp(-z.s * log(x)); }
__device__ double zhint(const Zipf& z, double x) {
  const double lx = log(x), t = (1.0 - z.s) * lx;
  const double f = fabs(t) > 1e-8 ? expm1(t) / t : 1.0 + t * 0.5 * (1.0 + t / 3.0);
  return f * lx;
}
__device__ double zhinv(const Zipf& z, double x) {
  double t = x * (1.0 - z.s);
  if (t < -1.0) t = -1.0;
  const double f = fabs(t) > 1e-8 ? log1p(t) / t : 1.0 - t * (0.5 - t / 3.0);
  return exp(f * x);
}
__device__ Zipf zipf_make(double s, double n) {
  Zipf z;
  z.s = s;
  z.n = n;
  z.hx1 = zhint(z, 1.5) - 1.0;
  z.hn = zhint(z, n + 0.5);
  z.sq = 2.0 - zhinv(z, zhint(z, 2.5) - zh(z, 2.0));
  return z;
}
__device__ uint64_t zipf_draw(const Zipf& z, uint64_t seed, uint64_t i, uint64_t j0) {
  for (uint64_t a = 0; a < 64; a++) {
    const double u = z.hn + unit_open(rnd(seed, i, j0 + a)) * (z.hx1 - z.hn);
    const double x = zhinv(z, u);
    double k = floor(x + 0.5);
    if (k < 1) k = 1;
    if (k > z.n) k = z.n;
    if (k - x <= z.sq || u >= zhint(z, k + 0.5) - zh(z, k)) return (uint64_t)k;
  }
  return 1;
}
__device__ __forceinline__ uint64_t rank_key(uint64_t rank) { return mix64(rank ^ 0x2545F4914F6CDD1Dull) >> 1; }
__device__ uint64_t clamp_key(double v) {
  if (!(v >= 0)) return 0;
  if (v >= 18446744073709549568.0) return 0xFFFFFFFFFFFFF7FFull;
  return (uint64_t)llrint(v);
}
__device__ uint64_t draw_key(int dist, const Zipf& z, uint64_t seed, uint64_t i, uint64_t j0) {
  switch (dist) {
    case 1: return rank_key(zipf_draw(z, seed, i, j0));
    case 2: {
      const double u1 = unit_open(rnd(seed, i, j0)), u2 = unit_open(rnd(seed, i, j0 + 1));
      const double g = sqrt(-2.0 * log(u1)) * cos(6.283185307179586 * u2);
      return clamp_key(4611686018427387904.0 + 288230376151711744.0 * g);
    }
    case 3: {
      const double u1 = unit_open(rnd(seed, i, j0)), u2 = unit_open(rnd(seed, i, j0 + 1));
      return clamp_key(72057594037927936.0 * (-log(u1) - log(u2)));
    }
    default: return rnd(seed, i, j0) >> 1;
  }
}

__global__ void gen_keys_kernel(int dist, uint64_t seed, size_t n, uint64_t* keys, uint64_t* vals) {
  const Zipf z = zipf_make(0.99, 4294967296.0);
  const size_t stride = (size_t)gridDim.x * blockDim.x;
  for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) {
    const uint64_t k = dist == 1 ? rank_key(i + 1) : draw_key(dist, z, seed, i, 0);
    keys[i] = k;
    if (vals) vals[i] = k ^ 0x9E3779B97F4A7C15ull;
  }
}

__global__ void gen_requests_kernel(int dist, uint64_t seed, const uint64_t* tree_keys, size_t n_tree, size_t n,
                                    uint32_t search_pct, uint64_t* keys, uint64_t* vals, uint8_t* ops) {
  const Zipf z = zipf_make(0.99, 4294967296.0);
  const size_t stride = (size_t)gridDim.x * blockDim.x;
  for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) {
    const uint64_t r0 = rnd(seed, i, 0);
    if (r0 % 100 < search_pct) {
      ops[i] = kOpGet;
      vals[i] = 0;
      const uint64_t r1 = rnd(seed, i, 1);
      if ((r1 & 1) && n_tree > 0) keys[i] = tree_keys[(r1 >> 1) % n_tree];
      else keys[i] = draw_key(dist, z, seed, i, 2);
    } else {
      ops[i] = kOpInsert;
      const uint64_t k = draw_key(dist, z, seed ^ 0x5851F42D4C957F2Dull, i, 2);
      keys[i] = k;
      vals[i] = k ^ 0x9E3779B97F4A7C15ull;
    }
  }
}

// Requests shaped like a sample of the caller's keys, whatever law they
// follow: GETs of sample keys (half) or of a sample key with its low 40 bits
// redrawn, INSERTs of a sample key with its low 40 bits redrawn (fresh keys
// where the sample is dense; a 2^22-key sample of 64-bit keys is about 2^42
// apart on average).  The node-fill tuner times its trial batches on these.
__global__ void gen_sample_requests_kernel(uint64_t seed, const uint64_t* sample, size_t n_sample, size_t n,
                                           uint32_t search_pct, uint64_t* keys, uint64_t* vals, uint8_t* ops) {
  constexpr uint64_t kLow = (1ull << 40) - 1;
  const size_t stride = (size_t)gridDim.x * blockDim.x;
  for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) {
    const uint64_t r0 = rnd(seed, i, 0), r1 = rnd(seed, i, 1), r2 = rnd(seed, i, 2);
    const uint64_t base = sample[(r1 >> 1) % n_sample];
    uint64_t near = (base & ~kLow) | (r2 & kLow);
    if (near == kKeyMax) near ^= 1;
    if (r0 % 100 < search_pct) {
      ops[i] = kOpGet;
      vals[i] = 0;
      keys[i] = (r1 & 1) ? base : near;
    } else {
      ops[i] = kOpInsert;
      keys[i] = near;
      vals[i] = near ^ 0x9E3779B97F4A7C15ull;
    }
  }
}

}  // namespace

cudaError_t gen_sample_requests(uint64_t seed, const uint64_t* sample, size_t n_sample, size_t n, uint32_t search_pct,
                                uint64_t* keys, uint64_t* vals, uint8_t* ops, cudaStream_t s) {
  if (n == 0 || n_sample == 0) return cudaSuccess;
  gen_sample_requests_kernel<<<1184, 256, 0, s>>>(seed, sample, n_sample, n, search_pct, keys, vals, ops);
  return cudaGetLastError();
}
}  // namespace bt

extern "C" {

/* Benchmark input generators (see include/eirene_b200.h). */
int bt_gen_keys(int dist, uint64_t seed, size_t n, uint64_t* keys, uint64_t* vals, void* stream) {
  if (n == 0) return BT_OK;
  if (!keys || dist < 0 || dist > 3) return BT_ERR_INVALID_ARG;
  bt::gen_keys_kernel<<<1184, 256, 0, (cudaStream_t)stream>>>(dist, seed, n, keys, vals);
  return cudaGetLastError() == cudaSuccess ? BT_OK : BT_ERR_CUDA;
}

int bt_gen_requests(int dist, uint64_t seed, const uint64_t* tree_keys, size_t n_tree, size_t n, uint32_t search_pct,
                    uint64_t* keys, uint64_t* vals, uint8_t* ops, void* stream) {
  if (n == 0) return BT_OK;
  if (!keys || !vals || !ops || dist < 0 || dist > 3 || search_pct > 100 || (n_tree && !tree_keys))
    return BT_ERR_INVALID_ARG;
  bt::gen_requests_kernel<<<1184, 256, 0, (cudaStream_t)stream>>>(dist, seed, tree_keys, n_tree, n, search_pct, keys,
                                                                   vals, ops);
  return cudaGetLastError() == cudaSuccess ? BT_OK : BT_ERR_CUDA;
}

}  // extern "C"
