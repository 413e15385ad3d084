// Hand-written stable LSD radix sort of (uint64 key, uint32 payload) pairs and
// a device-wide exclusive scan.  They replace the reference's CUB calls
// DeviceRadixSort::SortPairs, DeviceRunLengthEncode::Encode and
// DeviceScan::ExclusiveSum (src/gpu-stm-tree-v38/bpt-gpustm-kernel.cu:289-324).
//
// The sort follows the single-pass-per-digit scheme of Adinets & Merrill,
// "Onesweep: A Faster Least Significant Digit Radix Sort for GPUs" (2022):
//   1. one up-front kernel counts all eight 8-bit digits of every key;
//   2. per digit, one kernel: a tile of T x 8 items (T threads: 2048, 4096 or
//      8192 items; bt_autotune picks T) takes a dynamic tile id,
//      ranks its items stably with eight bit ballots per item (each warp owns a
//      contiguous 256-item chunk and walks it in 8 rounds), publishes its
//      per-digit counts, and finds its global offsets by decoupled look-back
//      over the preceding tiles; it then stages the tile in shared memory in
//      digit order and writes each digit run contiguously (coalesced).
// The look-back spins on words other tiles write; every spin is bounded and a
// timeout sets kErrSpin in the tree's error word instead of hanging.
#include <cstdint>
#include <cuda_runtime.h>

#include "bt_common.cuh"
#include "bt_internal.h"

namespace bt {

namespace {

constexpr int kSortThreads = 512;                  // the histogram kernel's block
constexpr int kSortItems = 8;                      // items per thread in a tile
constexpr int kMinTile = 256 * kSortItems;         // the smallest tile (T = 256)
constexpr int kRadix = 256;

constexpr int kScanThreads = 1024;
constexpr int kScanItems = 4;
constexpr int kScanTile = kScanThreads * kScanItems;  // 4096

__device__ __forceinline__ uint32_t digit_of(uint64_t k, int shift) { return (uint32_t)(k >> shift) & 0xff; }
// 2-bit op code carried in the payload: 0 insert, 1 get, 2 delete, 3 anything else (rejected)
__device__ __forceinline__ uint32_t op_code(uint8_t op) { return op <= 2 ? (uint32_t)op : 3u; }

// ---------------------------------------------------------------- scan ----
// block-wide exclusive scan of one value per thread (1024 threads)
__device__ __forceinline__ uint32_t block_exclusive_scan(uint32_t v, uint32_t* warp_sums, uint32_t* total) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  uint32_t x = v;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    uint32_t y = __shfl_up_sync(0xffffffffu, x, o);
    if (lane >= o) x += y;
  }
  if (lane == 31) warp_sums[warp] = x;
  __syncthreads();
  if (warp == 0) {
    const int nw = blockDim.x >> 5;
    uint32_t s = lane < nw ? warp_sums[lane] : 0;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      uint32_t y = __shfl_up_sync(0xffffffffu, s, o);
      if (lane >= o) s += y;
    }
    if (lane < nw) warp_sums[lane] = s;  // inclusive
    if (lane == nw - 1 && total) *total = s;
  }
  __syncthreads();
  uint32_t base = warp ? warp_sums[warp - 1] : 0;
  uint32_t r = base + x - v;
  __syncthreads();
  return r;
}

__global__ void __launch_bounds__(kScanThreads) scan_reduce_kernel(const uint32_t* in, size_t n,
                                                                   const uint32_t* n_dev, uint32_t* sums) {
  __shared__ uint32_t ws[32];
  __shared__ uint32_t tot;
  if (n_dev) n = min(n, (size_t)*n_dev);
  size_t base = (size_t)blockIdx.x * kScanTile + (size_t)threadIdx.x * kScanItems;
  uint32_t s = 0;
#pragma unroll
  for (int i = 0; i < kScanItems; i++)
    if (base + i < n) s += in[base + i];
  block_exclusive_scan(s, ws, &tot);
  if (threadIdx.x == 0) sums[blockIdx.x] = tot;
}

// single block; scans `n` values in place (exclusive); writes the grand total
__global__ void __launch_bounds__(kScanThreads) scan_single_kernel(uint32_t* data, size_t n, uint32_t* total_out) {
  __shared__ uint32_t ws[32];
  __shared__ uint32_t tot;
  uint32_t carry = 0;
  for (size_t chunk = 0; chunk < n; chunk += kScanTile) {
    size_t base = chunk + (size_t)threadIdx.x * kScanItems;
    uint32_t v[kScanItems];
    uint32_t s = 0;
#pragma unroll
    for (int i = 0; i < kScanItems; i++) {
      v[i] = base + i < n ? data[base + i] : 0;
      s += v[i];
    }
    uint32_t ex = block_exclusive_scan(s, ws, &tot) + carry;
#pragma unroll
    for (int i = 0; i < kScanItems; i++) {
      if (base + i < n) data[base + i] = ex;
      ex += v[i];
    }
    carry += tot;
    __syncthreads();
  }
  if (threadIdx.x == 0 && total_out) *total_out = carry;
}

__global__ void __launch_bounds__(kScanThreads) scan_apply_kernel(const uint32_t* in, uint32_t* out, size_t n,
                                                                  const uint32_t* n_dev, const uint32_t* sums) {
  __shared__ uint32_t ws[32];
  __shared__ uint32_t tot;
  if (n_dev) n = min(n, (size_t)*n_dev);
  if ((size_t)blockIdx.x * kScanTile >= n) return;
  size_t base = (size_t)blockIdx.x * kScanTile + (size_t)threadIdx.x * kScanItems;
  uint32_t v[kScanItems];
  uint32_t s = 0;
#pragma unroll
  for (int i = 0; i < kScanItems; i++) {
    v[i] = base + i < n ? in[base + i] : 0;
    s += v[i];
  }
  uint32_t ex = block_exclusive_scan(s, ws, &tot) + sums[blockIdx.x];
#pragma unroll
  for (int i = 0; i < kScanItems; i++) {
    if (base + i < n) out[base + i] = ex;
    ex += v[i];
  }
}

// Single-pass exclusive scan with decoupled look-back, for a count on the
// device far below its bound (the merge engine's scans: about 2^18 live
// entries under a 2^22 bound): one launch where the reduce / single / apply
// form takes three.  status[t] = epoch << 34 | state << 32 | value, state 1
// the tile's own sum, 2 its inclusive prefix; each call's epoch makes the
// words of earlier calls read as not ready, so the array is never cleared.
// ctr[0] hands tile ids out in the order blocks take them (a tile waits only
// on tiles taken before it); the last block to finish resets ctr.  The
// look-back spin is bounded: past kSpinLimit it sets kErrSpin in *err.
constexpr uint64_t kLbAgg = 1ull << 32, kLbInc = 2ull << 32;
constexpr uint32_t kLbSpinLimit = 1u << 22;

__global__ void __launch_bounds__(kScanThreads) scan_lb_kernel(const uint32_t* __restrict__ in,
                                                               uint32_t* __restrict__ out, size_t n_upper,
                                                               const uint32_t* __restrict__ n_dev,
                                                               uint32_t* __restrict__ total_out,
                                                               uint64_t* __restrict__ status,
                                                               uint32_t* __restrict__ ctr, uint32_t epoch,
                                                               uint32_t* __restrict__ err) {
  __shared__ uint32_t ws[32];
  __shared__ uint32_t tot, s_tile, s_prefix;
  const size_t n = n_dev ? min(n_upper, (size_t)*n_dev) : n_upper;
  const size_t n_tiles = (n + kScanTile - 1) / kScanTile;
  if (threadIdx.x == 0) s_tile = atomicAdd(&ctr[0], 1u);
  __syncthreads();
  const uint32_t tile = s_tile;
  const uint64_t tag = (uint64_t)epoch << 34;
  if (tile < n_tiles) {
    const size_t base = (size_t)tile * kScanTile + (size_t)threadIdx.x * kScanItems;
    uint32_t v[kScanItems];
    uint32_t sum = 0;
#pragma unroll
    for (int i = 0; i < kScanItems; i++) {
      v[i] = base + i < n ? in[base + i] : 0;
      sum += v[i];
    }
    uint32_t ex = block_exclusive_scan(sum, ws, &tot);
    if (threadIdx.x == 0) {
      uint32_t prefix = 0;
      if (tile > 0) {
        st_release(&status[tile], tag | kLbAgg | tot);
        int64_t t = (int64_t)tile - 1;
        uint32_t spins = 0;
        while (t >= 0) {
          const uint64_t w = ld_acquire(&status[t]);
          const uint32_t state = (uint32_t)(w >> 32) & 3u;
          if ((uint32_t)(w >> 34) != epoch || state == 0) {
            if (++spins > kLbSpinLimit) {
              if (err) atomicOr(err, kErrSpin);
              break;
            }
            if (spins > 64) __nanosleep(64);
            continue;
          }
          prefix += (uint32_t)w;
          if (state == 2) break;
          t--;
        }
      }
      st_release(&status[tile], tag | kLbInc | (uint64_t)(prefix + tot));
      s_prefix = prefix;
      if (tile == n_tiles - 1 && total_out) *total_out = prefix + tot;
    }
    __syncthreads();
    ex += s_prefix;
#pragma unroll
    for (int i = 0; i < kScanItems; i++) {
      if (base + i < n) out[base + i] = ex;
      ex += v[i];
    }
  } else if (tile == 0 && threadIdx.x == 0 && total_out) {
    *total_out = 0;  // nothing to scan
  }
  // the last block to finish makes the tile ids start at 0 again
  if (threadIdx.x == 0) {
    __threadfence();
    if (atomicAdd(&ctr[1], 1u) == gridDim.x - 1) {
      ctr[0] = 0;
      ctr[1] = 0;
      __threadfence();
    }
  }
}

// ---------------------------------------------------------------- sort ----
constexpr int kMaxPasses = 8;
constexpr uint32_t kFlagAgg = 1u << 30;
constexpr uint32_t kFlagPrefix = 2u << 30;
constexpr uint32_t kValMask = (1u << 30) - 1u;
constexpr uint32_t kSpinLimit = 1u << 22;

// all digit histograms in one read of the keys: hist[pass][256]
__global__ void __launch_bounds__(kSortThreads) sort_upfront_hist_kernel(const uint64_t* __restrict__ keys,
                                                                         size_t n, const uint32_t* __restrict__ n_dev,
                                                                         int begin_bit, int passes,
                                                                         uint32_t* __restrict__ hist) {
  __shared__ uint32_t h[kMaxPasses][kRadix];
  if (n_dev) n = min(n, (size_t)*n_dev);
  for (int i = threadIdx.x; i < kMaxPasses * kRadix; i += kSortThreads) (&h[0][0])[i] = 0;
  __syncthreads();
  const size_t stride = (size_t)gridDim.x * blockDim.x;
  for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) {
    const uint64_t k = keys[i];
    for (int p = 0; p < passes; p++) atomicAdd(&h[p][digit_of(k, begin_bit + 8 * p)], 1u);
  }
  __syncthreads();
  for (int i = threadIdx.x; i < passes * kRadix; i += kSortThreads) {
    const uint32_t c = (&h[0][0])[i];
    if (c) atomicAdd(hist + i, c);
  }
}

// exclusive scan of each pass's 256 counts -> global bucket starts
__global__ void sort_digit_scan_kernel(uint32_t* __restrict__ hist, int passes) {
  __shared__ uint32_t ws[32];
  for (int p = 0; p < passes; p++) {
    const uint32_t c = hist[p * kRadix + threadIdx.x];
    const uint32_t e = block_exclusive_scan(c, ws, nullptr);
    hist[p * kRadix + threadIdx.x] = e;
  }
}

template <int T>
struct ScatterSmem {
  uint64_t k[T * kSortItems];
  uint32_t v[T * kSortItems];
  uint32_t wh[T / 32][kRadix];
  uint32_t tstart[kRadix];
  uint32_t gofs[kRadix];
  uint32_t ws[32];
  uint32_t tile;
};

// payload_mode: 0 = read vals_in; 1 = generate (op code << 30 | i), ops nullable.
// Blocks take tiles in increasing order from tile_counter until the tiles run
// out; a block only ever waits on lower tiles, which running blocks hold, so
// any grid size is safe (the launcher uses at most the resident blocks).
template <int T>
__global__ void __launch_bounds__(T) sort_onesweep_kernel(
    const uint64_t* __restrict__ keys_in, const uint32_t* __restrict__ vals_in, const uint8_t* __restrict__ ops,
    int payload_mode, uint64_t* __restrict__ keys_out, uint32_t* __restrict__ vals_out, size_t n,
    const uint32_t* __restrict__ n_dev, int shift, const uint32_t* __restrict__ gbase,
    uint32_t* __restrict__ tile_counter, uint32_t* __restrict__ status, uint32_t* __restrict__ err) {
  static_assert(T >= kRadix, "one thread per digit");
  constexpr int kTile = T * kSortItems;
  constexpr int kWarps = T / 32;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  ScatterSmem<T>& S = *reinterpret_cast<ScatterSmem<T>*>(smem_raw);
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  if (n_dev) n = min(n, (size_t)*n_dev);
  const uint32_t lt_mask = (1u << lane) - 1u;
  for (;;) {
    if (threadIdx.x == 0) S.tile = atomicAdd(tile_counter, 1u);
    for (int i = threadIdx.x; i < kWarps * kRadix; i += T) (&S.wh[0][0])[i] = 0;
    __syncthreads();
    const uint32_t tile = S.tile;
    const size_t tile_base = (size_t)tile * kTile;
    if (tile_base >= n) return;  // tiles are handed out in order: later ones are empty too
    const size_t warp_base = tile_base + (size_t)warp * (32 * kSortItems);
    uint64_t key[kSortItems];
    uint32_t val[kSortItems];
    uint32_t rank[kSortItems];
#pragma unroll
    for (int r = 0; r < kSortItems; r++) {
      const size_t idx = warp_base + (size_t)r * 32 + lane;
      const bool valid = idx < n;
      key[r] = valid ? keys_in[idx] : 0;
      if (payload_mode == 0) val[r] = valid ? vals_in[idx] : 0;
      else val[r] = (uint32_t)idx | (ops && valid ? (op_code(ops[idx]) << 30) : 0u);
      const uint32_t d = valid ? digit_of(key[r], shift) : 0x1FFu;
      // lanes holding the same digit: AND of eight bit ballots (plus a validity bit)
      uint32_t peers = __ballot_sync(0xffffffffu, valid);
      peers = valid ? peers : ~peers;
#pragma unroll
      for (int b = 0; b < 8; b++) {
        const uint32_t bal = __ballot_sync(0xffffffffu, (d >> b) & 1u);
        peers &= ((d >> b) & 1u) ? bal : ~bal;
      }
      uint32_t before = 0;
      if (valid) before = S.wh[warp][d];
      __syncwarp();
      if (valid && lane == (uint32_t)(__ffs(peers) - 1)) S.wh[warp][d] = before + __popc(peers);
      __syncwarp();
      rank[r] = before + __popc(peers & lt_mask);
    }
    __syncthreads();
    // per digit: prefix over warps and the tile total
    uint32_t total = 0;
    if (threadIdx.x < kRadix) {
      const int d = threadIdx.x;
#pragma unroll
      for (int w = 0; w < kWarps; w++) {
        const uint32_t c = S.wh[w][d];
        S.wh[w][d] = total;
        total += c;
      }
      // publish this tile's count, then look back for the exclusive prefix
      uint32_t* my = status + (size_t)tile * kRadix + d;
      if (tile == 0) {
        st_relaxed32(my, kFlagPrefix | total);
        S.gofs[d] = gbase[d];
      } else {
        st_relaxed32(my, kFlagAgg | total);
        // look back eight predecessors per step (independent loads), in order
        uint32_t excl = 0;
        int64_t t = (int64_t)tile - 1;
        uint32_t spins = 0;
        while (t >= 0) {
          uint32_t wv[8];
#pragma unroll
          for (int j = 0; j < 8; j++)
            wv[j] = (t - j >= 0) ? ld_relaxed32(status + (size_t)(t - j) * kRadix + d) : kFlagPrefix;
          int used = 0;
          bool done = false, wait = false;
#pragma unroll
          for (int j = 0; j < 8; j++) {
            if (done || wait) continue;
            const uint32_t f = wv[j] & ~kValMask;
            if (f == 0) {
              wait = true;
              continue;
            }
            excl += wv[j] & kValMask;
            used++;
            if (f == kFlagPrefix) done = true;
          }
          if (done) break;
          t -= used;
          if (wait) {
            if (++spins > kSpinLimit) {
              atomicOr(err, kErrSpin);
              break;
            }
            if (spins > 64) __nanosleep(64);
          }
        }
        st_relaxed32(my, kFlagPrefix | (excl + total));
        S.gofs[d] = gbase[d] + excl;
      }
    }
    const uint32_t st = block_exclusive_scan(threadIdx.x < kRadix ? total : 0u, S.ws, nullptr);
    if (threadIdx.x < kRadix) S.tstart[threadIdx.x] = st;
    __syncthreads();
#pragma unroll
    for (int r = 0; r < kSortItems; r++) {
      const size_t idx = warp_base + (size_t)r * 32 + lane;
      if (idx < n) {
        const uint32_t d = digit_of(key[r], shift);
        const uint32_t pos = S.tstart[d] + S.wh[warp][d] + rank[r];
        S.k[pos] = key[r];
        S.v[pos] = val[r];
      }
    }
    __syncthreads();
    const uint32_t tile_n = (uint32_t)min((size_t)kTile, n - tile_base);
    for (uint32_t i = threadIdx.x; i < tile_n; i += T) {
      const uint64_t k = S.k[i];
      const uint32_t d = digit_of(k, shift);
      const uint32_t g = S.gofs[d] + (i - S.tstart[d]);
      keys_out[g] = k;
      vals_out[g] = S.v[i];
    }
    __syncthreads();  // the staging buffers and S.tile are reused by the next tile
  }
}

__global__ void iota_payload_kernel(uint32_t* out, const uint8_t* ops, size_t n) {
  size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) out[i] = (uint32_t)i | (ops ? (op_code(ops[i]) << 30) : 0u);
}

__global__ void copy_keys_kernel(const uint64_t* in, uint64_t* out, size_t n) {
  size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) out[i] = in[i];
}

}  // namespace

size_t scan_scratch_words(size_t n) { return (n + kScanTile - 1) / kScanTile + 1; }

cudaError_t scan_exclusive_u32(const uint32_t* in, uint32_t* out, size_t n, uint32_t* total_dev, uint32_t* scratch,
                               cudaStream_t s, const uint32_t* n_dev) {
  if (n == 0) {
    if (total_dev) return cudaMemsetAsync(total_dev, 0, sizeof(uint32_t), s);
    return cudaSuccess;
  }
  if (n <= (size_t)kScanTile && !n_dev) {
    if (in != out) {
      cudaError_t e = cudaMemcpyAsync(out, in, n * sizeof(uint32_t), cudaMemcpyDeviceToDevice, s);
      if (e != cudaSuccess) return e;
    }
    scan_single_kernel<<<1, kScanThreads, 0, s>>>(out, n, total_dev);
    count_launch();
    return cudaGetLastError();
  }
  size_t nb = (n + kScanTile - 1) / kScanTile;
  scan_reduce_kernel<<<(unsigned)nb, kScanThreads, 0, s>>>(in, n, n_dev, scratch);
  count_launch();
  scan_single_kernel<<<1, kScanThreads, 0, s>>>(scratch, nb, total_dev);
  count_launch();
  scan_apply_kernel<<<(unsigned)nb, kScanThreads, 0, s>>>(in, out, n, n_dev, scratch);
  count_launch();
  return cudaGetLastError();
}

size_t scan_lb_words(size_t n_upper) { return (n_upper + kScanTile - 1) / kScanTile + 1; }

cudaError_t scan_exclusive_u32_lb(const uint32_t* in, uint32_t* out, size_t n_upper, const uint32_t* n_dev,
                                  uint32_t* total_dev, uint64_t* status, uint32_t* ctr, uint32_t* epoch,
                                  uint32_t* err, cudaStream_t s) {
  *epoch = (*epoch + 1) & ((1u << 30) - 1);
  if (*epoch == 0) *epoch = 1;  // zeroed status words carry epoch 0
  const size_t blocks = n_upper ? (n_upper + kScanTile - 1) / kScanTile : 1;
  scan_lb_kernel<<<(unsigned)blocks, kScanThreads, 0, s>>>(in, out, n_upper, n_dev, total_dev, status, ctr, *epoch,
                                                           err);
  count_launch();
  return cudaGetLastError();
}

// Opt the onesweep kernels into >48 KB of shared memory on the current device.
cudaError_t sort_prepare() {
  cudaError_t e = cudaFuncSetAttribute(sort_onesweep_kernel<256>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       (int)sizeof(ScatterSmem<256>));
  if (e == cudaSuccess)
    e = cudaFuncSetAttribute(sort_onesweep_kernel<512>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)sizeof(ScatterSmem<512>));
  if (e == cudaSuccess)
    e = cudaFuncSetAttribute(sort_onesweep_kernel<1024>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)sizeof(ScatterSmem<1024>));
  return e;
}

// resident onesweep blocks on the current device (cached per device and block size)
template <int T>
static unsigned onesweep_resident() {
  static unsigned cache[64] = {};
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) return 148;
  if (!cache[dev]) {
    int per = 0, sms = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, sort_onesweep_kernel<T>, T, sizeof(ScatterSmem<T>)) !=
            cudaSuccess ||
        per < 1)
      per = 1;
    if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess || sms < 1) sms = 148;
    cache[dev] = (unsigned)(per * sms);
  }
  return cache[dev];
}

// one digit pass with T-thread tiles
template <int T>
static void onesweep_pass(const uint64_t* src_k, const uint32_t* src_v, const uint8_t* ops, int mode, uint64_t* dst_k,
                          uint32_t* dst_v, size_t n, const uint32_t* n_dev, int shift, const uint32_t* gbase,
                          uint32_t* counter, uint32_t* status, uint32_t* err, uint32_t n_tiles, cudaStream_t s) {
  const unsigned grid = min(n_tiles, onesweep_resident<T>());
  sort_onesweep_kernel<T><<<grid, T, sizeof(ScatterSmem<T>), s>>>(src_k, src_v, ops, mode, dst_k, dst_v, n, n_dev,
                                                                  shift, gbase, counter, status, err);
}

// scratch: hist[8][256] | tile counters[8] (+pad) | status[8][tiles][256]
static_assert(kSortTileKeys == (size_t)kMinTile && kSortMaxPasses == (size_t)kMaxPasses &&
                  kSortRadix == (size_t)kRadix,
              "the scratch layout in bt_internal.h must match the sort (sized for the smallest tile)");

size_t sort_scratch_words(size_t n) {
  const size_t w = sort_scratch_words_for(n);
  const size_t sc = scan_scratch_words(n);  // callers reuse this scratch for scans
  return w > sc ? w : sc;
}

// Sorts n pairs by bits [begin_bit, end_bit) of the key.  Input keys_in (and
// vals_in, or generated payload when vals_in == nullptr) are not modified.
// Result lands in (k_a, v_a) or (k_b, v_b); *k_out/*v_out name which.  A look-
// back timeout sets kErrSpin in *err (the result is then not sorted).  With
// n_dev the count is min(n, *n_dev), read on the device (n sizes the grids).
cudaError_t radix_sort_pairs(const uint64_t* keys_in, const uint32_t* vals_in, const uint8_t* ops, uint64_t* k_a,
                             uint32_t* v_a, uint64_t* k_b, uint32_t* v_b, size_t n, int begin_bit, int end_bit,
                             uint32_t* scratch, cudaStream_t s, uint64_t** k_out, uint32_t** v_out, uint32_t* err,
                             const uint32_t* n_dev, int tile_threads) {
  *k_out = k_a;
  *v_out = v_a;
  if (n == 0) return cudaSuccess;
  const int passes = (end_bit - begin_bit + 7) / 8;
  if (passes <= 0) {
    if (n_dev) return cudaErrorInvalidValue;
    copy_keys_kernel<<<(unsigned)((n + 255) / 256), 256, 0, s>>>(keys_in, k_a, n);
    count_launch();
    if (vals_in) cudaMemcpyAsync(v_a, vals_in, n * sizeof(uint32_t), cudaMemcpyDeviceToDevice, s);
    else {
      iota_payload_kernel<<<(unsigned)((n + 255) / 256), 256, 0, s>>>(v_a, ops, n);
      count_launch();
    }
    return cudaGetLastError();
  }
  if (passes > kMaxPasses) return cudaErrorInvalidValue;
  const int T = tile_threads == 256 || tile_threads == 1024 ? tile_threads : 512;
  const size_t tile = (size_t)T * kSortItems;
  const uint32_t n_tiles = (uint32_t)((n + tile - 1) / tile);
  uint32_t* hist = scratch;
  uint32_t* counters = scratch + kMaxPasses * kRadix;
  uint32_t* status = counters + 64;
  cudaError_t e = cudaMemsetAsync(scratch, 0,
                                  ((size_t)kMaxPasses * kRadix + 64 + (size_t)passes * n_tiles * kRadix) * 4, s);
  if (e != cudaSuccess) return e;
  unsigned hb = (unsigned)min((n + kSortThreads * kSortItems - 1) / (kSortThreads * kSortItems), (size_t)1024);
  sort_upfront_hist_kernel<<<hb, kSortThreads, 0, s>>>(keys_in, n, n_dev, begin_bit, passes, hist);
  count_launch();
  sort_digit_scan_kernel<<<1, kRadix, 0, s>>>(hist, passes);
  count_launch();
  const uint64_t* src_k = keys_in;
  const uint32_t* src_v = vals_in;
  int mode = vals_in ? 0 : 1;
  uint64_t* dst_k = k_a;
  uint32_t* dst_v = v_a;
  for (int p = 0; p < passes; p++) {
    uint32_t* st = status + (size_t)p * n_tiles * kRadix;
    if (T == 256)
      onesweep_pass<256>(src_k, src_v, ops, mode, dst_k, dst_v, n, n_dev, begin_bit + 8 * p, hist + p * kRadix,
                         counters + p, st, err, n_tiles, s);
    else if (T == 1024)
      onesweep_pass<1024>(src_k, src_v, ops, mode, dst_k, dst_v, n, n_dev, begin_bit + 8 * p, hist + p * kRadix,
                          counters + p, st, err, n_tiles, s);
    else
      onesweep_pass<512>(src_k, src_v, ops, mode, dst_k, dst_v, n, n_dev, begin_bit + 8 * p, hist + p * kRadix,
                         counters + p, st, err, n_tiles, s);
    count_launch();
    e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    src_k = dst_k;
    src_v = dst_v;
    mode = 0;
    dst_k = (dst_k == k_a) ? k_b : k_a;
    dst_v = (dst_v == v_a) ? v_b : v_a;
  }
  *k_out = const_cast<uint64_t*>(src_k);
  *v_out = const_cast<uint32_t*>(src_v);
  return cudaSuccess;
}

// ---------------------------------------------------------- merge sort ----
// Sort of the hash front end's touched requests: at 95/5 a batch of 2^22
// has about 2^18 of them, too few for the onesweep passes to be bound by
// bytes: each of the eight is a launch, a one-wave tile pass and a look-back.
// Here:
//   1. ms_tile_kernel: each block sorts a tile of kMsTile pairs (bitonic
//      network in registers, shuffles and shared memory), giving sorted runs;
//   2. ms_merge_kernel, once per round: pairs of sorted runs merge into runs
//      of twice the length (merge path: two warps find where the block's
//      output range splits the two runs with 32-way searches, the block
//      stages the two pieces in shared memory, each thread merges 4
//      outputs), until one run remains.
// The order is by key, then by the request index in the payload's low 30
// bits.  Those indices are unique and increase in input order, so the order
// is the stable one (the onesweep passes' order) and every comparison is
// strict.  The device count n_dev fixes the number of rounds R: the host
// launches the most rounds the capacity can need, the surplus ones return at
// once, and the tile kernel writes its runs where R rounds of ping-pong leave
// the result in (k_a, v_a).
namespace {

constexpr int kMsThreads = 512;
constexpr int kMsItems = 4;
constexpr int kMsTile = kMsThreads * kMsItems;  // 2048 pairs
constexpr uint32_t kMsIdx = 0x3FFFFFFFu;

// without short-circuit branches: the callers select on the result
__device__ __forceinline__ bool ms_less(uint64_t ka, uint32_t va, uint64_t kb, uint32_t vb) {
  return (ka < kb) | ((ka == kb) & ((va & kMsIdx) < (vb & kMsIdx)));
}

__device__ __forceinline__ size_t ms_count(size_t n_upper, const uint32_t* n_dev) {
  return n_dev ? min((size_t)*n_dev, n_upper) : n_upper;
}

// merge rounds that turn ceil(n / kMsTile) sorted runs into one
__host__ __device__ __forceinline__ int ms_rounds(size_t n) {
  const size_t runs = (n + kMsTile - 1) / kMsTile;
  int r = 0;
  while (((size_t)1 << r) < runs) r++;
  return r;
}

// compare-exchange so that (a, b) ends in ascending order when `asc`
__device__ __forceinline__ void ms_cx(uint64_t& ka, uint32_t& va, uint64_t& kb, uint32_t& vb, bool asc) {
  const bool sw = ms_less(kb, vb, ka, va) == asc;
  const uint64_t k0 = sw ? kb : ka, k1 = sw ? ka : kb;
  const uint32_t v0 = sw ? vb : va, v1 = sw ? va : vb;
  ka = k0;
  kb = k1;
  va = v0;
  vb = v1;
}

// a thread's element of index i meets its partner of index i ^ j: the lower
// index keeps the smaller one where the bitonic sequence ascends
__device__ __forceinline__ void ms_keep(uint64_t& k, uint32_t& v, uint64_t pk, uint32_t pv, int i, int j, int kk) {
  const bool asc = (i & kk) == 0, lower = (i & j) == 0;
  const bool p_lt = ms_less(pk, pv, k, v);
  const bool m_lt = ms_less(k, v, pk, pv);
  const bool take = (lower == asc) ? p_lt : m_lt;
  k = take ? pk : k;
  v = take ? pv : v;
}

// the stride-J exchanges inside a thread's registers (J < kMsItems)
template <int J>
__device__ __forceinline__ void ms_reg_stage(uint64_t (&K)[kMsItems], uint32_t (&V)[kMsItems], int base, int kk) {
#pragma unroll
  for (int e = 0; e < kMsItems; e++)
    if ((e & J) == 0) ms_cx(K[e], V[e], K[e | J], V[e | J], ((base + e) & kk) == 0);
}

__device__ __forceinline__ int ms_phys(int i) { return i + (i >> 3); }  // padding: fewer bank conflicts

// Bitonic sort of a tile: element i of the tile is register i % 4 of thread
// i / 4.  Exchanges at strides 1-2 stay in registers, 4-64 are shuffles
// within the warp, 128 and up go through shared memory (10 of the 66
// stages).  Compares and exchanges are selects, not branches: with one tile
// per SM the kernel is bound by its dependent instructions.
__global__ void __launch_bounds__(kMsThreads) ms_tile_kernel(const uint64_t* __restrict__ kin,
                                                             const uint32_t* __restrict__ vin, size_t n_upper,
                                                             const uint32_t* __restrict__ n_dev, uint64_t* k_a,
                                                             uint32_t* v_a, uint64_t* k_b, uint32_t* v_b) {
  __shared__ uint64_t sk[kMsTile + kMsTile / 8];
  __shared__ uint32_t sv[kMsTile + kMsTile / 8];
  const size_t n = ms_count(n_upper, n_dev);
  const bool to_a = (ms_rounds(n) & 1) == 0;
  uint64_t* ko = to_a ? k_a : k_b;
  uint32_t* vo = to_a ? v_a : v_b;
  const int base = threadIdx.x * kMsItems;
  for (size_t t0 = (size_t)blockIdx.x * kMsTile; t0 < n; t0 += (size_t)gridDim.x * kMsTile) {
    const int cnt = (int)min((size_t)kMsTile, n - t0);
    uint64_t K[kMsItems];
    uint32_t V[kMsItems];
    // the tail of the last tile sorts after every request (index bits all ones)
#pragma unroll
    for (int e = 0; e < kMsItems; e++) {
      const int i = base + e;
      K[e] = i < cnt ? kin[t0 + i] : ~0ull;
      V[e] = i < cnt ? vin[t0 + i] : 0xFFFFFFFFu;
    }
    for (int kk = 2; kk <= kMsTile; kk <<= 1) {
      for (int j = kk >> 1; j >= kMsItems; j >>= 1) {
        if (j >= 32 * kMsItems) {
          __syncthreads();  // the previous exchange's reads are done
#pragma unroll
          for (int e = 0; e < kMsItems; e++) {
            sk[ms_phys(base + e)] = K[e];
            sv[ms_phys(base + e)] = V[e];
          }
          __syncthreads();
#pragma unroll
          for (int e = 0; e < kMsItems; e++) {
            const int p = ms_phys((base + e) ^ j);
            ms_keep(K[e], V[e], sk[p], sv[p], base + e, j, kk);
          }
        } else {
          const int lm = j / kMsItems;
#pragma unroll
          for (int e = 0; e < kMsItems; e++) {
            const uint64_t pk = __shfl_xor_sync(0xffffffffu, K[e], lm);
            const uint32_t pv = __shfl_xor_sync(0xffffffffu, V[e], lm);
            ms_keep(K[e], V[e], pk, pv, base + e, j, kk);
          }
        }
      }
      static_assert(kMsItems == 4, "register stages below are for 4 items per thread");
      if (kk >= 4) ms_reg_stage<2>(K, V, base, kk);
      ms_reg_stage<1>(K, V, base, kk);
    }
#pragma unroll
    for (int e = 0; e < kMsItems; e++) {
      const int i = base + e;
      if (i < cnt) {
        ko[t0 + i] = K[e];
        vo[t0 + i] = V[e];
      }
    }
    __syncthreads();  // shared memory is reused by the next tile
  }
}

// a = the number of elements of A among the first d of merge(A, B): the
// first a in [max(0, d - nb), min(d, na)] with !(A[a] < B[d - 1 - a]); one
// warp, 32 candidates per step
__device__ __forceinline__ size_t ms_split(const uint64_t* __restrict__ k, const uint32_t* __restrict__ v,
                                           size_t a_beg, size_t na, size_t b_beg, size_t nb, size_t d) {
  const uint32_t lane = threadIdx.x & 31;
  size_t lo = d > nb ? d - nb : 0, hi = min(d, na);
  while (lo < hi) {
    const size_t stride = (hi - lo + 31) / 32;
    const size_t a = lo + (size_t)lane * stride;
    bool p = false;
    if (a < hi) {
      const size_t b = b_beg + d - 1 - a;
      p = ms_less(k[a_beg + a], v[a_beg + a], k[b], v[b]);
    }
    const int c = __popc(__ballot_sync(0xffffffffu, p));
    if (c == 0) {
      hi = lo;
    } else {
      const size_t top = lo + (size_t)c * stride;
      lo += (size_t)(c - 1) * stride + 1;
      hi = min(hi, top);
    }
  }
  return lo;
}

__global__ void __launch_bounds__(kMsThreads) ms_merge_kernel(uint64_t* k_a, uint32_t* v_a, uint64_t* k_b,
                                                              uint32_t* v_b, size_t n_upper,
                                                              const uint32_t* __restrict__ n_dev, int round) {
  __shared__ uint64_t sk[kMsTile];
  __shared__ uint32_t sv[kMsTile];
  __shared__ size_t split[2];
  const size_t n = ms_count(n_upper, n_dev);
  const int R = ms_rounds(n);
  if (round >= R) return;
  const bool from_a = ((R - round) & 1) == 0;
  const uint64_t* __restrict__ ks = from_a ? k_a : k_b;
  const uint32_t* __restrict__ vs = from_a ? v_a : v_b;
  uint64_t* __restrict__ kd = from_a ? k_b : k_a;
  uint32_t* __restrict__ vd = from_a ? v_b : v_a;
  const size_t L = (size_t)kMsTile << round;  // input run length
  const int warp = threadIdx.x >> 5;
  for (size_t o0 = (size_t)blockIdx.x * kMsTile; o0 < n; o0 += (size_t)gridDim.x * kMsTile) {
    const int cnt = (int)min((size_t)kMsTile, n - o0);
    const size_t ps = o0 / (2 * L) * (2 * L);
    const size_t a_beg = ps, a_end = min(ps + L, n), b_end = min(ps + 2 * L, n);
    const size_t na = a_end - a_beg, nb = b_end - a_end;
    if (nb == 0) {  // the last run has no partner this round
      for (int i = threadIdx.x; i < cnt; i += kMsThreads) {
        kd[o0 + i] = ks[o0 + i];
        vd[o0 + i] = vs[o0 + i];
      }
      continue;
    }
    const size_t d0 = o0 - ps;
    if (warp < 2) {
      const size_t a = ms_split(ks, vs, a_beg, na, a_end, nb, warp == 0 ? d0 : d0 + cnt);
      if ((threadIdx.x & 31) == 0) split[warp] = a;
    }
    __syncthreads();
    const size_t a0 = split[0], a1 = split[1];
    const int la = (int)(a1 - a0), lb = cnt - la;
    const size_t b0 = a_end + (d0 - a0);
    for (int i = threadIdx.x; i < la; i += kMsThreads) {
      sk[i] = ks[a_beg + a0 + i];
      sv[i] = vs[a_beg + a0 + i];
    }
    for (int i = threadIdx.x; i < lb; i += kMsThreads) {
      sk[la + i] = ks[b0 + i];
      sv[la + i] = vs[b0 + i];
    }
    __syncthreads();
    // this thread's outputs: merge path in shared memory, then a serial merge
    const int d = threadIdx.x * kMsItems;
    uint64_t ok[kMsItems];
    uint32_t ov[kMsItems];
    const int m = d < cnt ? min(kMsItems, cnt - d) : 0;
    if (m > 0) {
      int lo = d > lb ? d - lb : 0, hi = min(d, la);
      while (lo < hi) {
        const int mid = (lo + hi) >> 1;
        if (ms_less(sk[mid], sv[mid], sk[la + d - 1 - mid], sv[la + d - 1 - mid])) lo = mid + 1;
        else hi = mid;
      }
      int ia = lo, ib = d - lo;
#pragma unroll
      for (int j = 0; j < kMsItems; j++) {
        if (j < m) {
          const bool take_a = ib >= lb || (ia < la && ms_less(sk[ia], sv[ia], sk[la + ib], sv[la + ib]));
          const int at = take_a ? ia++ : la + ib++;
          ok[j] = sk[at];
          ov[j] = sv[at];
        }
      }
    }
    __syncthreads();
#pragma unroll
    for (int j = 0; j < kMsItems; j++)
      if (j < m) {
        sk[d + j] = ok[j];
        sv[d + j] = ov[j];
      }
    __syncthreads();
    for (int i = threadIdx.x; i < cnt; i += kMsThreads) {
      kd[o0 + i] = sk[i];
      vd[o0 + i] = sv[i];
    }
    __syncthreads();
  }
}

}  // namespace

cudaError_t merge_sort_pairs(const uint64_t* keys_in, const uint32_t* vals_in, uint64_t* k_a, uint32_t* v_a,
                             uint64_t* k_b, uint32_t* v_b, size_t n, const uint32_t* n_dev, int sm_count,
                             cudaStream_t s, uint64_t** k_out, uint32_t** v_out) {
  *k_out = k_a;
  *v_out = v_a;
  if (n == 0) return cudaSuccess;
  // two blocks per SM (a wave at most): rounds past the count return at once,
  // and a large count loops over its tiles
  const size_t tiles = (n + kMsTile - 1) / kMsTile;
  const unsigned grid = (unsigned)min(tiles, (size_t)(sm_count > 0 ? sm_count : 148) * 2);
  ms_tile_kernel<<<grid, kMsThreads, 0, s>>>(keys_in, vals_in, n, n_dev, k_a, v_a, k_b, v_b);
  count_launch();
  const int r_max = ms_rounds(n);
  for (int r = 0; r < r_max; r++) {
    ms_merge_kernel<<<grid, kMsThreads, 0, s>>>(k_a, v_a, k_b, v_b, n, n_dev, r);
    count_launch();
  }
  return cudaGetLastError();
}

}  // namespace bt
