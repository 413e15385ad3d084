// Hand-written stable LSD radix sort of (uint64 key, uint32 payload) pairs and
// a device-wide exclusive scan.  They replace the reference's CUB calls
// DeviceRadixSort::SortPairs, DeviceRunLengthEncode::Encode and
// DeviceScan::ExclusiveSum (src/gpu-stm-tree-v38/bpt-gpustm-kernel.cu:289-324).
//
// Sort pass structure (8-bit digits, tile = 4096 items, 512 threads):
//   1. tile histogram      reads 8 B/item
//   2. exclusive scan of the digit-major [256 x tiles] count table
//   3. scatter             reads 12 B/item, writes 12 B/item
// The scatter ranks items stably inside the tile with __match_any_sync
// (each warp owns a contiguous 256-item chunk and walks it in 8 rounds),
// stages the tile in shared memory in digit order and writes each digit run
// contiguously, so global writes are coalesced.  No inter-CTA waits.
#include <cstdint>
#include <cuda_runtime.h>

#include "bt_common.cuh"
#include "bt_internal.h"

namespace bt {

namespace {

constexpr int kSortThreads = 512;
constexpr int kSortItems = 8;
constexpr int kTile = kSortThreads * kSortItems;  // 4096
constexpr int kWarps = kSortThreads / 32;           // 16
constexpr int kRadix = 256;

constexpr int kScanThreads = 1024;
constexpr int kScanItems = 4;
constexpr int kScanTile = kScanThreads * kScanItems;  // 4096

__device__ __forceinline__ uint32_t digit_of(uint64_t k, int shift) { return (uint32_t)(k >> shift) & 0xff; }
// 2-bit op code carried in the payload: 0 insert, 1 get, 3 anything else (rejected)
__device__ __forceinline__ uint32_t op_code(uint8_t op) { return op <= 1 ? (uint32_t)op : 3u; }

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

__global__ void __launch_bounds__(kScanThreads) scan_reduce_kernel(const uint32_t* in, size_t n, uint32_t* sums) {
  __shared__ uint32_t ws[32];
  __shared__ uint32_t tot;
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
                                                                  const uint32_t* sums) {
  __shared__ uint32_t ws[32];
  __shared__ uint32_t tot;
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

// ---------------------------------------------------------------- sort ----
__global__ void __launch_bounds__(kSortThreads) sort_hist_kernel(const uint64_t* __restrict__ keys, size_t n,
                                                                 int shift, uint32_t* __restrict__ tile_hist,
                                                                 uint32_t n_tiles) {
  __shared__ uint32_t h[kRadix];
  for (int i = threadIdx.x; i < kRadix; i += kSortThreads) h[i] = 0;
  __syncthreads();
  const size_t base = (size_t)blockIdx.x * kTile;
#pragma unroll
  for (int i = 0; i < kSortItems; i++) {
    size_t idx = base + (size_t)i * kSortThreads + threadIdx.x;
    bool valid = idx < n;
    uint32_t d = valid ? digit_of(keys[idx], shift) : 0xFFFFu;
    // warp-aggregated shared atomics: one add per distinct digit per warp
    uint32_t peers = __match_any_sync(0xffffffffu, d);
    if (valid && (lane_id() == (uint32_t)(__ffs(peers) - 1))) atomicAdd(&h[d], (uint32_t)__popc(peers));
  }
  __syncthreads();
  for (int d = threadIdx.x; d < kRadix; d += kSortThreads) tile_hist[(size_t)d * n_tiles + blockIdx.x] = h[d];
}

struct ScatterSmem {
  uint64_t k[kTile];
  uint32_t v[kTile];
  uint32_t wh[kWarps][kRadix];
  uint32_t tstart[kRadix];
  uint32_t gofs[kRadix];
  uint32_t ws[32];
};

// payload_mode: 0 = read vals_in; 1 = generate (ops[i] << 30 | i), ops nullable
__global__ void __launch_bounds__(kSortThreads) sort_scatter_kernel(
    const uint64_t* __restrict__ keys_in, const uint32_t* __restrict__ vals_in, const uint8_t* __restrict__ ops,
    int payload_mode, uint64_t* __restrict__ keys_out, uint32_t* __restrict__ vals_out, size_t n, int shift,
    const uint32_t* __restrict__ tile_off, uint32_t n_tiles) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  ScatterSmem& S = *reinterpret_cast<ScatterSmem*>(smem_raw);
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  for (int i = threadIdx.x; i < kWarps * kRadix; i += kSortThreads) (&S.wh[0][0])[i] = 0;
  for (int d = threadIdx.x; d < kRadix; d += kSortThreads)
    S.gofs[d] = tile_off[(size_t)d * n_tiles + blockIdx.x];
  __syncthreads();

  const size_t tile_base = (size_t)blockIdx.x * kTile;
  const size_t warp_base = tile_base + (size_t)warp * (32 * kSortItems);
  uint64_t key[kSortItems];
  uint32_t val[kSortItems];
  uint32_t rank[kSortItems];
  const uint32_t lt_mask = (1u << lane) - 1u;
#pragma unroll
  for (int r = 0; r < kSortItems; r++) {
    size_t idx = warp_base + (size_t)r * 32 + lane;
    bool valid = idx < n;
    key[r] = valid ? keys_in[idx] : 0;
    if (payload_mode == 0) val[r] = valid ? vals_in[idx] : 0;
    else val[r] = (uint32_t)idx | (ops && valid ? (op_code(ops[idx]) << 30) : 0u);
    uint32_t d = valid ? digit_of(key[r], shift) : 0xFFFFu;
    uint32_t peers = __match_any_sync(0xffffffffu, d);
    uint32_t before = 0;
    if (valid) before = S.wh[warp][d];
    __syncwarp();
    if (valid && lane == (uint32_t)(__ffs(peers) - 1)) S.wh[warp][d] = before + __popc(peers);
    __syncwarp();
    rank[r] = before + __popc(peers & lt_mask);
  }
  __syncthreads();
  // per digit: prefix over warps, and tile totals
  uint32_t total = 0;
  if (threadIdx.x < kRadix) {
    const int d = threadIdx.x;
#pragma unroll
    for (int w = 0; w < kWarps; w++) {
      uint32_t c = S.wh[w][d];
      S.wh[w][d] = total;
      total += c;
    }
  }
  // exclusive scan of the 256 digit totals (threads >= 256 contribute 0)
  uint32_t st = block_exclusive_scan(threadIdx.x < kRadix ? total : 0u, S.ws, nullptr);
  if (threadIdx.x < kRadix) S.tstart[threadIdx.x] = st;
  __syncthreads();
#pragma unroll
  for (int r = 0; r < kSortItems; r++) {
    size_t idx = warp_base + (size_t)r * 32 + lane;
    if (idx < n) {
      uint32_t d = digit_of(key[r], shift);
      uint32_t pos = S.tstart[d] + S.wh[warp][d] + rank[r];
      S.k[pos] = key[r];
      S.v[pos] = val[r];
    }
  }
  __syncthreads();
  const uint32_t tile_n = (uint32_t)min((size_t)kTile, n - tile_base);
  for (uint32_t i = threadIdx.x; i < tile_n; i += kSortThreads) {
    uint64_t k = S.k[i];
    uint32_t d = digit_of(k, shift);
    uint32_t g = S.gofs[d] + (i - S.tstart[d]);
    keys_out[g] = k;
    vals_out[g] = S.v[i];
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
                               cudaStream_t s) {
  if (n == 0) {
    if (total_dev) return cudaMemsetAsync(total_dev, 0, sizeof(uint32_t), s);
    return cudaSuccess;
  }
  if (n <= (size_t)kScanTile) {
    if (in != out) {
      cudaError_t e = cudaMemcpyAsync(out, in, n * sizeof(uint32_t), cudaMemcpyDeviceToDevice, s);
      if (e != cudaSuccess) return e;
    }
    scan_single_kernel<<<1, kScanThreads, 0, s>>>(out, n, total_dev);
    count_launch();
    return cudaGetLastError();
  }
  size_t nb = (n + kScanTile - 1) / kScanTile;
  scan_reduce_kernel<<<(unsigned)nb, kScanThreads, 0, s>>>(in, n, scratch);
  count_launch();
  scan_single_kernel<<<1, kScanThreads, 0, s>>>(scratch, nb, total_dev);
  count_launch();
  scan_apply_kernel<<<(unsigned)nb, kScanThreads, 0, s>>>(in, out, n, scratch);
  count_launch();
  return cudaGetLastError();
}

size_t sort_tiles(size_t n) { return (n + kTile - 1) / kTile; }

// Opt the scatter kernel into >48 KB of shared memory on the current device.
cudaError_t sort_prepare() {
  return cudaFuncSetAttribute(sort_scatter_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                              (int)sizeof(ScatterSmem));
}
size_t sort_scratch_words(size_t n) {
  size_t t = sort_tiles(n);
  return t * kRadix + scan_scratch_words(t * kRadix);
}

// Sorts n pairs by bits [begin_bit, end_bit) of the key.  Input keys_in (and
// vals_in, or generated payload when vals_in == nullptr) are not modified.
// Result lands in (k_a, v_a) or (k_b, v_b); *k_out/*v_out name which.
cudaError_t radix_sort_pairs(const uint64_t* keys_in, const uint32_t* vals_in, const uint8_t* ops, uint64_t* k_a,
                             uint32_t* v_a, uint64_t* k_b, uint32_t* v_b, size_t n, int begin_bit, int end_bit,
                             uint32_t* scratch, cudaStream_t s, uint64_t** k_out, uint32_t** v_out) {
  *k_out = k_a;
  *v_out = v_a;
  if (n == 0) return cudaSuccess;
  const uint32_t n_tiles = (uint32_t)sort_tiles(n);
  uint32_t* tile_hist = scratch;
  uint32_t* scan_tmp = scratch + (size_t)n_tiles * kRadix;
  const uint64_t* src_k = keys_in;
  const uint32_t* src_v = vals_in;
  int mode = vals_in ? 0 : 1;
  uint64_t* dst_k = k_a;
  uint32_t* dst_v = v_a;
  int passes = 0;
  for (int bit = begin_bit; bit < end_bit; bit += 8) {
    sort_hist_kernel<<<n_tiles, kSortThreads, 0, s>>>(src_k, n, bit, tile_hist, n_tiles);
    count_launch();
    cudaError_t e = scan_exclusive_u32(tile_hist, tile_hist, (size_t)n_tiles * kRadix, nullptr, scan_tmp, s);
    if (e != cudaSuccess) return e;
    sort_scatter_kernel<<<n_tiles, kSortThreads, sizeof(ScatterSmem), s>>>(src_k, src_v, ops, mode, dst_k, dst_v, n,
                                                                           bit, tile_hist, n_tiles);
    count_launch();
    e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    src_k = dst_k;
    src_v = dst_v;
    mode = 0;
    dst_k = (dst_k == k_a) ? k_b : k_a;
    dst_v = (dst_v == v_a) ? v_b : v_a;
    passes++;
  }
  if (passes == 0) {
    // nothing to sort: copy through with generated payload
    copy_keys_kernel<<<(unsigned)((n + 255) / 256), 256, 0, s>>>(keys_in, k_a, n);
    count_launch();
    if (vals_in) cudaMemcpyAsync(v_a, vals_in, n * sizeof(uint32_t), cudaMemcpyDeviceToDevice, s);
    else iota_payload_kernel<<<(unsigned)((n + 255) / 256), 256, 0, s>>>(v_a, ops, n);
    count_launch();
    return cudaGetLastError();
  }
  *k_out = const_cast<uint64_t*>(src_k);
  *v_out = const_cast<uint32_t*>(src_v);
  return cudaSuccess;
}

}  // namespace bt
