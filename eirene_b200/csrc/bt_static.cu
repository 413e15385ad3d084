// bt_bulk_build_static: the bulk build without any allocation.
//
// Some callers cannot allocate GPU memory when they load a tree: services
// whose device memory is reserved up front by another allocator (a
// framework's caching allocator, or a pool sized at start-up), where a
// cudaMalloc at request time fails or fragments that pool; and
// latency-critical threads, because cudaFree synchronises the whole device
// and stalls every other stream.  bt_bulk_build (the allocating entry point)
// takes its sort and compaction scratch from cudaMallocAsync; this variant
// takes it from the file-scope device array below instead.
//
// The array is kStaticMaxKeys keys' worth of scratch (about 2.6 MB).  Every
// GPU that loads this library holds it until the process exits.  All calls on
// one device share it and it keeps whatever the last call left there, so calls
// that overlap on the GPU (different streams, or different host threads) race
// and must be serialised by the caller.
//
// Host code cannot use the array's name as a device address (it names a host
// shadow); the device address is fetched once per device with
// cudaGetSymbolAddress, with that device current, on the first call made on
// that device.  That first call should therefore come before any stream
// capture begins on the device.  The address is kept for the life of the
// process: calls after cudaDeviceReset on that device are not supported (the
// reset unloads the module the address belongs to).
#include <mutex>

#include <cuda_runtime.h>

#include "../../include/eirene_b200.h"
#include "bt_common.cuh"
#include "bt_internal.h"

namespace {

constexpr size_t kStaticMaxKeys = BT_STATIC_BUILD_MAX_KEYS;
constexpr size_t up256(size_t x) { return (x + 255) & ~size_t(255); }
// the radix sort's scratch for kStaticMaxKeys keys (the sort's own layout,
// bt_internal.h); the scan's scratch, which shares it, is far smaller
constexpr size_t kSortWords = bt::sort_scratch_words_for(kStaticMaxKeys);
constexpr size_t kOffKa = 0;
constexpr size_t kOffKb = kOffKa + up256(kStaticMaxKeys * 8);
constexpr size_t kOffVa = kOffKb + up256(kStaticMaxKeys * 8);
constexpr size_t kOffVb = kOffVa + up256(kStaticMaxKeys * 4);
constexpr size_t kOffSort = kOffVb + up256(kStaticMaxKeys * 4);
constexpr size_t kOffPos = kOffSort + up256(kSortWords * 4);
constexpr size_t kOffUv = kOffPos + up256(kStaticMaxKeys * 4);
constexpr size_t kOffTot = kOffUv + up256(kStaticMaxKeys * 8);
constexpr size_t kStaticBytes = kOffTot + 256;

}  // namespace

static __device__ __align__(256) unsigned char g_build_scratch[kStaticBytes];

namespace {

constexpr int kMaxDevices = 64;
std::mutex g_mu;
unsigned char* g_dev_ptr[kMaxDevices] = {};

// Device address of g_build_scratch on `dev` (which must be current).
int scratch_for_device(int dev, unsigned char** out) {
  if (dev < 0 || dev >= kMaxDevices) return BT_ERR_INVALID_ARG;
  std::lock_guard<std::mutex> lk(g_mu);
  if (!g_dev_ptr[dev]) {
    void* p = nullptr;
    if (cudaGetSymbolAddress(&p, g_build_scratch) != cudaSuccess || p == nullptr) return BT_ERR_CUDA;
    g_dev_ptr[dev] = static_cast<unsigned char*>(p);
  }
  *out = g_dev_ptr[dev];
  return BT_OK;
}

int map_rc(int rc) {
  switch (rc) {
    case 0: return BT_OK;
    case -4: return BT_ERR_CAPACITY;
    case -5: return BT_ERR_RESERVED_KEY;
    case -6: return BT_ERR_STATIC_LIMIT;
    default: return BT_ERR_CUDA;
  }
}

}  // namespace

extern "C" int bt_bulk_build_static(bt_handle* H, const uint64_t* keys, const uint64_t* vals, size_t n,
                                    void* stream) {
  if (!H || (n && (!keys || !vals))) return BT_ERR_INVALID_ARG;
  if (n > kStaticMaxKeys) return BT_ERR_STATIC_LIMIT;
  int prev = -1;
  if (cudaGetDevice(&prev) != cudaSuccess) return BT_ERR_CUDA;
  const int dev = H->h.device;
  if (prev != dev && cudaSetDevice(dev) != cudaSuccess) return BT_ERR_CUDA;
  unsigned char* base = nullptr;
  int rc = scratch_for_device(dev, &base);
  if (rc == BT_OK && bt::tree_join(&H->h, static_cast<cudaStream_t>(stream)) != cudaSuccess) rc = BT_ERR_CUDA;
  if (rc == BT_OK) {
    if (bt::sort_scratch_words(n ? n : 1) > kSortWords) {
      // n is within the limit, so this means the sort's scratch layout and
      // the array's sizing disagree: an internal error, not a size error
      rc = BT_ERR_CUDA;
    } else {
      bt::BuildScratch sc;
      sc.ka = reinterpret_cast<uint64_t*>(base + kOffKa);
      sc.kb = reinterpret_cast<uint64_t*>(base + kOffKb);
      sc.va = reinterpret_cast<uint32_t*>(base + kOffVa);
      sc.vb = reinterpret_cast<uint32_t*>(base + kOffVb);
      sc.sort_scratch = reinterpret_cast<uint32_t*>(base + kOffSort);
      sc.pos = reinterpret_cast<uint32_t*>(base + kOffPos);
      sc.uv = reinterpret_cast<uint64_t*>(base + kOffUv);
      sc.tot = reinterpret_cast<uint32_t*>(base + kOffTot);
      sc.cap = kStaticMaxKeys;
      cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
      // the scan total is the only word read before it is written in this call;
      // clear it so nothing from an earlier call can leak in
      if (cudaMemsetAsync(sc.tot, 0, 256, s) != cudaSuccess) rc = BT_ERR_CUDA;
      else {
        H->h.L.valid = false;
        rc = map_rc(bt::tree_bulk_build_scratch(&H->h, keys, vals, n, s, sc));
      }
    }
  }
  if (prev != dev) cudaSetDevice(prev);
  return rc;
}
