// Snapshot of a tree's contents to a file and back (checkpoint / resume).
// The reference has no counterpart: its tree lives only as long as the
// process (src/gpu-stm-tree-v39/bpt-gpustm.h:145).
//
// The snapshot is logical: the sorted (key, value) pairs, not the node pool.
// Loading bulk-builds them with the loading handle's fill settings, so the
// loaded tree has the same contents and answers every request the same way,
// but its leaf layout is a fresh bulk load, not the saved one.
//
// File layout (little endian):
//   0   8 B  magic "EIRB2SNP"
//   8   4 B  format version (1)
//   12  4 B  0
//   16  8 B  n, the number of pairs
//   24  8 B  FNV-1a 64 over the key and value arrays
//   32  8n B keys, ascending
//   ... 8n B values
#include <cstdio>
#include <cstring>
#include <vector>

#include <cuda_runtime.h>

#include "../../include/eirene_b200.h"
#include "bt_internal.h"

namespace {

constexpr char kMagic[8] = {'E', 'I', 'R', 'B', '2', 'S', 'N', 'P'};
constexpr uint32_t kVersion = 1;
constexpr char kImgMagic[8] = {'E', 'I', 'R', 'B', '2', 'I', 'M', 'G'};
constexpr uint32_t kImgVersion = 2;

uint64_t fnv1a(const void* p, size_t bytes, uint64_t h) {
  const unsigned char* b = static_cast<const unsigned char*>(p);
  for (size_t i = 0; i < bytes; i++) {
    h ^= b[i];
    h *= 0x100000001B3ull;
  }
  return h;
}

struct DevBuf {
  void* p = nullptr;
  ~DevBuf() {
    if (p) cudaFree(p);
  }
};

}  // namespace

extern "C" {

int bt_save(bt_handle* h, const char* path) {
  if (!h || !path) return BT_ERR_INVALID_ARG;
  uint64_t n = 0;
  int rc = bt_size(h, &n);
  if (rc != BT_OK) return rc;
  int prev = -1;
  cudaGetDevice(&prev);
  cudaSetDevice(h->h.device);
  h->h.chain_open = false;
  std::vector<uint64_t> keys(n), vals(n);
  if (n) {
    DevBuf dk, dv;  // freed with the handle's device current
    size_t got = 0;
    if (cudaMalloc(&dk.p, n * 8) != cudaSuccess || cudaMalloc(&dv.p, n * 8) != cudaSuccess) rc = BT_ERR_NO_MEMORY;
    if (rc == BT_OK) rc = bt_dump_sorted(h, (uint64_t*)dk.p, (uint64_t*)dv.p, n, &got, nullptr);
    if (rc == BT_OK && got != n) rc = BT_ERR_CUDA;
    if (rc == BT_OK && (cudaMemcpy(keys.data(), dk.p, n * 8, cudaMemcpyDeviceToHost) != cudaSuccess ||
                        cudaMemcpy(vals.data(), dv.p, n * 8, cudaMemcpyDeviceToHost) != cudaSuccess))
      rc = BT_ERR_CUDA;
  }
  if (prev >= 0) cudaSetDevice(prev);
  if (rc != BT_OK) return rc;
  uint64_t sum = fnv1a(keys.data(), n * 8, 0xCBF29CE484222325ull);
  sum = fnv1a(vals.data(), n * 8, sum);
  FILE* f = std::fopen(path, "wb");
  if (!f) return BT_ERR_IO;
  const uint32_t ver[2] = {kVersion, 0};
  bool ok = std::fwrite(kMagic, 1, 8, f) == 8 && std::fwrite(ver, 4, 2, f) == 2 && std::fwrite(&n, 8, 1, f) == 1 &&
            std::fwrite(&sum, 8, 1, f) == 1 && (n == 0 || (std::fwrite(keys.data(), 8, n, f) == n &&
                                                           std::fwrite(vals.data(), 8, n, f) == n));
  ok = (std::fclose(f) == 0) && ok;
  return ok ? BT_OK : BT_ERR_IO;
}

int bt_load(bt_handle* h, const char* path) {
  if (!h || !path) return BT_ERR_INVALID_ARG;
  FILE* f = std::fopen(path, "rb");
  if (!f) return BT_ERR_IO;
  char magic[8];
  uint32_t ver[2];
  uint64_t n = 0, sum = 0;
  bool ok = std::fread(magic, 1, 8, f) == 8 && std::memcmp(magic, kMagic, 8) == 0 && std::fread(ver, 4, 2, f) == 2 &&
            ver[0] == kVersion && std::fread(&n, 8, 1, f) == 1 && std::fread(&sum, 8, 1, f) == 1;
  // the pairs must fit the file that holds them
  long here = ok ? std::ftell(f) : -1;
  if (ok && std::fseek(f, 0, SEEK_END) == 0) {
    const long end = std::ftell(f);
    ok = here >= 0 && end >= here && (uint64_t)(end - here) == n * 16 && std::fseek(f, here, SEEK_SET) == 0;
  } else {
    ok = false;
  }
  std::vector<uint64_t> keys, vals;
  if (ok) {
    keys.resize(n);
    vals.resize(n);
    ok = n == 0 || (std::fread(keys.data(), 8, n, f) == n && std::fread(vals.data(), 8, n, f) == n);
  }
  std::fclose(f);
  if (!ok) return BT_ERR_IO;
  uint64_t chk = fnv1a(keys.data(), n * 8, 0xCBF29CE484222325ull);
  chk = fnv1a(vals.data(), n * 8, chk);
  if (chk != sum) return BT_ERR_IO;
  for (uint64_t i = 1; i < n; i++)
    if (keys[i] <= keys[i - 1]) return BT_ERR_IO;  // not strictly ascending: not a snapshot of a tree
  int prev = -1;
  cudaGetDevice(&prev);
  cudaSetDevice(h->h.device);
  h->h.chain_open = false;
  int rc = BT_OK;
  {
    DevBuf dk, dv;  // freed with the handle's device current
    if (n && (cudaMalloc(&dk.p, n * 8) != cudaSuccess || cudaMalloc(&dv.p, n * 8) != cudaSuccess))
      rc = BT_ERR_NO_MEMORY;
    if (rc == BT_OK && n &&
        (cudaMemcpy(dk.p, keys.data(), n * 8, cudaMemcpyHostToDevice) != cudaSuccess ||
         cudaMemcpy(dv.p, vals.data(), n * 8, cudaMemcpyHostToDevice) != cudaSuccess))
      rc = BT_ERR_CUDA;
    if (rc == BT_OK) rc = bt_bulk_build(h, (const uint64_t*)dk.p, (const uint64_t*)dv.p, n, nullptr);
  }
  if (prev >= 0) cudaSetDevice(prev);
  return rc;
}

// Pool image: the node pool itself (the rows of every allocated node, their
// low fences and the control block), so a loaded tree keeps the saved leaf
// layout and goes on exactly as the saved one would (the merge engine is
// deterministic).  The loading handle needs a pool of at least n_nodes
// nodes and the saving handle's leaf and inner fills (later splits follow
// them); its learned model and separator prefixes are rebuilt on demand.
//
// File layout (little endian):
//   0   8 B  magic "EIRB2IMG"
//   8   4 B  format version (2)
//   12  4 B  sizeof(Ctrl)
//   16  8 B  n_nodes
//   24  8 B  FNV-1a 64 over the fills, control block, key rows, value rows, lows
//   32  4 B  leaf fill, 4 B inner fill
//   40       control block
//   ...      n_nodes key rows (256 B), n_nodes value rows, n_nodes low fences (8 B)
int bt_save_image(bt_handle* h, const char* path) {
  if (!h || !path) return BT_ERR_INVALID_ARG;
  bt::Handle& H = h->h;
  int prev = -1;
  cudaGetDevice(&prev);
  cudaSetDevice(H.device);
  H.chain_open = false;
  int rc = BT_OK;
  bt::Ctrl c{};
  std::vector<uint64_t> keys, vals, low;
  uint64_t nn = 0;
  if (cudaDeviceSynchronize() != cudaSuccess || bt::tree_sync(&H) != cudaSuccess ||
      cudaMemcpy(&c, H.tree.ctrl, sizeof(c), cudaMemcpyDeviceToHost) != cudaSuccess) {
    rc = BT_ERR_CUDA;
  } else {
    nn = c.n_nodes < H.tree.cap ? c.n_nodes : H.tree.cap;
    keys.resize(nn * 32);
    vals.resize(nn * 32);
    low.resize(nn);
    if (nn && (cudaMemcpy(keys.data(), H.tree.keys, nn * 256, cudaMemcpyDeviceToHost) != cudaSuccess ||
               cudaMemcpy(vals.data(), H.tree.vals, nn * 256, cudaMemcpyDeviceToHost) != cudaSuccess ||
               cudaMemcpy(low.data(), H.tree.low, nn * 8, cudaMemcpyDeviceToHost) != cudaSuccess))
      rc = BT_ERR_CUDA;
  }
  if (prev >= 0) cudaSetDevice(prev);
  if (rc != BT_OK) return rc;
  const uint32_t fills[2] = {H.leaf_fill, H.inner_fill};
  uint64_t sum = fnv1a(fills, sizeof(fills), 0xCBF29CE484222325ull);
  sum = fnv1a(&c, sizeof(c), sum);
  sum = fnv1a(keys.data(), nn * 256, sum);
  sum = fnv1a(vals.data(), nn * 256, sum);
  sum = fnv1a(low.data(), nn * 8, sum);
  FILE* f = std::fopen(path, "wb");
  if (!f) return BT_ERR_IO;
  const uint32_t ver[2] = {kImgVersion, (uint32_t)sizeof(c)};
  bool ok = std::fwrite(kImgMagic, 1, 8, f) == 8 && std::fwrite(ver, 4, 2, f) == 2 &&
            std::fwrite(&nn, 8, 1, f) == 1 && std::fwrite(&sum, 8, 1, f) == 1 && std::fwrite(fills, 4, 2, f) == 2 &&
            std::fwrite(&c, sizeof(c), 1, f) == 1 &&
            (nn == 0 || (std::fwrite(keys.data(), 256, nn, f) == nn && std::fwrite(vals.data(), 256, nn, f) == nn &&
                         std::fwrite(low.data(), 8, nn, f) == nn));
  ok = (std::fclose(f) == 0) && ok;
  return ok ? BT_OK : BT_ERR_IO;
}

int bt_load_image(bt_handle* h, const char* path) {
  if (!h || !path) return BT_ERR_INVALID_ARG;
  bt::Handle& H = h->h;
  FILE* f = std::fopen(path, "rb");
  if (!f) return BT_ERR_IO;
  char magic[8];
  uint32_t ver[2];
  uint64_t nn = 0, sum = 0;
  uint32_t fills[2] = {0, 0};
  bt::Ctrl c{};
  bool ok = std::fread(magic, 1, 8, f) == 8 && std::memcmp(magic, kImgMagic, 8) == 0 && std::fread(ver, 4, 2, f) == 2 &&
            ver[0] == kImgVersion && ver[1] == sizeof(c) && std::fread(&nn, 8, 1, f) == 1 &&
            std::fread(&sum, 8, 1, f) == 1 && std::fread(fills, 4, 2, f) == 2 && std::fread(&c, sizeof(c), 1, f) == 1;
  // the rows must fill the rest of the file exactly
  long here = ok ? std::ftell(f) : -1;
  if (ok && std::fseek(f, 0, SEEK_END) == 0) {
    const long end = std::ftell(f);
    ok = here >= 0 && end >= here && (uint64_t)(end - here) == nn * 520 && std::fseek(f, here, SEEK_SET) == 0;
  } else {
    ok = false;
  }
  std::vector<uint64_t> keys, vals, low;
  if (ok) {
    keys.resize(nn * 32);
    vals.resize(nn * 32);
    low.resize(nn);
    ok = nn == 0 || (std::fread(keys.data(), 256, nn, f) == nn && std::fread(vals.data(), 256, nn, f) == nn &&
                     std::fread(low.data(), 8, nn, f) == nn);
  }
  std::fclose(f);
  if (!ok) return BT_ERR_IO;
  uint64_t chk = fnv1a(fills, sizeof(fills), 0xCBF29CE484222325ull);
  chk = fnv1a(&c, sizeof(c), chk);
  chk = fnv1a(keys.data(), nn * 256, chk);
  chk = fnv1a(vals.data(), nn * 256, chk);
  chk = fnv1a(low.data(), nn * 8, chk);
  if (chk != sum || c.n_nodes != nn || (c.root != bt::kNil && c.root >= nn) || c.epoch == 0 || c.epoch > 0x7fffu)
    return BT_ERR_IO;
  if (nn > H.tree.cap) return BT_ERR_NO_MEMORY;  // the pool cannot hold the saved nodes
  // later splits follow the fills: a handle with other fills would not go on as the saved one
  if (fills[0] != H.leaf_fill || fills[1] != H.inner_fill) return BT_ERR_INVALID_ARG;
  int prev = -1;
  cudaGetDevice(&prev);
  cudaSetDevice(H.device);
  H.chain_open = false;
  int rc = BT_OK;
  c.root_lock &= ~1u;  // saved at rest: unlocked
  // the loading handle starts with its own record: no sticky error bits or
  // counters of the saving one (the key count is the tree's)
  c.error = 0;
  c.commits = c.aborts = c.leaf_splits = c.inner_splits = c.new_roots = c.retry_exhausted = 0;
  c.learned_hits = c.learned_fallbacks = c.learned_probe_sum = 0;
  if (cudaDeviceSynchronize() != cudaSuccess || bt::tree_sync(&H) != cudaSuccess ||
      (nn && (cudaMemcpy(H.tree.keys, keys.data(), nn * 256, cudaMemcpyHostToDevice) != cudaSuccess ||
              cudaMemcpy(H.tree.vals, vals.data(), nn * 256, cudaMemcpyHostToDevice) != cudaSuccess ||
              cudaMemcpy(H.tree.low, low.data(), nn * 8, cudaMemcpyHostToDevice) != cudaSuccess)) ||
      cudaMemcpy(H.tree.ctrl, &c, sizeof(c), cudaMemcpyHostToDevice) != cudaSuccess)
    rc = BT_ERR_CUDA;
  // rows past the loaded ones may hold an earlier tree's nodes; clear their
  // headers (epoch 0, never used) so that none can pass for a row of this tree
  if (rc == BT_OK && (bt::clear_headers(&H, (uint32_t)nn, H.tree.cap, H.internal_stream) != cudaSuccess ||
                      cudaStreamSynchronize(H.internal_stream) != cudaSuccess))
    rc = BT_ERR_CUDA;
  if (rc == BT_OK) {
    H.epoch = c.epoch;  // the rows carry the saved tree's epoch
    H.L.valid = false;
    H.pfx_valid = false;
  }
  if (prev >= 0) cudaSetDevice(prev);
  return rc;
}

}  // extern "C"
