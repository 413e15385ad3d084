// Device-side layout and helpers for the B200 B+tree.
//
// Node pool (structure of arrays, like the reference's g_key_section /
// g_val_section, src/gpu-stm-tree-v39/bpt-gpustm.h:41-60, widened to uint64):
//   keys[node*32 + i], i < 31 : sorted keys, padding BT_KEY_MAX
//   keys[node*32 + 31]         : header word (size, level, lock, version)
//   vals[node*32 + i]          : leaf values / inner child ids
//   vals[node*32 + 31]         : leaf right fence (min key of the right sibling)
//   low[node]                  : low fence, written once when the node is created
// One node row is 256 B of keys (two 128 B lines) and 256 B of values.
//
// The header replaces the reference's side lock table (g_lock_table,
// src/gpu-stm-tree-v39/bpt-gpustm-kernel-tx.cuh:16-18): the version lives in
// the same word a reader loads with the keys, so the seqlock costs no extra
// sector per level.
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

namespace bt {

constexpr int kOrder = 32;
constexpr int kMaxKeys = 31;
constexpr uint64_t kKeyMax = ~0ull;
constexpr uint32_t kNil = 0xFFFFFFFFu;

constexpr uint8_t kOpInsert = 0;  // src/input-helper.h:14
constexpr uint8_t kOpGet = 1;     // src/input-helper.h:15
constexpr uint8_t kOpDelete = 2;  // src/input-helper.h:16 (declared there, implemented by no reference version)

// per-request status byte
constexpr uint8_t kAbsent = 0;
constexpr uint8_t kFound = 1;
constexpr uint8_t kRejected = 2;
constexpr uint8_t kRetryExhausted = 3;
constexpr uint8_t kNoCapacity = 4;

// sticky device error bits (Ctrl::error)
constexpr uint32_t kErrCapacity = 1u;
constexpr uint32_t kErrRetry = 2u;
constexpr uint32_t kErrSpin = 4u;

// ---- header word ----------------------------------------------------------
// bits 0..7 level (0 = leaf), 8..15 size, 16 lock, 17..31 tree epoch,
// 32..63 version.  The epoch changes with every bulk build; a reader that
// reaches a node without validating the path rejects a header from another
// epoch (a node row left over from an earlier tree, or never written: the pool
// is zeroed at creation and epochs start at 1).
__host__ __device__ __forceinline__ uint32_t hdr_level(uint64_t h) { return (uint32_t)(h & 0xff); }
__host__ __device__ __forceinline__ uint32_t hdr_size(uint64_t h) { return (uint32_t)((h >> 8) & 0xff); }
__host__ __device__ __forceinline__ bool hdr_locked(uint64_t h) { return (h >> 16) & 1; }
__host__ __device__ __forceinline__ uint32_t hdr_epoch(uint64_t h) { return (uint32_t)((h >> 17) & 0x7fff); }
__host__ __device__ __forceinline__ uint32_t hdr_version(uint64_t h) { return (uint32_t)(h >> 32); }
__host__ __device__ __forceinline__ uint64_t make_hdr(uint32_t size, uint32_t level, uint32_t version,
                                                      uint32_t epoch) {
  return ((uint64_t)version << 32) | ((uint64_t)(epoch & 0x7fff) << 17) | ((uint64_t)size << 8) | (uint64_t)level;
}
// next version of an unlocked header with a new size (level and epoch kept)
__host__ __device__ __forceinline__ uint64_t hdr_next(uint64_t h, uint32_t size) {
  return make_hdr(size, hdr_level(h), hdr_version(h) + 1, hdr_epoch(h));
}
__host__ __device__ __forceinline__ uint64_t hdr_lock(uint64_t h) { return h | (1ull << 16); }

// ---- tree control block (device memory) -----------------------------------
struct Ctrl {
  uint32_t root;       // kNil when empty
  uint32_t root_lock;  // version << 1 | lock  (reference: g_lock_table[MAX_NODE_NUM-1])
  uint32_t n_nodes;    // bump allocator
  uint32_t error;      // sticky kErr* bits
  uint32_t root_level; // level of the root node (0 = the root is a leaf)
  uint32_t epoch;      // current tree epoch (header bits 17..31)
  unsigned long long n_keys;
  unsigned long long commits;
  unsigned long long aborts;
  unsigned long long leaf_splits;
  unsigned long long inner_splits;
  unsigned long long new_roots;
  unsigned long long retry_exhausted;
  unsigned long long learned_hits;
  unsigned long long learned_fallbacks;
  unsigned long long learned_probe_sum;
};

struct DevTree {
  uint64_t* keys;
  uint64_t* vals;
  uint64_t* low;
  Ctrl* ctrl;
  uint32_t cap;  // node capacity
  // [cap][32] high 32 bits of an inner node's separators (slot 31 unused):
  // the batch lookups compare these first and read the full keys of a row
  // only when a prefix equals the key's.  Kept by the merge engine's inner
  // merge; rebuilt from the rows after other writers (Handle::pfx_valid).
  uint32_t* pfx;
};

// ---- memory-order helpers --------------------------------------------------
__device__ __forceinline__ uint64_t ld_acquire(const uint64_t* p) {
  uint64_t v;
  asm volatile("ld.acquire.gpu.global.u64 %0, [%1];" : "=l"(v) : "l"(p) : "memory");
  return v;
}
__device__ __forceinline__ uint64_t ld_relaxed(const uint64_t* p) {
  uint64_t v;
  asm volatile("ld.relaxed.gpu.global.u64 %0, [%1];" : "=l"(v) : "l"(p) : "memory");
  return v;
}
__device__ __forceinline__ uint32_t ld_acquire32(const uint32_t* p) {
  uint32_t v;
  asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}
__device__ __forceinline__ void st_relaxed32(uint32_t* p, uint32_t v) {
  asm volatile("st.relaxed.gpu.global.u32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}
__device__ __forceinline__ uint32_t ld_relaxed32(const uint32_t* p) {
  uint32_t v;
  asm volatile("ld.relaxed.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}
__device__ __forceinline__ void st_release(uint64_t* p, uint64_t v) {
  asm volatile("st.release.gpu.global.u64 [%0], %1;" ::"l"(p), "l"(v) : "memory");
}
__device__ __forceinline__ void st_release32(uint32_t* p, uint32_t v) {
  asm volatile("st.release.gpu.global.u32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}
__device__ __forceinline__ void st_relaxed(uint64_t* p, uint64_t v) {
  asm volatile("st.relaxed.gpu.global.u64 [%0], %1;" ::"l"(p), "l"(v) : "memory");
}
__device__ __forceinline__ void fence_acq_rel() { asm volatile("fence.acq_rel.gpu;" ::: "memory"); }

__device__ __forceinline__ uint32_t lane_id() { return threadIdx.x & 31; }

}  // namespace bt
