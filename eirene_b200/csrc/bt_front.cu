// Hash front end of the sorted-merge batch (the v38 meaning,
// src/gpu-stm-tree-v38/bpt-gpustm-kernel-aux.cuh:16-56).
//
// The meaning only couples requests whose key is written (INSERT or DELETE)
// somewhere in the batch: a request for a key with no write in the batch, or
// one that comes before the first write of its key, sees the pre-batch tree.  So instead
// of sorting the whole batch, the front end
//
//   1. counts the write requests and sizes an open-addressing table for
//      their keys (a power of two >= 4x the count, at least 1024 slots:
//      most lookups ask for a key the table does not hold, and a linear probe
//      for an absent key runs about (1 + 1/(1-a)^2)/2 slots at load a: 1.4
//      at a = 1/4, 5 at a = 2/3),
//   2. records, per written key, the index of its first write,
//   3. classifies every request: "touched" if its op code is invalid or its
//      key has a write at or before it; otherwise it is a plain lookup,
//      and compacts both classes in input order (a flag pass, a scan of
//      the per-tile counts, a scatter pass).
//
// The touched requests go through the sort + segmented-scan path (their
// runs all start with a write, so the pre-batch value reaches them from the
// delete or insert phase, which return each key's previous value); the plain lookups
// run on the pre-batch tree, unsorted, writing their answers in place.  For a
// read-mostly batch the sort shrinks to the INSERTs.
//
// HBM traffic per request: count (1 B op), table insert (1 B op, plus the key
// of a write), flag (8 B key + 1 B op + the probe, which is L2-resident for
// small write counts, then a 1 B flag), scatter (1 B flag, then a 4 B list
// entry, or 9 B read and a 12 B touched entry).
#include <cuda_runtime.h>

#include "bt_block.cuh"
#include "bt_common.cuh"
#include "bt_internal.h"

namespace bt {

namespace {

constexpr uint32_t kNone = 0xFFFFFFFFu;
constexpr int kThreads = 256;

struct Slot {
  unsigned long long key;  // kKeyMax = empty
  uint32_t first;          // index of the first INSERT of the key
  uint32_t pad;
};

// SplitMix64's finaliser (Steele, Lea, Flood 2014) as the slot hash
__device__ __forceinline__ uint64_t slot_hash(uint64_t x) {
  x ^= x >> 30;
  x *= 0xBF58476D1CE4E5B9ull;
  x ^= x >> 27;
  x *= 0x94D049BB133111EBull;
  return x ^ (x >> 31);
}

// INSERT or DELETE: the requests that couple the others of their key
__device__ __forceinline__ uint32_t is_write(uint8_t op) { return (op == kOpInsert || op == kOpDelete) ? 1u : 0u; }

__device__ __forceinline__ uint32_t table_cap(uint32_t n_ins, size_t cap_max) {
  uint64_t c = 1024;
  while (c < 4ull * n_ins) c <<= 1;  // load factor at most 1/4 (up to the allocation)
  return (uint32_t)(c < cap_max ? c : cap_max);
}

// INSERT and DELETE op codes (an upper bound of the keys to hold: reserved keys count too)
__global__ void __launch_bounds__(kThreads) front_count_kernel(const uint8_t* __restrict__ ops, size_t n,
                                                               BatchCounts* __restrict__ counts) {
  uint32_t c = 0;
  // four op codes per load when the array is 4-byte aligned
  const size_t n4 = ((uintptr_t)ops & 3u) ? 0 : n / 4;
  const uchar4* o4 = reinterpret_cast<const uchar4*>(ops);
  for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n4; i += (size_t)gridDim.x * blockDim.x) {
    const uchar4 o = o4[i];
    c += is_write(o.x) + is_write(o.y) + is_write(o.z) + is_write(o.w);
  }
  for (size_t i = n4 * 4 + (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x)
    c += is_write(ops[i]);
  c = __reduce_add_sync(0xffffffffu, c);
  if ((threadIdx.x & 31) == 0 && c) atomicAdd(&counts->n_ins_req, c);
}

__global__ void __launch_bounds__(kThreads) front_clear_kernel(Slot* __restrict__ tab, size_t cap_max,
                                                               BatchCounts* __restrict__ counts) {
  const uint32_t cap = table_cap(counts->n_ins_req, cap_max);
  if (blockIdx.x == 0 && threadIdx.x == 0) counts->cap = cap;
  for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < cap; i += (size_t)gridDim.x * blockDim.x) {
    tab[i].key = kKeyMax;
    tab[i].first = kNone;
    tab[i].pad = 0;
  }
}

// linear probing; the table holds at most 2/3 of its slots, so a probe ends
__global__ void __launch_bounds__(kThreads) front_insert_kernel(const uint64_t* __restrict__ keys,
                                                                const uint8_t* __restrict__ ops, size_t n,
                                                                Slot* __restrict__ tab,
                                                                const BatchCounts* __restrict__ counts) {
  const uint32_t mask = counts->cap - 1;
  auto put = [&](size_t i) {
    const uint64_t k = keys[i];
    if (k == kKeyMax) return;
    uint32_t h = (uint32_t)slot_hash(k) & mask;
    for (uint32_t probe = 0; probe <= mask; probe++) {
      const unsigned long long prev = atomicCAS(&tab[h].key, (unsigned long long)kKeyMax, (unsigned long long)k);
      if (prev == kKeyMax || prev == k) {
        atomicMin(&tab[h].first, (uint32_t)i);
        return;
      }
      h = (h + 1) & mask;
    }
  };
  // four op codes per load when the array is 4-byte aligned
  const size_t n4 = ((uintptr_t)ops & 3u) ? 0 : n / 4;
  const uchar4* o4 = reinterpret_cast<const uchar4*>(ops);
  for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n4; i += (size_t)gridDim.x * blockDim.x) {
    const uchar4 o = o4[i];
    if (is_write(o.x)) put(4 * i);
    if (is_write(o.y)) put(4 * i + 1);
    if (is_write(o.z)) put(4 * i + 2);
    if (is_write(o.w)) put(4 * i + 3);
  }
  for (size_t i = n4 * 4 + (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x)
    if (is_write(ops[i])) put(i);
}

// Classify, then compact, in three launches over tiles of kTile requests:
//   front_flag_kernel     one flag byte per request ("touched": invalid op
//                         code, or its key has a write at or before it) and
//                         the touched count of each tile;
//   front_tile_scan_kernel  exclusive offsets of the tiles (one block) and
//                         the two class counts;
//   front_scatter_kernel  touched requests to (tk, tv), the rest to list and
//                         their keys to lk, both in input order.
// Every launch is fully parallel (no look-back chain between tiles): the
// probes of the flag pass are its only dependent loads, and the scatter
// reads the request's key and op again only when it is touched.
constexpr int kTileThreads = 256;
constexpr int kTileItems = 8;
constexpr int kTile = kTileThreads * kTileItems;  // 2048
constexpr int kTileWarps = kTileThreads / 32;

__global__ void __launch_bounds__(kTileThreads) front_flag_kernel(const uint64_t* __restrict__ keys,
                                                                  const uint8_t* __restrict__ ops, size_t n,
                                                                  const Slot* __restrict__ tab,
                                                                  const BatchCounts* __restrict__ counts,
                                                                  uint8_t* __restrict__ flags,
                                                                  uint32_t* __restrict__ tile_cnt) {
  __shared__ uint32_t wsum[kTileWarps];
  const uint32_t mask = counts->cap - 1;
  const bool any = counts->n_ins_req != 0;
  const size_t base = (size_t)blockIdx.x * kTile;
  uint64_t k[kTileItems];
  uint8_t op[kTileItems];
  uint64_t sk[kTileItems];
  uint32_t sf[kTileItems], sh[kTileItems];
  // loads first, then every item's first probe slot (independent loads in
  // flight), then the rare longer probes
#pragma unroll
  for (int j = 0; j < kTileItems; j++) {
    const size_t i = base + (size_t)j * kTileThreads + threadIdx.x;
    k[j] = i < n ? keys[i] : kKeyMax;
    op[j] = i < n ? ops[i] : 0;
  }
#pragma unroll
  for (int j = 0; j < kTileItems; j++) {
    sh[j] = (uint32_t)slot_hash(k[j]) & mask;
    sk[j] = kKeyMax;
    sf[j] = kNone;
    if (any && k[j] != kKeyMax) {
      const ulonglong2 e = __ldg(reinterpret_cast<const ulonglong2*>(tab + sh[j]));
      sk[j] = e.x;
      sf[j] = (uint32_t)e.y;
    }
  }
  // the longer probes, all of this thread's unresolved items one slot per
  // round (their loads in flight together), instead of item after item
  uint32_t first[kTileItems];
  uint32_t todo = 0;
#pragma unroll
  for (int j = 0; j < kTileItems; j++) {
    first[j] = kNone;
    if (sk[j] == k[j] && k[j] != kKeyMax) first[j] = sf[j];
    else if (sk[j] != kKeyMax) todo |= 1u << j;
  }
  for (uint32_t probe = 0; todo && probe < mask; probe++) {
#pragma unroll
    for (int j = 0; j < kTileItems; j++) {
      if (!((todo >> j) & 1u)) continue;
      sh[j] = (sh[j] + 1) & mask;
      const ulonglong2 e = __ldg(reinterpret_cast<const ulonglong2*>(tab + sh[j]));
      sk[j] = e.x;
      sf[j] = (uint32_t)e.y;
    }
#pragma unroll
    for (int j = 0; j < kTileItems; j++) {
      if (!((todo >> j) & 1u)) continue;
      if (sk[j] == k[j]) {
        first[j] = sf[j];
        todo &= ~(1u << j);
      } else if (sk[j] == kKeyMax) {
        todo &= ~(1u << j);
      }
    }
  }
  uint32_t c = 0;
#pragma unroll
  for (int j = 0; j < kTileItems; j++) {
    const size_t i = base + (size_t)j * kTileThreads + threadIdx.x;
    if (i < n) {
      bool f = op[j] > 2;  // invalid op codes are rejected on the sorted path
      if (!f && any && k[j] != kKeyMax) f = first[j] != kNone && (uint32_t)i >= first[j];
      flags[i] = f ? 1 : 0;
      c += f ? 1u : 0u;
    }
  }
  c = __reduce_add_sync(0xffffffffu, c);
  if ((threadIdx.x & 31) == 0) wsum[threadIdx.x >> 5] = c;
  __syncthreads();
  if (threadIdx.x == 0) {
    uint32_t t = 0;
#pragma unroll
    for (int w = 0; w < kTileWarps; w++) t += wsum[w];
    tile_cnt[blockIdx.x] = t;
  }
}

// exclusive offsets of n_tiles counts, in place, with one block
__global__ void __launch_bounds__(1024) front_tile_scan_kernel(uint32_t* __restrict__ tile, uint32_t n_tiles,
                                                               size_t n, BatchCounts* __restrict__ counts,
                                                               uint32_t* hint) {
  __shared__ uint32_t wtot[32];
  const uint32_t lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  uint32_t carry = 0;
  for (uint32_t b = 0; b < n_tiles; b += 1024) {
    const uint32_t i = b + threadIdx.x;
    const uint32_t v = i < n_tiles ? tile[i] : 0u;
    uint32_t incl = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const uint32_t y = __shfl_up_sync(0xffffffffu, incl, o);
      if (lane >= (uint32_t)o) incl += y;
    }
    if (lane == 31) wtot[warp] = incl;
    __syncthreads();
    if (warp == 0) {
      uint32_t t = wtot[lane];
#pragma unroll
      for (int o = 1; o < 32; o <<= 1) {
        const uint32_t y = __shfl_up_sync(0xffffffffu, t, o);
        if (lane >= (uint32_t)o) t += y;
      }
      wtot[lane] = t;  // inclusive over warps
    }
    __syncthreads();
    const uint32_t before = warp ? wtot[warp - 1] : 0u;
    if (i < n_tiles) tile[i] = carry + before + incl - v;
    carry += wtot[31];
    __syncthreads();  // wtot is reused by the next chunk
  }
  if (threadIdx.x == 0) {
    counts->n_touch = carry;
    counts->n_lookup = (uint32_t)n - carry;
    if (hint) *reinterpret_cast<volatile uint32_t*>(hint) = carry;  // host memory: a later batch's sort choice
  }
}

__global__ void __launch_bounds__(kTileThreads) front_scatter_kernel(const uint64_t* __restrict__ keys,
                                                                     const uint8_t* __restrict__ ops, size_t n,
                                                                     const uint8_t* __restrict__ flags,
                                                                     const uint32_t* __restrict__ tile_off,
                                                                     uint64_t* __restrict__ tk,
                                                                     uint32_t* __restrict__ tv,
                                                                     uint32_t* __restrict__ list,
                                                                     uint64_t* __restrict__ lk) {
  __shared__ uint32_t cnt[kTileItems][kTileWarps];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const uint32_t lt = (1u << lane) - 1u;
  const size_t base = (size_t)blockIdx.x * kTile;
  uint32_t bal[kTileItems];
#pragma unroll
  for (int j = 0; j < kTileItems; j++) {
    const size_t i = base + (size_t)j * kTileThreads + threadIdx.x;
    bal[j] = __ballot_sync(0xffffffffu, i < n && flags[i] != 0);
    if (lane == 0) cnt[j][warp] = __popc(bal[j]);
  }
  __syncthreads();
  // exclusive prefix over (item, warp) in index order
  if (warp == 0) {
    uint32_t carry = 0;
#pragma unroll
    for (int j = 0; j < kTileItems; j++) {
      const uint32_t c = lane < kTileWarps ? cnt[j][lane] : 0u;
      uint32_t incl = c;
#pragma unroll
      for (int o = 1; o < kTileWarps; o <<= 1) {
        const uint32_t y = __shfl_up_sync(0xffffffffu, incl, o);
        if (lane >= o) incl += y;
      }
      if (lane < kTileWarps) cnt[j][lane] = carry + incl - c;
      carry += __shfl_sync(0xffffffffu, incl, kTileWarps - 1);
    }
  }
  __syncthreads();
  const uint32_t excl = tile_off[blockIdx.x];
#pragma unroll
  for (int j = 0; j < kTileItems; j++) {
    const size_t i = base + (size_t)j * kTileThreads + threadIdx.x;
    if (i < n) {
      const uint32_t p = excl + cnt[j][warp] + __popc(bal[j] & lt);  // touched before i
      const uint64_t k = keys[i];
      if ((bal[j] >> lane) & 1u) {
        const uint8_t op = ops[i];
        tk[p] = k;
        tv[p] = (uint32_t)i | ((op <= 2 ? (uint32_t)op : 3u) << 30);
      } else {
        list[i - p] = (uint32_t)i;
        lk[i - p] = k;
      }
    }
  }
}

// Packed INSERT values (bt_execute_batch_host_packed_async): the caller sends
// the values of the batch's INSERTs only, in request order.  Value j belongs
// to the j-th INSERT; two launches around a scan of the per-tile INSERT
// counts put it at that request's slot, so the batch reads vals[r] as usual.
// HBM traffic per request: 2 B of op codes (read twice), plus 16 B per INSERT.
__device__ __forceinline__ uint32_t tile_ballot(const uint8_t* __restrict__ ops, size_t n, size_t i) {
  return __ballot_sync(0xffffffffu, i < n && ops[i] == kOpInsert);
}

__global__ void __launch_bounds__(kTileThreads) pack_count_kernel(const uint8_t* __restrict__ ops, size_t n,
                                                                  uint32_t* __restrict__ tile_cnt) {
  __shared__ uint32_t wsum[kTileWarps];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const size_t base = (size_t)blockIdx.x * kTile;
  uint32_t c = 0;
#pragma unroll
  for (int j = 0; j < kTileItems; j++) c += __popc(tile_ballot(ops, n, base + (size_t)j * kTileThreads + threadIdx.x));
  if (lane == 0) wsum[warp] = c;
  __syncthreads();
  if (warp == 0) {
    uint32_t v = lane < kTileWarps ? wsum[lane] : 0u;
    v = __reduce_add_sync(0xffffffffu, v);
    if (lane == 0) tile_cnt[blockIdx.x] = v;
  }
}

__global__ void __launch_bounds__(kTileThreads) pack_expand_kernel(const uint8_t* __restrict__ ops, size_t n,
                                                                   const uint32_t* __restrict__ tile_off,
                                                                   const uint64_t* __restrict__ packed,
                                                                   size_t n_packed, uint64_t* __restrict__ vals) {
  __shared__ uint32_t cnt[kTileItems][kTileWarps];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const uint32_t lt = (1u << lane) - 1u;
  const size_t base = (size_t)blockIdx.x * kTile;
  uint32_t bal[kTileItems];
#pragma unroll
  for (int j = 0; j < kTileItems; j++) {
    bal[j] = tile_ballot(ops, n, base + (size_t)j * kTileThreads + threadIdx.x);
    if (lane == 0) cnt[j][warp] = __popc(bal[j]);
  }
  __syncthreads();
  // exclusive prefix over (item, warp) in index order
  if (warp == 0) {
    uint32_t carry = 0;
#pragma unroll
    for (int j = 0; j < kTileItems; j++) {
      const uint32_t c = lane < kTileWarps ? cnt[j][lane] : 0u;
      uint32_t incl = c;
#pragma unroll
      for (int o = 1; o < kTileWarps; o <<= 1) {
        const uint32_t y = __shfl_up_sync(0xffffffffu, incl, o);
        if (lane >= o) incl += y;
      }
      if (lane < kTileWarps) cnt[j][lane] = carry + incl - c;
      carry += __shfl_sync(0xffffffffu, incl, kTileWarps - 1);
    }
  }
  __syncthreads();
  const size_t excl = tile_off[blockIdx.x];
#pragma unroll
  for (int j = 0; j < kTileItems; j++) {
    if ((bal[j] >> lane) & 1u) {
      const size_t p = excl + cnt[j][warp] + __popc(bal[j] & lt);  // INSERTs before this one
      // the host checked the count; the bound keeps a wrong one inside the buffer
      vals[base + (size_t)j * kTileThreads + threadIdx.x] = p < n_packed ? packed[p] : 0;
    }
  }
}

// A count of packed values that differs from the batch's INSERTs: every op
// code becomes invalid, so every request is answered kRejected and nothing
// is applied (the front end reads the op codes after this kernel)
__global__ void __launch_bounds__(kThreads) pack_check_kernel(const uint32_t* __restrict__ total, size_t n_packed,
                                                              uint8_t* __restrict__ ops, size_t n,
                                                              uint32_t* __restrict__ err) {
  const bool bad = (size_t)*total != n_packed;
  if (blockIdx.x == 0 && threadIdx.x == 0) *err = bad ? 1u : 0u;
  if (!bad) return;
  for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x)
    ops[i] = 0xFF;
}

// ---- INSERT combining for BT_MODE_STM batches ----
// Requests of an STM batch are concurrent transactions (the v39 meaning), so
// any serial order of them is a valid outcome.  The INSERTs of one key are
// put in the order in which they reach the key's table slot (an atomic
// exchange on the slot's tail): the first one (the representative) runs in
// the STM kernel and stores the value of the last one; every other INSERT is
// answered at once with the value of the one before it (FOUND), as if the
// key's INSERTs ran back to back at the representative's commit.  A key that
// the batch also DELETEs is not combined.  A slot's `first` holds the tail
// index, and `pad` the representative's index (bit 31: the key has a DELETE).
constexpr uint32_t kDelBit = 1u << 31;

// The requests of an STM batch split in two lists, in no particular order,
// with one atomic per warp and list: the valid GETs (with their keys, for
// the lookup kernels) and the rest (INSERT, DELETE, invalid op codes and the
// reserved key, which the STM kernel answers).  counts->n_lookup and
// counts->n_ins_req end as the lists' lengths.
__device__ __forceinline__ uint32_t warp_append(uint32_t m, uint32_t* __restrict__ counter) {
  const uint32_t lane = threadIdx.x & 31;
  const uint32_t c = __popc(m);
  uint32_t incl = c;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const uint32_t y = __shfl_up_sync(0xffffffffu, incl, o);
    if (lane >= (uint32_t)o) incl += y;
  }
  const uint32_t total = __shfl_sync(0xffffffffu, incl, 31);
  uint32_t base = 0;
  if (lane == 31 && total) base = atomicAdd(counter, total);
  base = __shfl_sync(0xffffffffu, base, 31);
  return base + incl - c;  // this lane's first slot
}

__global__ void __launch_bounds__(kThreads) stm_split_kernel(const uint64_t* __restrict__ keys,
                                                             const uint8_t* __restrict__ ops, size_t n,
                                                             uint32_t* __restrict__ get_list,
                                                             uint64_t* __restrict__ get_keys,
                                                             uint32_t* __restrict__ wr_list,
                                                             BatchCounts* __restrict__ counts) {
  const uint32_t lane = threadIdx.x & 31;
  const size_t stride = (size_t)gridDim.x * blockDim.x;
  // whole warps iterate together (the appends are warp-aggregated); four
  // requests per lane
  const size_t warp0 = ((size_t)blockIdx.x * blockDim.x + (threadIdx.x & ~31u)) * 4;
  for (size_t w = warp0; w < n; w += stride * 4) {
    const size_t i0 = w + 4 * (size_t)lane;
    uint32_t gm = 0, wm = 0;
    uint64_t k[4];
#pragma unroll
    for (int j = 0; j < 4; j++) {
      k[j] = kKeyMax;
      if (i0 + j < n) {
        k[j] = keys[i0 + j];
        const bool get = ops[i0 + j] == kOpGet && k[j] != kKeyMax;
        gm |= (get ? 1u : 0u) << j;
        wm |= (get ? 0u : 1u) << j;
      }
    }
    uint32_t pg = warp_append(gm, &counts->n_lookup);
    uint32_t pw = warp_append(wm, &counts->n_ins_req);
#pragma unroll
    for (int j = 0; j < 4; j++) {
      if ((gm >> j) & 1u) {
        get_list[pg] = (uint32_t)(i0 + j);
        get_keys[pg++] = k[j];
      } else if ((wm >> j) & 1u) {
        wr_list[pw++] = (uint32_t)(i0 + j);
      }
    }
  }
}

__global__ void __launch_bounds__(kThreads) combine_arrive_kernel(const uint64_t* __restrict__ keys,
                                                                  const uint8_t* __restrict__ ops,
                                                                  const uint32_t* __restrict__ list,
                                                                  Slot* __restrict__ tab,
                                                                  const BatchCounts* __restrict__ counts,
                                                                  uint32_t* __restrict__ pred,
                                                                  uint32_t* __restrict__ slot_of) {
  const uint32_t mask = counts->cap - 1;
  const size_t m = counts->n_ins_req;
  for (size_t q = (size_t)blockIdx.x * blockDim.x + threadIdx.x; q < m; q += (size_t)gridDim.x * blockDim.x) {
    const uint32_t i = list[q];
    const uint8_t op = ops[i];
    if (op != kOpInsert && op != kOpDelete) continue;  // an invalid request: the STM kernel rejects it
    const uint64_t k = keys[i];
    if (k == kKeyMax) continue;
    uint32_t h = (uint32_t)slot_hash(k) & mask;
    uint32_t at = kNone;
    for (uint32_t probe = 0; probe <= mask; probe++) {
      const unsigned long long prev = atomicCAS(&tab[h].key, (unsigned long long)kKeyMax, (unsigned long long)k);
      if (prev == kKeyMax || prev == k) {
        at = h;
        break;
      }
      h = (h + 1) & mask;
    }
    if (op == kOpDelete) {
      if (at != kNone) atomicOr(&tab[at].pad, kDelBit);
      continue;
    }
    slot_of[i] = at;
    if (at == kNone) continue;  // no slot (cannot happen below load 1): runs uncombined
    const uint32_t p = atomicExch(&tab[at].first, i);
    pred[i] = p;
    if (p == kNone) atomicOr(&tab[at].pad, i);
  }
}

// per INSERT: its value for the STM kernel, or (combined with an earlier one)
// its answer and a skip mark
__global__ void __launch_bounds__(kThreads) combine_mark_kernel(const uint64_t* __restrict__ keys,
                                                                const uint64_t* __restrict__ vals,
                                                                const uint8_t* __restrict__ ops,
                                                                const uint32_t* __restrict__ list,
                                                                const BatchCounts* __restrict__ counts,
                                                                const Slot* __restrict__ tab,
                                                                const uint32_t* __restrict__ pred,
                                                                const uint32_t* __restrict__ slot_of,
                                                                uint8_t* __restrict__ skip,
                                                                uint64_t* __restrict__ cvals,
                                                                uint64_t* __restrict__ out_vals,
                                                                uint8_t* __restrict__ out_st) {
  const size_t m = counts->n_ins_req;
  for (size_t q = (size_t)blockIdx.x * blockDim.x + threadIdx.x; q < m; q += (size_t)gridDim.x * blockDim.x) {
    const uint32_t i = list[q];
    if (ops[i] != kOpInsert) continue;
    const uint32_t at = keys[i] != kKeyMax ? slot_of[i] : kNone;
    uint8_t sk = 0;
    if (at == kNone || (tab[at].pad & kDelBit)) {
      cvals[i] = vals[i];
    } else if (pred[i] != kNone) {
      out_vals[i] = vals[pred[i]];
      out_st[i] = kFound;
      sk = 1;
    } else {
      cvals[i] = vals[tab[at].first];  // the last INSERT of the key
    }
    skip[i] = sk;
  }
}

// a representative that did not commit (retry limit, full node pool): the
// INSERTs combined with it report the same status
__global__ void __launch_bounds__(kThreads) combine_fixup_kernel(const uint8_t* __restrict__ ops,
                                                                 const uint32_t* __restrict__ list,
                                                                 const BatchCounts* __restrict__ counts,
                                                                 const uint8_t* __restrict__ skip,
                                                                 const Slot* __restrict__ tab,
                                                                 const uint32_t* __restrict__ slot_of,
                                                                 uint64_t* __restrict__ out_vals,
                                                                 uint8_t* __restrict__ out_st) {
  const size_t m = counts->n_ins_req;
  for (size_t q = (size_t)blockIdx.x * blockDim.x + threadIdx.x; q < m; q += (size_t)gridDim.x * blockDim.x) {
    const uint32_t i = list[q];
    if (ops[i] != kOpInsert || !skip[i]) continue;
    const uint32_t rep = tab[slot_of[i]].pad & ~kDelBit;
    const uint8_t st = out_st[rep];
    if (st == kRetryExhausted || st == kNoCapacity) {
      out_st[i] = st;
      out_vals[i] = 0;
    }
  }
}

}  // namespace

int stm_split(Handle* h, const uint64_t* keys, const uint8_t* ops, size_t n, cudaStream_t s) {
  Work& w = h->w;
  const unsigned g = (unsigned)min((size_t)h->sm_count * 8, (n / 4 + kThreads) / kThreads);
  if (cudaMemsetAsync(w.counts, 0, sizeof(BatchCounts), s) != cudaSuccess) return -2;
  stm_split_kernel<<<g, kThreads, 0, s>>>(keys, ops, n, w.get_list, w.ukeys, w.ins_list, w.counts);
  count_launch();
  return cudaGetLastError() == cudaSuccess ? 0 : -2;
}

int stm_combine(Handle* h, const uint64_t* keys, const uint64_t* vals, const uint8_t* ops, size_t n,
                uint64_t* out_vals, uint8_t* out_st, cudaStream_t s, const uint8_t** skip, const uint64_t** cvals) {
  Work& w = h->w;
  BatchCounts* c = w.counts;
  Slot* tab = reinterpret_cast<Slot*>(w.f_tab);
  uint8_t* sk = reinterpret_cast<uint8_t*>(w.f_flags);
  uint64_t* cv = w.f_lk;
  uint32_t* pred = w.f_list;
  uint32_t* slot_of = w.f_pos;
  uint32_t* list = w.ins_list;
  const unsigned g = (unsigned)min((size_t)h->sm_count * 8, (n / 4 + kThreads) / kThreads);
  front_clear_kernel<<<(unsigned)h->sm_count * 4, kThreads, 0, s>>>(tab, w.f_tab_cap, c);
  combine_arrive_kernel<<<g, kThreads, 0, s>>>(keys, ops, list, tab, c, pred, slot_of);
  combine_mark_kernel<<<g, kThreads, 0, s>>>(keys, vals, ops, list, c, tab, pred, slot_of, sk, cv, out_vals, out_st);
  count_launch(3);
  *skip = sk;
  *cvals = cv;
  return cudaGetLastError() == cudaSuccess ? 0 : -2;
}

int stm_combine_fixup(Handle* h, const uint8_t* ops, size_t n, uint64_t* out_vals, uint8_t* out_st, cudaStream_t s) {
  Work& w = h->w;
  const unsigned g = (unsigned)min((size_t)h->sm_count * 8, (n / 4 + kThreads) / kThreads);
  combine_fixup_kernel<<<g, kThreads, 0, s>>>(ops, w.ins_list, w.counts, reinterpret_cast<const uint8_t*>(w.f_flags),
                                              reinterpret_cast<const Slot*>(w.f_tab), w.f_pos, out_vals, out_st);
  count_launch();
  return cudaGetLastError() == cudaSuccess ? 0 : -2;
}

// scratch: tile counts, tile offsets, the INSERT total, the mismatch flag,
// then the scan's own words
size_t pack_scratch_words(size_t n) {
  const size_t tiles = (n + kTile - 1) / kTile;
  return 2 * (tiles + 1) + 2 + scan_scratch_words(tiles);
}

uint32_t* pack_error_word(uint32_t* scratch, size_t n_cap) {
  const size_t tiles = (n_cap + kTile - 1) / kTile;
  return scratch + 2 * (tiles + 1) + 1;
}

cudaError_t pack_check(uint8_t* ops, size_t n, size_t n_packed, uint32_t* scratch, size_t n_cap, int sm_count,
                       cudaStream_t s) {
  const size_t tiles = (n + kTile - 1) / kTile;
  const size_t cap_tiles = (n_cap + kTile - 1) / kTile;
  uint32_t* cnt = scratch;
  uint32_t* off = cnt + cap_tiles + 1;
  uint32_t* total = off + cap_tiles + 1;
  uint32_t* scan = total + 2;
  pack_count_kernel<<<(unsigned)tiles, kTileThreads, 0, s>>>(ops, n, cnt);
  count_launch();
  cudaError_t e = scan_exclusive_u32(cnt, off, tiles, total, scan, s);
  if (e != cudaSuccess) return e;
  pack_check_kernel<<<(unsigned)sm_count * 2, kThreads, 0, s>>>(total, n_packed, ops, n, total + 1);
  count_launch();
  return cudaGetLastError();
}

cudaError_t pack_expand(const uint8_t* ops, size_t n, const uint64_t* packed, size_t n_packed, uint64_t* vals,
                        const uint32_t* scratch, size_t n_cap, cudaStream_t s) {
  if (n == 0 || n_packed == 0) return cudaSuccess;
  const size_t tiles = (n + kTile - 1) / kTile;
  const size_t cap_tiles = (n_cap + kTile - 1) / kTile;
  pack_expand_kernel<<<(unsigned)tiles, kTileThreads, 0, s>>>(ops, n, scratch + cap_tiles + 1, packed, n_packed,
                                                              vals);
  count_launch();
  return cudaGetLastError();
}

// Fills w.f_tk/w.f_tv (touched requests, input order, count counts->n_touch)
// and w.f_list/w.f_lk (plain lookups and their keys, input order, count
// counts->n_lookup).
int front_classify(Handle* h, const uint64_t* keys, const uint8_t* ops, size_t n, cudaStream_t s) {
  Work& w = h->w;
  BatchCounts* c = w.counts;
  const size_t n_tiles = (n + kTile - 1) / kTile;
  if (cudaMemsetAsync(c, 0, sizeof(BatchCounts), s) != cudaSuccess) return -2;
  const unsigned g = (unsigned)min((size_t)h->sm_count * 8, (n + kThreads - 1) / kThreads);
  Slot* tab = reinterpret_cast<Slot*>(w.f_tab);
  uint8_t* flags = reinterpret_cast<uint8_t*>(w.f_flags);
  uint32_t* tile = w.f_pos;  // per-tile counts, then offsets
  front_count_kernel<<<(unsigned)h->sm_count * 2, kThreads, 0, s>>>(ops, n, c);
  front_clear_kernel<<<(unsigned)h->sm_count * 4, kThreads, 0, s>>>(tab, w.f_tab_cap, c);
  front_insert_kernel<<<g, kThreads, 0, s>>>(keys, ops, n, tab, c);
  front_flag_kernel<<<(unsigned)n_tiles, kTileThreads, 0, s>>>(keys, ops, n, tab, c, flags, tile);
  front_tile_scan_kernel<<<1, 1024, 0, s>>>(tile, (uint32_t)n_tiles, n, c, h->touch_hint_dev);
  front_scatter_kernel<<<(unsigned)n_tiles, kTileThreads, 0, s>>>(keys, ops, n, flags, tile, w.f_tk, w.f_tv,
                                                                  w.f_list, w.f_lk);
  count_launch(6);
  return cudaGetLastError() == cudaSuccess ? 0 : -2;
}

}  // namespace bt
