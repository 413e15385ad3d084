// Segmented leaf merge: the deterministic insert engine of the sorted batch
// (BT_MODE_SORTED | BT_MODE_MERGE_ENGINE).  No counterpart in the reference,
// which inserts one key per warp under STM (src/gpu-stm-tree-v39/
// bpt-gpustm-kernel.cu:14-256); the batch meaning is still v38's.
//
// With the batch's unique INSERT keys in ascending order:
//   locate    each 8-lane group walks a contiguous run of the keys (path reuse,
//             as in the sorted search), records the root-to-leaf path, answers
//             the previous value and records where an existing key's value
//             lives;
//   update    writes the new values of the existing keys in place;
//   compact   the new keys, then runs of new keys sharing a leaf (segments);
//   leaf      one 8-lane group per touched leaf merges its new keys by rank scatter
//             (each element computes its merged position by binary search in
//             the other sequence) and cuts an overflowing leaf into
//             p = ceil(m / leaf_fill) leaves of even size; the first keys of
//             pieces 1..p-1 become separator entries for the parent;
//   inner     one block applies the entries level by level the same way
//             (children spread evenly over q = ceil((s+1)/(inner_fill+1))
//             nodes, the key between two pieces moves up) and rebuilds an
//             overflowing root with the bulk-load rule.
// Locate only reads the tree, so it may run beside the batch's plain
// lookups (the hash front end does so); the in-place value update, compact,
// leaf and inner run after them and alone, so no locks are taken.  The rules are
// restated by the CPU oracle (bto_execute_merged with BTO_ENGINE_MERGE) and
// the resulting leaf layout is compared exactly.
#include <cuda_runtime.h>

#include "bt_block.cuh"
#include "bt_common.cuh"
#include "bt_internal.h"
#include "bt_search.cuh"

namespace bt {

struct MergeEntry {
  uint64_t key;
  uint32_t child;
  uint32_t rep;  // index of a new key whose path passes through this piece's parent
};

struct MergeCounts {
  uint32_t n_new;
  uint32_t n_segs;
  uint32_t n_leaf_entries;
  uint32_t node_base;
  uint32_t cap_fail;
  uint32_t pad[3];
};

namespace {

constexpr int kPathLevels = 8;
constexpr uint64_t kNoPos = ~0ull;  // merge_locate_kernel: no value to update in place
constexpr unsigned kFull = 0xffffffffu;

__device__ __forceinline__ uint32_t ceil_div(uint32_t a, uint32_t b) { return (a + b - 1) / b; }

// piece index and slot of merged position `pos` when m items are spread over p
// pieces (the first m % p pieces hold one more)
__device__ __forceinline__ void piece_of(uint32_t pos, uint32_t m, uint32_t p, uint32_t& c, uint32_t& slot) {
  const uint32_t b = m / p, rem = m % p;
  const uint32_t big = rem * (b + 1);
  if (pos < big) {
    c = pos / (b + 1);
    slot = pos % (b + 1);
  } else {
    const uint32_t q = pos - big;
    c = rem + q / b;
    slot = q % b;
  }
}
__device__ __forceinline__ uint32_t piece_size(uint32_t c, uint32_t m, uint32_t p) {
  return m / p + (c < m % p ? 1u : 0u);
}
__device__ __forceinline__ uint32_t piece_start(uint32_t c, uint32_t m, uint32_t p) {
  const uint32_t b = m / p, rem = m % p;
  return c * b + (c < rem ? c : rem);
}

// number of a[0..n) strictly below key (a ascending)
__device__ __forceinline__ uint32_t count_less(const uint64_t* a, uint32_t n, uint64_t key) {
  uint32_t lo = 0, hi = n;
  while (lo < hi) {
    const uint32_t mid = (lo + hi) >> 1;
    if (a[mid] < key) lo = mid + 1;
    else hi = mid;
  }
  return lo;
}

// ------------------------------------------------------------- root ----
__global__ void merge_ensure_root_kernel(DevTree t) {
  Ctrl* C = t.ctrl;
  if (C->root != kNil) return;
  const uint32_t id = atomicAdd(&C->n_nodes, 1u);
  if (id >= t.cap) {
    atomicOr(&C->error, kErrCapacity);
    return;
  }
  for (int i = 0; i < 31; i++) {
    t.keys[(size_t)id * 32 + i] = kKeyMax;
    t.vals[(size_t)id * 32 + i] = 0;
  }
  t.vals[(size_t)id * 32 + 31] = kKeyMax;
  t.keys[(size_t)id * 32 + 31] = make_hdr(0, 0, 0, C->epoch);
  t.low[id] = 0;
  C->root = id;
  C->root_level = 0;
}

// ------------------------------------------------------------- locate ----
template <int G>
__global__ void __launch_bounds__(256) merge_locate_kernel(DevTree t, const uint64_t* __restrict__ ukeys,
                                                           const uint64_t* __restrict__ uvals,
                                                           const uint32_t* __restrict__ ins_list,
                                                           const uint32_t* __restrict__ n_dev,
                                                           uint32_t* __restrict__ path, uint32_t* __restrict__ mleaf,
                                                           uint32_t* __restrict__ isnew,
                                                           uint64_t* __restrict__ vpos, uint64_t* __restrict__ uans,
                                                           uint8_t* __restrict__ uans_st, int use_pfx) {
  constexpr int S = 32 / G;
  const uint32_t lane = threadIdx.x & 31;
  const uint32_t g = lane % G;
  const uint32_t gmask = group_mask<G>(lane);
  const size_t n = *n_dev;
  const uint32_t root = t.ctrl->root;
  const uint32_t root_level = t.ctrl->root_level;
  const size_t n_groups = ((size_t)gridDim.x * blockDim.x) / G;
  const size_t gid = ((size_t)blockIdx.x * blockDim.x + threadIdx.x) / G;
  const size_t chunk = (n + n_groups - 1) / n_groups;
  const size_t q0 = gid * chunk;
  const size_t q1 = min(n, q0 + chunk);
  const bool usable = root != kNil && root_level < (uint32_t)kPathLevels;
  uint32_t c_node = root;
  uint64_t c_hi = 0;
  bool c_valid = (g == root_level);
  if (c_valid) c_hi = kKeyMax;
  uint64_t k[S];
  uint64_t v[S];
  uint32_t leaf = kNil;
  for (size_t q = q0; q < q1; q++) {
    const uint32_t u = ins_list[q];
    const uint64_t key = ukeys[u];
    if (!usable) {  // no root (pool exhausted) or a tree too tall for the path record
      if (g == 0) {
        uans[u] = 0;
        uans_st[u] = kNoCapacity;
        isnew[q] = 0;
        vpos[q] = kNoPos;
      }
      continue;
    }
    const uint32_t hit = (__ballot_sync(gmask, c_valid && key < c_hi) >> (lane - g)) & ((1u << G) - 1u);
    uint32_t level = hit ? (uint32_t)(__ffs(hit) - 1) : root_level;
    uint32_t node = __shfl_sync(gmask, c_node, level, G);
    uint64_t hi = __shfl_sync(gmask, c_hi, level, G);
    if (!hit) {
      node = root;
      hi = kKeyMax;
    }
    if (g < level) c_valid = false;
    uint32_t cnt = 0;
    if (level == 0 && node == leaf) {
      uint32_t c = 0;
#pragma unroll
      for (int i = 0; i < S; i++) c += (k[i] <= key) ? 1u : 0u;
      cnt = group_sum<G>(c, gmask);
    } else {
      for (;;) {
        const size_t row = (size_t)node * 32 + g * S;
        if (use_pfx && level > 0) {
          // inner level from the separators' prefixes, then the one separator
          // (the child's upper bound) and the one child id
          uint32_t pf[S];
          load_pfx<S>(t.pfx + row, pf, l2_keep());
          const uint32_t x = pfx_rank<G, S>(pf, key, g, gmask);
          cnt = x & 0xffffu;
          if (x >> 16) {  // a separator shares the key's prefix: rank with the full keys
            load_slots<S>(t.keys + row, k);
            if (g == G - 1) k[S - 1] = kKeyMax;
            uint32_t c = 0;
#pragma unroll
            for (int i = 0; i < S; i++) c += (k[i] <= key) ? 1u : 0u;
            cnt = group_sum<G>(c, gmask);
          }
          // the separator after the chosen child (slot 31 is the header: none)
          const uint64_t sep = cnt < 31 ? t.keys[(size_t)node * 32 + cnt] : kKeyMax;
          const uint64_t child_hi = sep < hi ? sep : hi;
          node = (uint32_t)t.vals[(size_t)node * 32 + cnt];
          hi = child_hi;
          level--;
          if (g == level) {
            c_node = node;
            c_hi = hi;
            c_valid = true;
          }
          continue;
        }
        load_slots<S>(t.keys + row, k);
        if (level > 0) load_slots<S>(t.vals + row, v);
        if (g == G - 1) k[S - 1] = kKeyMax;
        uint32_t c = 0;
#pragma unroll
        for (int i = 0; i < S; i++) c += (k[i] <= key) ? 1u : 0u;
        cnt = group_sum<G>(c, gmask);
        if (level == 0) break;
        const uint64_t sep = __shfl_sync(gmask, pick<S>(k, cnt % S), cnt / S, G);
        const uint64_t child_hi = sep < hi ? sep : hi;
        node = (uint32_t)__shfl_sync(gmask, pick<S>(v, cnt % S), cnt / S, G);
        hi = child_hi;
        level--;
        if (g == level) {
          c_node = node;
          c_hi = hi;
          c_valid = true;
        }
      }
      leaf = node;
    }
    // record the path: lane g holds level g
    if (g <= root_level) path[q * kPathLevels + g] = c_node;
    bool exists = false;
    uint32_t slot = 0;
    if (cnt > 0) {
      slot = cnt - 1;
      const uint64_t kk = __shfl_sync(gmask, pick<S>(k, slot % S), slot / S, G);
      exists = kk == key;
    }
    if (g == 0) {
      if (exists) {
        // the new value goes in later (merge_update_kernel): a plain lookup
        // of this key that comes before its first write must still see it
        const uint64_t p = (uint64_t)leaf * 32 + slot;
        uans[u] = t.vals[p];
        uans_st[u] = kFound;
        vpos[q] = p;
        isnew[q] = 0;
      } else {
        uans[u] = 0;
        uans_st[u] = kAbsent;
        isnew[q] = 1;
        vpos[q] = kNoPos;
        mleaf[q] = leaf;
      }
    }
  }
}

// new values of the keys the batch finds in the tree, in place (keys do not
// move); after the batch's plain lookups, before its DELETE apply
__global__ void merge_update_kernel(DevTree t, const uint64_t* __restrict__ uvals,
                                    const uint32_t* __restrict__ ins_list, const uint32_t* __restrict__ n_dev,
                                    const uint64_t* __restrict__ vpos) {
  const size_t n = *n_dev;
  const size_t stride = (size_t)gridDim.x * blockDim.x;
  for (size_t q = (size_t)blockIdx.x * blockDim.x + threadIdx.x; q < n; q += stride) {
    const uint64_t p = vpos[q];
    if (p != kNoPos) t.vals[p] = uvals[ins_list[q]];
  }
}

// ------------------------------------------------------------- compact ----
__global__ void merge_compact_kernel(const uint32_t* __restrict__ ins_list, const uint32_t* __restrict__ n_dev,
                                     const uint32_t* __restrict__ isnew, const uint32_t* __restrict__ pos,
                                     const uint64_t* __restrict__ ukeys, const uint64_t* __restrict__ uvals,
                                     const uint32_t* __restrict__ mleaf, uint64_t* __restrict__ newk,
                                     uint64_t* __restrict__ newv, uint32_t* __restrict__ nq,
                                     uint32_t* __restrict__ nleaf) {
  const size_t n = *n_dev;
  const size_t stride = (size_t)gridDim.x * blockDim.x;
  for (size_t q = (size_t)blockIdx.x * blockDim.x + threadIdx.x; q < n; q += stride) {
    if (!isnew[q]) continue;
    const uint32_t p = pos[q];
    const uint32_t u = ins_list[q];
    newk[p] = ukeys[u];
    newv[p] = uvals[u];
    nq[p] = (uint32_t)q;
    nleaf[p] = mleaf[q];
  }
}

__global__ void merge_seg_flags_kernel(const MergeCounts* __restrict__ mc, const uint32_t* __restrict__ nleaf,
                                       size_t n_upper, uint32_t* __restrict__ flags) {
  const size_t n_new = min(n_upper, (size_t)mc->n_new);  // the scan reads n_new flags
  const size_t stride = (size_t)gridDim.x * blockDim.x;
  for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n_new; i += stride)
    flags[i] = (i == 0 || nleaf[i] != nleaf[i - 1]) ? 1u : 0u;
}

// segment starts and each segment's leaf (so the leaf merge loads it without
// a dependent hop through the segment start)
__global__ void merge_seg_start_kernel(const MergeCounts* __restrict__ mc, const uint32_t* __restrict__ flags,
                                       const uint32_t* __restrict__ idx, const uint32_t* __restrict__ nleaf,
                                       uint32_t* __restrict__ seg_start, uint32_t* __restrict__ seg_leaf) {
  const uint32_t n_new = mc->n_new;
  const size_t stride = (size_t)gridDim.x * blockDim.x;
  for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n_new; i += stride)
    if (flags[i]) {
      seg_start[idx[i]] = (uint32_t)i;
      seg_leaf[idx[i]] = nleaf[i];
    }
}

__device__ __forceinline__ void seg_bounds(const MergeCounts* mc, const uint32_t* seg_start, uint32_t s,
                                           uint32_t& a, uint32_t& b) {
  a = seg_start[s];
  b = (s + 1 < mc->n_segs) ? seg_start[s + 1] : mc->n_new;
}

// pieces - 1 per segment (new leaves it creates)
__global__ void merge_leaf_count_kernel(DevTree t, uint32_t leaf_fill, const MergeCounts* __restrict__ mc,
                                        const uint32_t* __restrict__ seg_start, const uint32_t* __restrict__ nleaf,
                                        size_t n_upper, uint32_t* __restrict__ extra) {
  const size_t n_segs = min(n_upper, (size_t)mc->n_segs);  // the scan reads n_segs entries
  const size_t stride = (size_t)gridDim.x * blockDim.x;
  for (size_t s = (size_t)blockIdx.x * blockDim.x + threadIdx.x; s < n_segs; s += stride) {
    uint32_t a, b;
    seg_bounds(mc, seg_start, (uint32_t)s, a, b);
    const uint32_t leaf = nleaf[a];
    const uint32_t m = hdr_size(t.keys[(size_t)leaf * 32 + 31]) + (b - a);
    extra[s] = m <= (uint32_t)kMaxKeys ? 0u : ceil_div(m, leaf_fill) - 1;
  }
}

// reserve the leaf pieces (and headroom for the inner levels) in one step;
// all-or-nothing: on failure no leaf is touched and the new keys report
// kNoCapacity.  entry_cap bounds the separator-entry buffers.
__global__ void merge_alloc_kernel(DevTree t, MergeCounts* mc, uint32_t entry_cap) {
  const uint32_t T = mc->n_leaf_entries;
  const uint32_t need = T + T / 4 + 64;
  const uint32_t have = atomicAdd(&t.ctrl->n_nodes, 0u);
  if ((uint64_t)have + need > t.cap || T > entry_cap) {
    mc->cap_fail = 1;
    atomicOr(&t.ctrl->error, kErrCapacity);
    return;
  }
  mc->cap_fail = 0;
  mc->node_base = atomicAdd(&t.ctrl->n_nodes, T);
}

// a batch whose pieces did not fit answers kNoCapacity for all its new keys
__global__ void merge_fail_mark_kernel(const MergeCounts* __restrict__ mc, const uint32_t* __restrict__ nq,
                                       const uint32_t* __restrict__ ins_list, uint8_t* __restrict__ uans_st) {
  if (mc->cap_fail == 0) return;
  const uint32_t n_new = mc->n_new;
  const size_t stride = (size_t)gridDim.x * blockDim.x;
  for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n_new; i += stride)
    uans_st[ins_list[nq[i]]] = kNoCapacity;
}

// ------------------------------------------------------------- leaf ----
// One group of G lanes per touched leaf (segment); lane g holds slots
// g*S .. g*S+S-1 of the row.  Several leaves per warp keep more row loads in
// flight than a warp per leaf (the kernel is bound by the dependent chain
// segment bounds -> leaf id -> row).
template <int G>
__global__ void __launch_bounds__(256) merge_leaf_kernel(DevTree t, uint32_t leaf_fill, const MergeCounts* mc,
                                                         const uint32_t* __restrict__ seg_start,
                                                         const uint32_t* __restrict__ eoff,
                                                         const uint64_t* __restrict__ newk,
                                                         const uint64_t* __restrict__ newv,
                                                         const uint32_t* __restrict__ nq,
                                                         const uint32_t* __restrict__ seg_leaf,
                                                         MergeEntry* __restrict__ ent) {
  constexpr int S = 32 / G;
  __shared__ uint64_t s_keys[256 / G][32];
  __shared__ __align__(16) uint64_t s_mk[256 / G][32];  // merged row when it fits one leaf
  __shared__ __align__(16) uint64_t s_mv[256 / G][32];
  const uint32_t lane = threadIdx.x & 31;
  const uint32_t g = lane % G;
  const uint32_t grp = threadIdx.x / G;
  const uint32_t gmask = group_mask<G>(lane);
  const uint32_t n_segs = mc->n_segs;
  const bool fail = mc->cap_fail != 0;
  const uint32_t base = mc->node_base;
  const uint32_t n_groups = (gridDim.x * blockDim.x) / G;
  unsigned long long added = 0, splits = 0;
  for (uint32_t s = (blockIdx.x * blockDim.x + threadIdx.x) / G; s < n_segs; s += n_groups) {
    uint32_t a, b;
    seg_bounds(mc, seg_start, s, a, b);
    const uint32_t leaf = seg_leaf[s];
    const uint32_t cnt = b - a;
    if (fail) continue;  // merge_fail_mark_kernel answered these keys
    uint64_t ok[S], ov[S];
    load_slots<S>(t.keys + (size_t)leaf * 32 + g * S, ok);
    load_slots<S>(t.vals + (size_t)leaf * 32 + g * S, ov);
    const uint64_t h = __shfl_sync(gmask, ok[S - 1], G - 1, G);
    const uint64_t fence = __shfl_sync(gmask, ov[S - 1], G - 1, G);
    const uint32_t sz = hdr_size(h);
#pragma unroll
    for (int i = 0; i < S; i++) {
      const uint32_t slot = g * S + i;
      s_keys[grp][slot] = slot < sz ? ok[i] : kKeyMax;
    }
    __syncwarp(gmask);
    const uint32_t m = sz + cnt;
    const uint32_t p = m <= (uint32_t)kMaxKeys ? 1u : ceil_div(m, leaf_fill);
    if (p == 1) {
      // no split (the common case): merge into shared memory, then write
      // the row with one 16-byte store per lane and pair of slots
#pragma unroll
      for (int i = 0; i < S; i++) {
        const uint32_t slot = g * S + i;
        if (slot < sz) {
          const uint32_t pos = slot + count_less(newk + a, cnt, ok[i]);
          s_mk[grp][pos] = ok[i];
          s_mv[grp][pos] = ov[i];
        }
      }
      for (uint32_t j = g; j < cnt; j += G) {
        const uint64_t key = newk[a + j];
        const uint32_t pos = j + count_less(s_keys[grp], sz, key);
        s_mk[grp][pos] = key;
        s_mv[grp][pos] = newv[a + j];
      }
      __syncwarp(gmask);
      uint64_t wk[S], wv[S];
#pragma unroll
      for (int i = 0; i < S; i++) {
        const uint32_t slot = g * S + i;
        wk[i] = slot < m ? s_mk[grp][slot] : kKeyMax;
        wv[i] = slot < m ? s_mv[grp][slot] : 0;
      }
      if (g == G - 1) {
        wk[S - 1] = make_hdr(m, 0, hdr_version(h) + 1, hdr_epoch(h));
        wv[S - 1] = fence;
      }
      uint64_t* kr = t.keys + (size_t)leaf * 32 + g * S;
      uint64_t* vr = t.vals + (size_t)leaf * 32 + g * S;
#pragma unroll
      for (int i = 0; i < S; i += 2) {
        *reinterpret_cast<ulonglong2*>(kr + i) = make_ulonglong2(wk[i], wk[i + 1]);
        *reinterpret_cast<ulonglong2*>(vr + i) = make_ulonglong2(wv[i], wv[i + 1]);
      }
      __syncwarp(gmask);  // s_mk / s_mv are reused by the next segment
      if (g == 0) added += cnt;
      continue;
    }
    const uint32_t eo = eoff[s];
    auto node_of = [&](uint32_t c) -> uint32_t { return c == 0 ? leaf : base + eo + c - 1; };
    auto place = [&](uint32_t pos, uint64_t key, uint64_t val) {
      uint32_t c, slot;
      piece_of(pos, m, p, c, slot);
      const uint32_t nd = node_of(c);
      t.keys[(size_t)nd * 32 + slot] = key;
      t.vals[(size_t)nd * 32 + slot] = val;
      if (slot == 0 && c >= 1) {
        t.low[nd] = key;
        t.vals[(size_t)node_of(c - 1) * 32 + 31] = key;  // right fence of the piece before
        MergeEntry e;
        e.key = key;
        e.child = nd;
        e.rep = nq[a];
        ent[eo + c - 1] = e;
      }
    };
    // old keys and new keys to their merged positions (all reads happened above)
#pragma unroll
    for (int i = 0; i < S; i++) {
      const uint32_t slot = g * S + i;
      if (slot < sz) place(slot + count_less(newk + a, cnt, ok[i]), ok[i], ov[i]);
    }
    for (uint32_t j = g; j < cnt; j += G) {
      const uint64_t key = newk[a + j];
      place(j + count_less(s_keys[grp], sz, key), key, newv[a + j]);
    }
    __syncwarp(gmask);
    // padding, headers, last fence
    for (uint32_t c = 0; c < p; c++) {
      const uint32_t nd = node_of(c);
      const uint32_t kc = piece_size(c, m, p);
#pragma unroll
      for (int i = 0; i < S; i++) {
        const uint32_t slot = g * S + i;
        if (slot >= kc && slot < 31) {
          t.keys[(size_t)nd * 32 + slot] = kKeyMax;
          t.vals[(size_t)nd * 32 + slot] = 0;
        }
      }
      if (g == G - 1) {
        t.keys[(size_t)nd * 32 + 31] = make_hdr(kc, 0, c == 0 ? hdr_version(h) + 1 : 0, hdr_epoch(h));
        if (c == p - 1) t.vals[(size_t)nd * 32 + 31] = fence;
      }
    }
    __syncwarp(gmask);
    if (g == 0) {
      added += cnt;
      splits += p - 1;
    }
  }
  if (g == 0 && (added | splits)) {
    atomicAdd(&t.ctrl->n_keys, added);
    atomicAdd(&t.ctrl->leaf_splits, splits);
  }
}

// ------------------------------------------------------------- inner ----
// The separator entries are applied level by level by one cooperative grid
// (all blocks resident), with a grid barrier between the steps of a level.
// Entries are in ascending key order; those of one parent are contiguous.
// The barrier's wait is bounded: past kBarrierSpin it sets kErrSpin and every
// block leaves.
constexpr int kInnerThreads = 512;
constexpr int kInnerWarps = kInnerThreads / 32;
constexpr uint32_t kBarrierSpin = 1u << 24;

struct InnerSync {
  unsigned count;
  unsigned gen;
  uint32_t fail;
  uint32_t n_groups;
  uint32_t total;  // 1 when the capacity check failed
  uint32_t base;
  uint32_t pad[2];
  uint32_t partial[1024];  // per block
};

__device__ bool grid_sync(InnerSync* gs, uint32_t* err) {
  __shared__ int s_ok;
  __syncthreads();
  if (threadIdx.x == 0) {
    int ok = 1;
    const unsigned g = ld_acquire32(&gs->gen);
    __threadfence();
    if (atomicAdd(&gs->count, 1u) == gridDim.x - 1) {
      gs->count = 0;
      __threadfence();
      atomicAdd(&gs->gen, 1u);
    } else {
      uint32_t spins = 0;
      while (ld_acquire32(&gs->gen) == g) {
        if (++spins > kBarrierSpin) {
          atomicOr(err, kErrSpin);
          atomicExch(&gs->fail, 1u);
          ok = 0;
          break;
        }
        if (spins > 32) __nanosleep(128);
      }
    }
    __threadfence();
    if (ld_acquire32(&gs->fail)) ok = 0;
    s_ok = ok;
  }
  __syncthreads();
  return s_ok != 0;
}

// grid-wide exclusive scan of f(i), i < n: out[i] and the total.  Each block
// takes one contiguous chunk.  Contains two grid barriers.
template <typename F>
__device__ bool grid_scan_n(uint32_t n, F f, uint32_t* out, InnerSync* gs, uint32_t* err, uint32_t* ws,
                            uint32_t* total) {
  const uint32_t chunk = ceil_div(n, gridDim.x);
  const uint32_t c0 = min(n, blockIdx.x * chunk), c1 = min(n, c0 + chunk);
  uint32_t sum = 0;
  for (uint32_t base = c0; base < c1; base += kInnerThreads) {
    const uint32_t i = base + threadIdx.x;
    uint32_t tot;
    blk_exclusive_sum(i < c1 ? f(i) : 0u, ws, &tot);
    sum += tot;
  }
  if (threadIdx.x == 0) gs->partial[blockIdx.x] = sum;
  if (!grid_sync(gs, err)) return false;
  // this block's offset: sum of the lower blocks' partials
  uint32_t off = 0, all = 0;
  for (uint32_t b = threadIdx.x; b < gridDim.x; b += kInnerThreads) {
    const uint32_t v = gs->partial[b];
    all += v;
    if (b < blockIdx.x) off += v;
  }
  uint32_t t0, t1;
  blk_exclusive_sum(off, ws, &t0);
  blk_exclusive_sum(all, ws, &t1);
  uint32_t carry = t0;
  for (uint32_t base = c0; base < c1; base += kInnerThreads) {
    const uint32_t i = base + threadIdx.x;
    const uint32_t v = i < c1 ? f(i) : 0u;
    uint32_t tot;
    const uint32_t ex = blk_exclusive_sum(v, ws, &tot);
    if (i < c1) out[i] = carry + ex;
    carry += tot;
  }
  *total = t1;
  return grid_sync(gs, err);  // out[] complete before anyone reads it
}

__global__ void __launch_bounds__(kInnerThreads) merge_inner_kernel(DevTree t, uint32_t inner_fill, uint32_t entry_cap,
                                                                    MergeCounts* mc, InnerSync* gs,
                                                                    MergeEntry* ea, MergeEntry* eb,
                                                                    const uint32_t* __restrict__ path,
                                                                    uint32_t* __restrict__ gstart,
                                                                    uint32_t* __restrict__ goff,
                                                                    uint32_t* __restrict__ kids_a,
                                                                    uint32_t* __restrict__ kids_b) {
  __shared__ uint32_t ws[32];
  __shared__ uint32_t s_base;
  __shared__ uint64_t s_keys[kInnerWarps][32];
  if (mc->cap_fail) return;
  Ctrl* C = t.ctrl;
  uint32_t* err = &C->error;
  const uint32_t lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  const uint32_t gw = blockIdx.x * kInnerWarps + w, n_warps = gridDim.x * kInnerWarps;
  const uint32_t epoch = C->epoch;
  uint32_t n_e = mc->n_leaf_entries;
  MergeEntry* cur = ea;
  MergeEntry* nxt = eb;
  unsigned long long inner_new = 0, roots_new = 0;
  for (uint32_t lvl = 1; n_e > 0; lvl++) {
    const uint32_t root_level = C->root_level;
    if (lvl > root_level) {
      // the root split: block 0 rebuilds upward from [root, pieces...] with the bulk rule
      if (blockIdx.x != 0) break;
      uint32_t cnt = n_e + 1;
      if ((uint64_t)C->n_nodes + cnt > t.cap) {
        if (threadIdx.x == 0) atomicOr(&C->error, kErrCapacity);
        return;
      }
      for (uint32_t i = threadIdx.x; i < cnt; i += kInnerThreads) kids_a[i] = i == 0 ? C->root : cur[i - 1].child;
      __syncthreads();
      uint32_t* ka = kids_a;
      uint32_t* kb = kids_b;
      uint32_t level = lvl;
      while (cnt > 1) {
        const uint32_t per = inner_fill + 1;
        const uint32_t nn = ceil_div(cnt, per);
        if (threadIdx.x == 0) s_base = atomicAdd(&C->n_nodes, nn);
        __syncthreads();
        const uint32_t nb = s_base;
        for (uint32_t pidx = w; pidx < nn; pidx += kInnerWarps) {
          const uint32_t kc = piece_size(pidx, cnt, nn), cs = piece_start(pidx, cnt, nn);
          const uint32_t nd = nb + pidx;
          if (lane < 31) {
            const uint64_t sep = (lane + 1 < kc) ? t.low[ka[cs + lane + 1]] : kKeyMax;
            t.keys[(size_t)nd * 32 + lane] = sep;
            t.pfx[(size_t)nd * 32 + lane] = (uint32_t)(sep >> 32);
          } else {
            t.keys[(size_t)nd * 32 + 31] = make_hdr(kc - 1, level, 0, epoch);
          }
          t.vals[(size_t)nd * 32 + lane] = lane < kc ? (uint64_t)ka[cs + lane] : 0;
          if (lane == 0) {
            t.low[nd] = t.low[ka[cs]];
            kb[pidx] = nd;
          }
        }
        __syncthreads();
        roots_new += nn;
        uint32_t* tmp = ka;
        ka = kb;
        kb = tmp;
        cnt = nn;
        level++;
      }
      if (threadIdx.x == 0) {
        __threadfence();
        C->root = ka[0];
        C->root_level = level - 1;
      }
      __syncthreads();
      break;
    }
    // groups of entries sharing a parent at this level
    auto parent_of = [&](uint32_t i) { return path[(size_t)cur[i].rep * kPathLevels + lvl]; };
    auto is_head = [&](uint32_t i) -> uint32_t { return (i == 0 || parent_of(i) != parent_of(i - 1)) ? 1u : 0u; };
    uint32_t ng = 0;
    if (!grid_scan_n(n_e, is_head, goff, gs, err, ws, &ng)) return;
    for (uint32_t i = blockIdx.x * kInnerThreads + threadIdx.x; i < n_e; i += gridDim.x * kInnerThreads)
      if (is_head(i)) gstart[goff[i]] = i;
    if (!grid_sync(gs, err)) return;
    // pieces - 1 per group
    auto group_extra = [&](uint32_t gi) -> uint32_t {
      const uint32_t a = gstart[gi], b = gi + 1 < ng ? gstart[gi + 1] : n_e;
      const uint32_t P = parent_of(a);
      const uint32_t tot = hdr_size(t.keys[(size_t)P * 32 + 31]) + (b - a);
      return tot <= (uint32_t)kMaxKeys ? 0u : ceil_div(tot + 1, inner_fill + 1) - 1;
    };
    uint32_t total = 0;
    if (!grid_scan_n(ng, group_extra, goff, gs, err, ws, &total)) return;
    // one thread checks the capacity and allocates; everyone reads the outcome
    if (blockIdx.x == 0 && threadIdx.x == 0) {
      if (total > entry_cap || (uint64_t)C->n_nodes + total > t.cap) {
        // cannot happen with inner_fill >= 16 and the headroom reserved
        // above; stop before writing out of bounds and flag the error
        atomicOr(&C->error, kErrCapacity);
        gs->total = 1;
      } else {
        gs->total = 0;
        gs->base = total ? atomicAdd(&C->n_nodes, total) : 0;
      }
    }
    if (!grid_sync(gs, err)) return;
    if (gs->total) return;
    const uint32_t nb = gs->base;
    for (uint32_t gi = gw; gi < ng; gi += n_warps) {
      const uint32_t a = gstart[gi], b = gi + 1 < ng ? gstart[gi + 1] : n_e;
      const uint32_t cnt = b - a;
      const uint32_t P = parent_of(a);
      const uint64_t pk = t.keys[(size_t)P * 32 + lane];
      const uint64_t pv = t.vals[(size_t)P * 32 + lane];
      const uint64_t h = __shfl_sync(kFull, pk, 31);
      const uint32_t sz = hdr_size(h);
      s_keys[w][lane] = lane < sz ? pk : kKeyMax;
      const uint64_t child0 = __shfl_sync(kFull, pv, 0);
      __syncwarp();
      const uint32_t tot = sz + cnt;
      const uint32_t ch = tot + 1;
      const uint32_t q = tot <= (uint32_t)kMaxKeys ? 1u : ceil_div(ch, inner_fill + 1);
      const uint32_t go = goff[gi];
      auto node_of = [&](uint32_t c) -> uint32_t { return c == 0 ? P : nb + go + c - 1; };
      // separator at merged position x with right child rc: its child index is x + 1
      auto place = [&](uint32_t x, uint64_t key, uint64_t rc) {
        uint32_t c, slot;
        piece_of(x + 1, ch, q, c, slot);
        const uint32_t nd = node_of(c);
        if (slot == 0) {  // first child of piece c >= 1: the separator moves up
          t.vals[(size_t)nd * 32] = rc;
          t.low[nd] = key;
          MergeEntry e;
          e.key = key;
          e.child = nd;
          e.rep = cur[a].rep;
          nxt[go + c - 1] = e;
        } else {
          t.keys[(size_t)nd * 32 + slot - 1] = key;
          t.pfx[(size_t)nd * 32 + slot - 1] = (uint32_t)(key >> 32);
          t.vals[(size_t)nd * 32 + slot] = rc;
        }
      };
      const uint64_t rc_next = __shfl_down_sync(kFull, pv, 1);  // right child of separator `lane`
      if (lane < sz) {
        const uint64_t rc = rc_next;
        uint32_t lo = 0, hi = cnt;
        while (lo < hi) {
          const uint32_t mid = (lo + hi) >> 1;
          if (cur[a + mid].key < pk) lo = mid + 1;
          else hi = mid;
        }
        place(lane + lo, pk, rc);
      }
      __syncwarp();
      for (uint32_t j = lane; j < cnt; j += 32) {
        const MergeEntry e = cur[a + j];
        place(j + count_less(s_keys[w], sz, e.key), e.key, e.child);
      }
      __syncwarp();
      for (uint32_t c = 0; c < q; c++) {
        const uint32_t nd = node_of(c);
        const uint32_t kc = piece_size(c, ch, q);
        if (c == 0 && lane == 0) t.vals[(size_t)nd * 32] = child0;
        if (lane + 1 >= kc && lane < 31) {
          t.keys[(size_t)nd * 32 + lane] = kKeyMax;
          t.pfx[(size_t)nd * 32 + lane] = 0xffffffffu;
        }
        if (lane >= kc) t.vals[(size_t)nd * 32 + lane] = 0;
        if (lane == 31) t.keys[(size_t)nd * 32 + 31] =
            make_hdr(kc - 1, lvl, c == 0 ? hdr_version(h) + 1 : 0, hdr_epoch(h));
      }
      __syncwarp();
    }
    if (blockIdx.x == 0) inner_new += total;
    if (!grid_sync(gs, err)) return;  // this level's nodes and the next entries are written
    n_e = total;
    MergeEntry* tmp = cur;
    cur = nxt;
    nxt = tmp;
  }
  if (blockIdx.x == 0 && threadIdx.x == 0 && (inner_new | roots_new)) {
    atomicAdd(&C->inner_splits, inner_new + roots_new);
    atomicAdd(&C->new_roots, roots_new);
  }
}

inline unsigned nblk(size_t n, int per) { return (unsigned)((n + per - 1) / per); }

}  // namespace

// cooperative launch of merge_inner_kernel: at most the resident blocks
static cudaError_t launch_inner(Handle* h, uint32_t entry_cap, MergeCounts* mc, cudaStream_t s) {
  Work& w = h->w;
  static unsigned resident[64] = {};
  const int dev = h->device;
  unsigned blocks = (unsigned)h->sm_count;
  if (dev >= 0 && dev < 64) {
    if (!resident[dev]) {
      int per = 0;
      if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, merge_inner_kernel, kInnerThreads, 0) != cudaSuccess ||
          per < 1)
        per = 1;
      resident[dev] = (unsigned)per * (unsigned)h->sm_count;
    }
    blocks = resident[dev];
  }
  if (blocks > 1024) blocks = 1024;  // InnerSync::partial
  InnerSync* gs = reinterpret_cast<InnerSync*>(w.m_sync);
  cudaError_t e = cudaMemsetAsync(gs, 0, sizeof(InnerSync), s);
  if (e != cudaSuccess) return e;
  DevTree tree = h->tree;
  uint32_t fill = h->inner_fill;
  MergeEntry* ea = reinterpret_cast<MergeEntry*>(w.m_ent_a);
  MergeEntry* eb = reinterpret_cast<MergeEntry*>(w.m_ent_b);
  const uint32_t* path = w.m_path;
  uint32_t* gstart = w.m_seg;
  uint32_t* goff = w.m_nleaf;
  uint32_t* kids_a = w.m_nq;
  uint32_t* kids_b = w.m_pos;
  void* args[] = {&tree, &fill, &entry_cap, &mc, &gs, &ea, &eb, &path, &gstart, &goff, &kids_a, &kids_b};
  e = cudaLaunchCooperativeKernel((const void*)merge_inner_kernel, dim3(blocks), dim3(kInnerThreads), args, 0, s);
  count_launch();
  return e;
}

// Runs the merge engine for the unique INSERT keys of the current batch
// (w.ins_list, count on the device).  n_upper bounds the count.
int merge_locate_phase(Handle* h, cudaStream_t s) {
  Work& w = h->w;
  MergeCounts* mc = reinterpret_cast<MergeCounts*>(w.m_counts);
  const uint32_t* n_ins = &w.counts->n_ins;
  merge_ensure_root_kernel<<<1, 1, 0, s>>>(h->tree);
  count_launch();
  const int use_pfx = h->use_pfx ? 1 : 0;
  if (use_pfx && ensure_pfx(h, s) != cudaSuccess) return -2;
  if (cudaMemsetAsync(mc, 0, sizeof(MergeCounts), s) != cudaSuccess) return -2;
  static int per_sm[64] = {};
  if (h->device < 64 && per_sm[h->device] == 0) {
    int b = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b, merge_locate_kernel<8>, 256, 0) != cudaSuccess || b < 1)
      b = 4;
    per_sm[h->device] = b;
  }
  const size_t blocks = (size_t)h->sm_count * (h->device < 64 ? per_sm[h->device] : 4);
  merge_locate_kernel<8><<<(unsigned)blocks, 256, 0, s>>>(h->tree, w.ukeys, w.uvals, w.ins_list, n_ins, w.m_path,
                                                          w.m_leaf, w.m_isnew, w.m_vpos, w.uans, w.uans_st, use_pfx);
  count_launch();
  return cudaGetLastError() == cudaSuccess ? 0 : -2;
}

int merge_update_phase(Handle* h, size_t n_upper, cudaStream_t s) {
  Work& w = h->w;
  const unsigned gb = (unsigned)min((size_t)h->sm_count * 8, (n_upper + 255) / 256);
  merge_update_kernel<<<gb, 256, 0, s>>>(h->tree, w.uvals, w.ins_list, &w.counts->n_ins, w.m_vpos);
  count_launch();
  return cudaGetLastError() == cudaSuccess ? 0 : -2;
}

int merge_group_phase(Handle* h, size_t n_upper, cudaStream_t s) {
  Work& w = h->w;
  MergeCounts* mc = reinterpret_cast<MergeCounts*>(w.m_counts);
  const uint32_t* n_ins = &w.counts->n_ins;
  uint32_t* err = &h->tree.ctrl->error;
  if (scan_exclusive_u32_lb(w.m_isnew, w.m_pos, n_upper, n_ins, &mc->n_new, w.lb_status, w.lb_ctr, &w.lb_epoch, err,
                            s) != cudaSuccess)
    return -2;
  const unsigned gb = (unsigned)min((size_t)h->sm_count * 8, (n_upper + 255) / 256);
  merge_compact_kernel<<<gb, 256, 0, s>>>(w.ins_list, n_ins, w.m_isnew, w.m_pos, w.ukeys, w.uvals, w.m_leaf, w.m_newk,
                                          w.m_newv, w.m_nq, w.m_nleaf);
  merge_seg_flags_kernel<<<gb, 256, 0, s>>>(mc, w.m_nleaf, n_upper, w.m_isnew);
  count_launch(2);
  if (scan_exclusive_u32_lb(w.m_isnew, w.m_pos, n_upper, &mc->n_new, &mc->n_segs, w.lb_status, w.lb_ctr, &w.lb_epoch,
                            err, s) != cudaSuccess)
    return -2;
  merge_seg_start_kernel<<<gb, 256, 0, s>>>(mc, w.m_isnew, w.m_pos, w.m_nleaf, w.m_seg, w.m_leaf);
  count_launch();
  return cudaGetLastError() == cudaSuccess ? 0 : -2;
}

int merge_reserve_phase(Handle* h, size_t n_upper, cudaStream_t s) {
  Work& w = h->w;
  MergeCounts* mc = reinterpret_cast<MergeCounts*>(w.m_counts);
  const unsigned gb = (unsigned)min((size_t)h->sm_count * 8, (n_upper + 255) / 256);
  merge_leaf_count_kernel<<<gb, 256, 0, s>>>(h->tree, h->leaf_fill, mc, w.m_seg, w.m_nleaf, n_upper, w.m_isnew);
  count_launch();
  if (scan_exclusive_u32_lb(w.m_isnew, w.m_pos, n_upper, &mc->n_segs, &mc->n_leaf_entries, w.lb_status, w.lb_ctr,
                            &w.lb_epoch, &h->tree.ctrl->error, s) !=
      cudaSuccess)
    return -2;
  merge_alloc_kernel<<<1, 1, 0, s>>>(h->tree, mc, (uint32_t)w.cap);
  merge_fail_mark_kernel<<<gb, 256, 0, s>>>(mc, w.m_nq, w.ins_list, w.uans_st);
  count_launch(2);
  return cudaGetLastError() == cudaSuccess ? 0 : -2;
}

int merge_write_phase(Handle* h, cudaStream_t s) {
  Work& w = h->w;
  MergeCounts* mc = reinterpret_cast<MergeCounts*>(w.m_counts);
  const uint32_t entry_cap = (uint32_t)w.cap;
  merge_leaf_kernel<8><<<(unsigned)((size_t)h->sm_count * 8), 256, 0, s>>>(
      h->tree, h->leaf_fill, mc, w.m_seg, w.m_pos, w.m_newk, w.m_newv, w.m_nq, w.m_leaf,
      reinterpret_cast<MergeEntry*>(w.m_ent_a));
  count_launch();
  if (launch_inner(h, entry_cap, mc, s) != cudaSuccess) return -2;
  return cudaGetLastError() == cudaSuccess ? 0 : -2;
}

int merge_engine(Handle* h, size_t n_upper, cudaStream_t s) {
  if (merge_locate_phase(h, s) != 0 || merge_update_phase(h, n_upper, s) != 0 ||
      merge_group_phase(h, n_upper, s) != 0 || merge_reserve_phase(h, n_upper, s) != 0)
    return -2;
  return merge_write_phase(h, s);
}

}  // namespace bt
