// Warp-level software transactional memory over the B+tree: one warp per
// request, lane i owns slot i of the node it is looking at.  Restates the
// reference's tx_insert_kernel (src/gpu-stm-tree-v39/bpt-gpustm-kernel.cu:14-256)
// with three design changes:
//   * the version/lock word is the node header (keys[31]) rather than a side
//     table, so the seqlock read of a node needs no extra sector;
//   * ordering is explicit: ld.acquire of the header, fence.acq_rel before
//     the validating re-read, release stores of the header on commit (the
//     reference relies on volatile loads, src/.../bpt-gpustm-kernel-tx.cuh:46-66);
//   * the parent is re-validated against its full header word (lock bit
//     included) after the child is read, and retries are bounded: a request
//     that cannot commit within the limit reports kRetryExhausted.
// Structure rules (early split of full inner nodes, 16|16 leaf split, new
// root) follow src/gpu-stm-tree-v39/bpt-gpustm-kernel-tree.cuh:150-467.
#include <cuda_runtime.h>

#include "bt_common.cuh"
#include "bt_internal.h"
#include "bt_learned.cuh"

namespace bt {

namespace {

constexpr unsigned kFull = 0xffffffffu;
enum : int { TX_DONE = 0, TX_ABORT = 1, TX_AGAIN = 2, TX_NOCAP = 3 };

__device__ __forceinline__ uint64_t* hdr_ptr(const DevTree& t, uint32_t n) { return t.keys + (size_t)n * 32 + 31; }

// Lock node n1 (expected header h1), node n2 (h2) and/or the root lock (rl).
// One lane takes them one after the other in a fixed order -- root lock, then
// the parent n2, then the node n1 -- and stops at the first that fails,
// restoring what it took.  Taking them in parallel let two transactions
// each hold one of a pair and fail each other again and again (observed: a
// second-long livelock of warps splitting the same inner node); in a fixed
// order whoever gets the first lock can go on to take the rest.
__device__ bool acquire_locks(const DevTree& t, uint32_t n1, uint64_t h1, uint32_t n2, uint64_t h2, bool lock_root,
                              uint32_t rl) {
  int ok = 1;
  if (lane_id() == 0) {
    bool got_root = false, got_n2 = false;
    if (lock_root) {
      got_root = atomicCAS(&t.ctrl->root_lock, rl, rl | 1u) == rl;
      ok = got_root;
    }
    if (ok && n2 != kNil) {
      got_n2 = atomicCAS((unsigned long long*)hdr_ptr(t, n2), h2, hdr_lock(h2)) == h2;
      ok = got_n2;
    }
    if (ok && n1 != kNil) ok = atomicCAS((unsigned long long*)hdr_ptr(t, n1), h1, hdr_lock(h1)) == h1;
    if (!ok) {  // nothing was written: put the same versions back
      if (got_n2) st_release(hdr_ptr(t, n2), h2);
      if (got_root) st_release32(&t.ctrl->root_lock, rl);
    }
  }
  ok = __shfl_sync(kFull, ok, 0);
  if (!ok) return false;
  __threadfence();
  return true;
}

__device__ void unlock_unchanged(const DevTree& t, uint32_t n1, uint64_t h1, uint32_t n2, uint64_t h2, bool root,
                                 uint32_t rl) {
  const uint32_t lane = lane_id();
  if (lane == 0 && n1 != kNil) st_release(hdr_ptr(t, n1), h1);
  if (lane == 1 && n2 != kNil) st_release(hdr_ptr(t, n2), h2);
  if (lane == 2 && root) st_release32(&t.ctrl->root_lock, rl);
  __syncwarp();
}

__device__ uint32_t alloc_nodes(const DevTree& t, uint32_t cnt) {
  uint32_t base = 0;
  if (lane_id() == 0) {
    base = atomicAdd(&t.ctrl->n_nodes, cnt);
    if (base >= t.cap || base + cnt > t.cap) {
      atomicOr(&t.ctrl->error, kErrCapacity);
      base = kNil;
    }
  }
  return __shfl_sync(kFull, base, 0);
}

// lane-parallel row write; the header slot (keys[31]) is written only for new
// nodes (write_hdr), existing nodes publish their header with a release store.
__device__ __forceinline__ void write_row(const DevTree& t, uint32_t n, uint64_t k, uint64_t v, bool write_hdr,
                                          uint64_t hdr) {
  const uint32_t lane = lane_id();
  uint64_t* kr = t.keys + (size_t)n * 32;
  uint64_t* vr = t.vals + (size_t)n * 32;
  if (lane < 31) kr[lane] = k;
  else if (write_hdr) kr[31] = hdr;
  vr[lane] = v;
}

// Split commit shared by the leaf split and the early inner split.
// left image (lk, lv, lhdr) replaces node `node` (read at header h);
// right image (rk, rv, rhdr) becomes a new node with low fence `up`; the
// parent (read at ph with lanes' slots pk/pv) gets separator `up` at pslot,
// or a new root is created above `node`.
__device__ int commit_split(const DevTree& t, uint32_t node, uint64_t h, uint64_t lk, uint64_t lv, uint64_t lhdr,
                            uint64_t rk, uint64_t rv, uint32_t rsize, uint32_t level, uint64_t up, uint32_t parent,
                            uint64_t ph, uint32_t pslot, uint64_t pk, uint64_t pv, uint32_t rl) {
  const uint32_t lane = lane_id();
  Ctrl* C = t.ctrl;
  // parent image shift (computed by all lanes before branching)
  const uint64_t upk = __shfl_up_sync(kFull, pk, 1);
  const uint64_t upv = __shfl_up_sync(kFull, pv, 1);
  const bool new_root = (parent == kNil);
  // an exhausted pool fails the split before any lock is taken, so readers of
  // these nodes are not aborted by lock churn once nothing can grow
  const uint32_t used = __shfl_sync(kFull, lane == 0 ? ld_relaxed32(&C->n_nodes) : 0u, 0);  // one value for the warp
  if (used + (new_root ? 2u : 1u) > t.cap) {
    if (lane == 0) atomicOr(&C->error, kErrCapacity);
    return TX_NOCAP;
  }
  if (!acquire_locks(t, node, h, parent, ph, new_root, rl)) return TX_ABORT;
  const uint32_t base = alloc_nodes(t, new_root ? 2u : 1u);
  if (base == kNil) {
    unlock_unchanged(t, node, h, parent, ph, new_root, rl);
    return TX_NOCAP;
  }
  const uint32_t right = base;
  // new right node (unreachable until the parent / root is published)
  write_row(t, right, rk, rv, false, 0);
  if (lane == 0) t.low[right] = up;
  write_row(t, node, lk, lv, false, 0);
  uint32_t psize = 0;
  if (!new_root) {
    psize = hdr_size(ph);
    const uint64_t npk = lane < pslot ? pk : (lane == pslot ? up : upk);
    const uint64_t npv = lane <= pslot ? pv : (lane == pslot + 1 ? (uint64_t)right : upv);
    write_row(t, parent, npk, npv, false, 0);
  } else {
    const uint32_t nr = base + 1;
    const uint64_t nk = lane == 0 ? up : kKeyMax;
    const uint64_t nv = lane == 0 ? (uint64_t)node : (lane == 1 ? (uint64_t)right : 0);
    write_row(t, nr, nk, nv, false, 0);
    if (lane == 0) t.low[nr] = t.low[node];
  }
  // new nodes become valid with a release store of their header after their
  // rows and low fences, so a reader that acquires the header sees them whole
  __threadfence();
  __syncwarp();
  const uint32_t ep = hdr_epoch(h);
  if (lane == 2) st_release(hdr_ptr(t, right), make_hdr(rsize, level, 0, ep));
  if (new_root && lane == 3) st_release(hdr_ptr(t, base + 1), make_hdr(1, level + 1, 0, ep));
  __threadfence();
  __syncwarp();
  if (lane == 0) st_release(hdr_ptr(t, node), lhdr);
  if (!new_root) {
    if (lane == 1) st_release(hdr_ptr(t, parent), hdr_next(ph, psize + 1));
  } else if (lane == 0) {
    C->root_level = level + 1;
    C->root = base + 1;
    __threadfence();
    st_release32(&C->root_lock, rl + 2u);
  }
  __syncwarp();
  if (lane == 0) {
    if (level == 0) atomicAdd(&C->leaf_splits, 1ull);
    else atomicAdd(&C->inner_splits, 1ull);
    if (new_root) {
      atomicAdd(&C->new_roots, 1ull);
      atomicAdd(&C->inner_splits, 1ull);
    }
  }
  return TX_DONE;
}

// DELETE in a leaf read under the seqlock (row k/v, header h): absent keys
// answer ABSENT without a write; a present key is removed by a shift under
// the leaf's lock (no merge with siblings; an emptied leaf stays).
__device__ int leaf_delete(const DevTree& t, uint32_t node, uint64_t h, uint64_t k, uint64_t v, uint32_t size,
                           uint32_t mm, uint64_t& ans, uint8_t& st) {
  const uint32_t lane = lane_id();
  if (!mm) {
    ans = 0;
    st = kAbsent;
    return TX_DONE;
  }
  const uint32_t at = __ffs(mm) - 1;
  const uint64_t old = __shfl_sync(kFull, v, at);
  const uint64_t dk = __shfl_down_sync(kFull, k, 1);
  const uint64_t dv = __shfl_down_sync(kFull, v, 1);
  if (!acquire_locks(t, node, h, kNil, 0, false, 0)) return TX_ABORT;
  if (lane >= at && lane < size) {
    const bool last = lane + 1 == size;
    t.keys[(size_t)node * 32 + lane] = last ? kKeyMax : dk;
    t.vals[(size_t)node * 32 + lane] = last ? 0 : dv;
  }
  __threadfence();
  __syncwarp();
  if (lane == 0) {
    st_release(hdr_ptr(t, node), hdr_next(h, size - 1));
    atomicAdd(&t.ctrl->n_keys, ~0ull);  // - 1
  }
  __syncwarp();
  ans = old;
  st = kFound;
  return TX_DONE;
}

// One transaction attempt for one request (all 32 lanes).
__device__ int tx_attempt(const DevTree& t, const uint64_t key, const uint64_t val, const bool is_insert,
                          const bool is_del, uint64_t& ans, uint8_t& st) {
  const uint32_t lane = lane_id();
  Ctrl* C = t.ctrl;
  // ---- root (reference TX_READ_ROOT, bpt-gpustm-kernel-tx.cuh:92-119)
  uint32_t rl = 0, root = 0;
  int bad0 = 0;
  if (lane == 0) {
    rl = ld_acquire32(&C->root_lock);
    root = ld_relaxed32(&C->root);
    fence_acq_rel();
    bad0 = (rl & 1u) || ld_relaxed32(&C->root_lock) != rl;
  }
  if (__shfl_sync(kFull, bad0, 0)) return TX_ABORT;
  rl = __shfl_sync(kFull, rl, 0);
  root = __shfl_sync(kFull, root, 0);
  if (root == kNil) {
    if (!is_insert) {
      ans = 0;
      st = kAbsent;
      return TX_DONE;
    }
    // CREATE_NEW_TREE (bpt-gpustm-kernel-tree.cuh:122-147): an empty leaf root
    if (!acquire_locks(t, kNil, 0, kNil, 0, true, rl)) return TX_ABORT;
    const uint32_t id = alloc_nodes(t, 1);
    if (id == kNil) {
      unlock_unchanged(t, kNil, 0, kNil, 0, true, rl);
      return TX_NOCAP;
    }
    write_row(t, id, kKeyMax, lane == 31 ? kKeyMax : 0, false, 0);
    if (lane == 0) t.low[id] = 0;
    __threadfence();
    __syncwarp();
    if (lane == 0) st_release(hdr_ptr(t, id), make_hdr(0, 0, 0, ld_relaxed32(&C->epoch)));
    __threadfence();
    __syncwarp();
    if (lane == 0) {
      C->root_level = 0;
      C->root = id;
      __threadfence();
      st_release32(&C->root_lock, rl + 2u);
    }
    __syncwarp();
    return TX_AGAIN;
  }
  // ---- descent with per-level validation (TX_READ, bpt-gpustm-kernel-tx.cuh:25-88)
  uint32_t node = root, parent = kNil, pslot = 0;
  uint64_t h = 0, ph = 0, k = 0, v = 0, pk = kKeyMax, pv = 0;
  for (int depth = 0;; depth++) {
    if (depth > 40) return TX_ABORT;  // defensive: no valid tree is this tall
    const uint64_t* krow = t.keys + (size_t)node * 32;
    const uint64_t* vrow = t.vals + (size_t)node * 32;
    h = ld_acquire(krow + 31);
    k = ld_relaxed(krow + lane);
    v = ld_relaxed(vrow + lane);
    fence_acq_rel();
    const uint64_t h2 = ld_relaxed(krow + 31);
    const uint64_t h_lane0 = __shfl_sync(kFull, h, 0);  // every lane must see one version
    const bool up_ok = (parent != kNil) ? (ld_relaxed(hdr_ptr(t, parent)) == ph)
                                        : (ld_relaxed32(&C->root_lock) == rl);
    const bool bad = hdr_locked(h) || h2 != h || h != h_lane0 || !up_ok;
    if (__any_sync(kFull, bad)) return TX_ABORT;
    if (lane == 31) k = kKeyMax;  // slot 31 is the header
    const uint32_t level = hdr_level(h), size = hdr_size(h);
    if (level > 0 && size >= (uint32_t)kMaxKeys && is_insert) {
      // early split of a full inner node (bpt-gpustm-kernel.cu:160-179,
      // NODE_SPLITTING bpt-gpustm-kernel-tree.cuh:150-224): up = key[15]
      const uint32_t mid = 15;
      const uint64_t up = __shfl_sync(kFull, k, mid);
      const uint64_t rk0 = __shfl_down_sync(kFull, k, mid + 1);
      const uint64_t rv0 = __shfl_down_sync(kFull, v, mid + 1);
      const uint64_t lk = lane < mid ? k : kKeyMax;
      const uint64_t lv = lane <= mid ? v : 0;
      const uint64_t rk = lane < mid ? rk0 : kKeyMax;
      const uint64_t rv = lane <= mid ? rv0 : 0;
      const int r = commit_split(t, node, h, lk, lv, hdr_next(h, mid), rk, rv, mid, level, up,
                                 parent, ph, pslot, pk, pv, rl);
      return r == TX_DONE ? TX_AGAIN : r;
    }
    if (level == 0) break;
    const uint32_t c = __popc(__ballot_sync(kFull, lane < 31 && k <= key));
    const uint32_t child = (uint32_t)__shfl_sync(kFull, v, c);
    parent = node;
    ph = h;
    pslot = c;
    pk = k;
    pv = v;
    node = child;
  }
  // ---- leaf (answer rule bpt-gpustm-kernel.cu:197-213)
  const uint32_t size = hdr_size(h);
  const uint32_t mm = __ballot_sync(kFull, lane < size && k == key);
  if (is_del) return leaf_delete(t, node, h, k, v, size, mm, ans, st);
  if (!is_insert) {
    if (mm) {
      ans = __shfl_sync(kFull, v, __ffs(mm) - 1);
      st = kFound;
    } else {
      ans = 0;
      st = kAbsent;
    }
    return TX_DONE;
  }
  if (mm) {
    // key present: update in place, answer the previous value (INSERT_LEAF :373-384)
    const uint32_t at = __ffs(mm) - 1;
    const uint64_t old = __shfl_sync(kFull, v, at);
    if (!acquire_locks(t, node, h, kNil, 0, false, 0)) return TX_ABORT;
    if (lane == at) t.vals[(size_t)node * 32 + at] = val;
    __threadfence();
    __syncwarp();
    if (lane == 0) st_release(hdr_ptr(t, node), hdr_next(h, size));
    __syncwarp();
    ans = old;
    st = kFound;
    return TX_DONE;
  }
  // shift-insert at p = number of keys < key
  const uint32_t p = __popc(__ballot_sync(kFull, lane < size && k < key));
  const uint64_t uk = __shfl_up_sync(kFull, k, 1);
  const uint64_t uv = __shfl_up_sync(kFull, v, 1);
  const uint64_t nk = lane < p ? k : (lane == p ? key : uk);
  const uint64_t nv = lane < p ? v : (lane == p ? val : uv);
  if (size < (uint32_t)kMaxKeys) {
    if (!acquire_locks(t, node, h, kNil, 0, false, 0)) return TX_ABORT;
    if (lane <= size && lane < 31) {
      t.keys[(size_t)node * 32 + lane] = nk;
      t.vals[(size_t)node * 32 + lane] = nv;
    }
    __threadfence();
    __syncwarp();
    if (lane == 0) {
      st_release(hdr_ptr(t, node), hdr_next(h, size + 1));
      atomicAdd(&C->n_keys, 1ull);
    }
    __syncwarp();
    ans = 0;
    st = kAbsent;
    return TX_DONE;
  }
  // full leaf: 32 entries split 16 | 16, up = first key of the right half;
  // left fence = up, right keeps the old fence (INSERT_LEAF :413-452)
  const uint64_t old_fence = __shfl_sync(kFull, v, 31);
  const uint64_t up = __shfl_sync(kFull, nk, 16);
  const uint64_t rk0 = __shfl_down_sync(kFull, nk, 16);
  const uint64_t rv0 = __shfl_down_sync(kFull, nv, 16);
  const uint64_t lk = lane < 16 ? nk : kKeyMax;
  const uint64_t lv = lane < 16 ? nv : (lane == 31 ? up : 0);
  const uint64_t rk = lane < 16 ? rk0 : kKeyMax;
  const uint64_t rv = lane < 16 ? rv0 : (lane == 31 ? old_fence : 0);
  const int r = commit_split(t, node, h, lk, lv, hdr_next(h, 16), rk, rv, 16, 0, up, parent, ph,
                             pslot, pk, pv, rl);
  if (r != TX_DONE) return r;
  if (lane == 0) atomicAdd(&C->n_keys, 1ull);
  ans = 0;
  st = kAbsent;
  return TX_DONE;
}

// Optimistic attempt (the idea of the reference's RADICAL_SEARCH_FOR_INSERT,
// src/gpu-stm-tree-v27/bpt-gpustm-kernel-radical-search.cuh:13-266, made
// exact): inner levels are read with plain loads and no validation; only the
// leaf is validated -- seqlock on its header, the tree epoch, and its fences
// low <= key < right fence.  A complete leaf image whose fence range holds the
// key is that key's leaf whatever path led to it, so the answer and an
// in-leaf update are exact.  Splits and failed checks go to tx_attempt.
// FAST_WRONG: the leaf's fences do not cover the key (unlocked unchanged)
enum : int { FAST_DONE = 0, FAST_SLOW = 1, FAST_RETRY = 2, FAST_WRONG = 3 };

// Insert into a candidate leaf by locking it first: CAS its header, then read
// the row under the lock (no concurrent writer can change it), check epoch and
// fences, and apply the update or the shift-insert.  A wrong leaf is unlocked
// unchanged (FAST_WRONG); a full leaf is unlocked unchanged and goes to the
// validated split path.
__device__ int fast_insert_locked(const DevTree& t, const uint32_t epoch, const uint32_t node, const uint64_t key,
                                  const uint64_t val, uint64_t& ans, uint8_t& st) {
  const uint32_t lane = lane_id();
  uint64_t* hp = hdr_ptr(t, node);
  int ok = 0;
  uint64_t h = 0;
  if (lane == 0) {
    h = ld_relaxed(hp);
    if (!hdr_locked(h) && hdr_level(h) == 0 && hdr_epoch(h) == epoch)
      ok = atomicCAS((unsigned long long*)hp, h, hdr_lock(h)) == h;
  }
  ok = __shfl_sync(kFull, ok, 0);
  if (!ok) return FAST_RETRY;
  h = __shfl_sync(kFull, h, 0);
  __threadfence();
  uint64_t k = ld_relaxed(t.keys + (size_t)node * 32 + lane);
  const uint64_t v = ld_relaxed(t.vals + (size_t)node * 32 + lane);
  const uint64_t lo = __shfl_sync(kFull, lane == 0 ? ld_relaxed(t.low + node) : 0, 0);
  const uint64_t fence_key = __shfl_sync(kFull, v, 31);
  const uint32_t size = hdr_size(h);
  if (!(lo <= key && key < fence_key)) {
    if (lane == 0) st_release(hp, h);
    __syncwarp();
    return FAST_WRONG;
  }
  if (lane == 31) k = kKeyMax;
  const uint32_t mm = __ballot_sync(kFull, lane < size && k == key);
  if (mm) {
    const uint32_t at = __ffs(mm) - 1;
    const uint64_t old = __shfl_sync(kFull, v, at);
    if (lane == at) t.vals[(size_t)node * 32 + at] = val;
    __threadfence();
    __syncwarp();
    if (lane == 0) st_release(hp, hdr_next(h, size));
    __syncwarp();
    ans = old;
    st = kFound;
    return FAST_DONE;
  }
  if (size >= (uint32_t)kMaxKeys) {
    if (lane == 0) st_release(hp, h);
    __syncwarp();
    return FAST_SLOW;
  }
  const uint32_t p = __popc(__ballot_sync(kFull, lane < size && k < key));
  const uint64_t uk = __shfl_up_sync(kFull, k, 1);
  const uint64_t uv = __shfl_up_sync(kFull, v, 1);
  const uint64_t nk = lane < p ? k : (lane == p ? key : uk);
  const uint64_t nv = lane < p ? v : (lane == p ? val : uv);
  if (lane <= size && lane < 31) {
    t.keys[(size_t)node * 32 + lane] = nk;
    t.vals[(size_t)node * 32 + lane] = nv;
  }
  __threadfence();
  __syncwarp();
  if (lane == 0) {
    st_release(hp, hdr_next(h, size + 1));
    atomicAdd(&t.ctrl->n_keys, 1ull);
  }
  __syncwarp();
  ans = 0;
  st = kAbsent;
  return FAST_DONE;
}

// DELETE in a candidate leaf, lock first (as fast_insert_locked): a wrong
// leaf is unlocked unchanged (FAST_WRONG); an absent key answers ABSENT.
__device__ int fast_delete_locked(const DevTree& t, const uint32_t epoch, const uint32_t node, const uint64_t key,
                                  uint64_t& ans, uint8_t& st) {
  const uint32_t lane = lane_id();
  uint64_t* hp = hdr_ptr(t, node);
  int ok = 0;
  uint64_t h = 0;
  if (lane == 0) {
    h = ld_relaxed(hp);
    if (!hdr_locked(h) && hdr_level(h) == 0 && hdr_epoch(h) == epoch)
      ok = atomicCAS((unsigned long long*)hp, h, hdr_lock(h)) == h;
  }
  ok = __shfl_sync(kFull, ok, 0);
  if (!ok) return FAST_RETRY;
  h = __shfl_sync(kFull, h, 0);
  __threadfence();
  uint64_t k = ld_relaxed(t.keys + (size_t)node * 32 + lane);
  const uint64_t v = ld_relaxed(t.vals + (size_t)node * 32 + lane);
  const uint64_t lo = __shfl_sync(kFull, lane == 0 ? ld_relaxed(t.low + node) : 0, 0);
  const uint64_t fence_key = __shfl_sync(kFull, v, 31);
  const uint32_t size = hdr_size(h);
  if (!(lo <= key && key < fence_key)) {
    if (lane == 0) st_release(hp, h);
    __syncwarp();
    return FAST_WRONG;
  }
  if (lane == 31) k = kKeyMax;
  const uint32_t mm = __ballot_sync(kFull, lane < size && k == key);
  if (!mm) {
    if (lane == 0) st_release(hp, h);
    __syncwarp();
    ans = 0;
    st = kAbsent;
    return FAST_DONE;
  }
  const uint32_t at = __ffs(mm) - 1;
  const uint64_t old = __shfl_sync(kFull, v, at);
  const uint64_t dk = __shfl_down_sync(kFull, k, 1);
  const uint64_t dv = __shfl_down_sync(kFull, v, 1);
  if (lane >= at && lane < size) {
    const bool last = lane + 1 == size;
    t.keys[(size_t)node * 32 + lane] = last ? kKeyMax : dk;
    t.vals[(size_t)node * 32 + lane] = last ? 0 : dv;
  }
  __threadfence();
  __syncwarp();
  if (lane == 0) {
    st_release(hp, hdr_next(h, size - 1));
    atomicAdd(&t.ctrl->n_keys, ~0ull);  // - 1
  }
  __syncwarp();
  ans = old;
  st = kFound;
  return FAST_DONE;
}

__device__ int tx_fast(const DevTree& t, const uint32_t epoch, const uint64_t key, const uint64_t val,
                       const bool is_insert, const bool is_del, uint64_t& ans, uint8_t& st, const LearnedDev* M) {
  const uint32_t lane = lane_id();
  Ctrl* C = t.ctrl;
  const uint32_t root = ld_relaxed32(&C->root);
  if (root == kNil) return FAST_SLOW;
  // the learned model proposes the leaf; the leaf checks below make any
  // proposal safe, and a miss falls back to the descent
  uint32_t guess = kNil;
  if (M) {
    uint32_t dist = 0;
    guess = learned_leaf<32>(*M, M->params, key, lane, kFull, dist);
    if (guess >= t.cap) guess = kNil;
  }
  // Two passes at most: the proposed leaf, then, when its fences show that
  // it is not the key's leaf (it split after the model was trained), the
  // descent from the root in the same attempt, without an abort.
  for (int pass = 0;; pass++) {
    uint32_t node = guess != kNil ? guess : root;
    for (int depth = 0; guess == kNil; depth++) {
      if (depth > 40 || node >= t.cap) return FAST_SLOW;
      const uint64_t* krow = t.keys + (size_t)node * 32;
      const uint64_t kr = krow[lane];
      const uint64_t hdr = __shfl_sync(kFull, kr, 31);
      if (hdr_level(hdr) == 0) break;
      const uint64_t v = t.vals[(size_t)node * 32 + lane];
      const uint32_t c = __popc(__ballot_sync(kFull, lane < 31 && kr <= key));
      node = (uint32_t)__shfl_sync(kFull, v, c);
    }
    int r;
    if (is_insert) {
      r = fast_insert_locked(t, epoch, node, key, val, ans, st);
    } else if (is_del) {
      r = fast_delete_locked(t, epoch, node, key, ans, st);
    } else {
      // seqlock read of the leaf
      const uint64_t* krow = t.keys + (size_t)node * 32;
      const uint64_t h = ld_acquire(krow + 31);
      uint64_t k = ld_relaxed(krow + lane);
      const uint64_t v = ld_relaxed(t.vals + (size_t)node * 32 + lane);
      const uint64_t lo = ld_relaxed(t.low + node);
      fence_acq_rel();
      const uint64_t h2 = ld_relaxed(krow + 31);
      const uint64_t h_lane0 = __shfl_sync(kFull, h, 0);
      const uint64_t fence_key = __shfl_sync(kFull, v, 31);
      const bool bad = hdr_locked(h) || h2 != h || h != h_lane0 || hdr_level(h) != 0 || hdr_epoch(h) != epoch;
      if (__any_sync(kFull, bad)) return FAST_RETRY;
      if (__any_sync(kFull, !(lo <= key && key < fence_key))) {
        r = FAST_WRONG;
      } else {
        if (lane == 31) k = kKeyMax;
        const uint32_t size = hdr_size(h);
        const uint32_t mm = __ballot_sync(kFull, lane < size && k == key);
        if (mm) {
          ans = __shfl_sync(kFull, v, __ffs(mm) - 1);
          st = kFound;
        } else {
          ans = 0;
          st = kAbsent;
        }
        return FAST_DONE;
      }
    }
    if (r != FAST_WRONG) return r;
    if (guess == kNil || pass > 0) return FAST_RETRY;  // a concurrent split moved the key: retry
    guess = kNil;
  }
}

// A GET by an 8-lane group (lane g owns slots 4g..4g+3), so that a warp
// serves four at once.  Lock-free like tx_fast's read: the descent takes the
// rows as they are, and the leaf is read under its seqlock and checked
// (unlocked and unchanged header, leaf level, current epoch,
// low <= key < right fence), the matched value inside the same window.
// Returns false when a check fails; the caller then runs the request on the
// warp path.
constexpr int kGetG = 8, kGetS = 32 / kGetG;

__device__ bool group_get(const DevTree& t, const uint32_t epoch, const uint64_t key, const uint32_t g,
                          const uint32_t gmask, uint64_t& ans, uint8_t& st) {
  uint32_t node = ld_relaxed32(&t.ctrl->root);
  if (node == kNil) return false;
  uint64_t k[kGetS];
  for (int depth = 0;; depth++) {
    if (depth > 40 || node >= t.cap) return false;
    const ulonglong2* row = reinterpret_cast<const ulonglong2*>(t.keys + (size_t)node * 32 + g * kGetS);
#pragma unroll
    for (int i = 0; i < kGetS / 2; i++) {
      const ulonglong2 w = row[i];
      k[2 * i] = w.x;
      k[2 * i + 1] = w.y;
    }
    const uint64_t hdr = __shfl_sync(gmask, k[kGetS - 1], kGetG - 1, kGetG);
    if (hdr_level(hdr) == 0) break;
    if (g == kGetG - 1) k[kGetS - 1] = kKeyMax;  // slot 31 holds the header
    uint32_t c = 0;
#pragma unroll
    for (int i = 0; i < kGetS; i++) c += (k[i] <= key) ? 1u : 0u;
    c = group_sum<kGetG>(c, gmask);
    node = (uint32_t)t.vals[(size_t)node * 32 + c];
  }
  // the leaf, under its seqlock
  const uint64_t* krow = t.keys + (size_t)node * 32;
  const uint64_t h = ld_acquire(krow + 31);
#pragma unroll
  for (int i = 0; i < kGetS; i++) k[i] = ld_relaxed(krow + g * kGetS + i);
  const uint64_t lo = ld_relaxed(t.low + node);
  const uint64_t fence = ld_relaxed(t.vals + (size_t)node * 32 + 31);
  const uint32_t size = hdr_size(h);
  uint32_t c = 0;
#pragma unroll
  for (int i = 0; i < kGetS; i++) c += (g * kGetS + i < size && k[i] <= key) ? 1u : 0u;
  c = group_sum<kGetG>(c, gmask);
  const uint32_t slot = c > 0 ? c - 1 : 0;
  const uint64_t kk = __shfl_sync(gmask, pick<kGetS>(k, slot % kGetS), slot / kGetS, kGetG);
  const bool found = c > 0 && kk == key;
  uint64_t v = 0;
  if (found) v = ld_relaxed(t.vals + (size_t)node * 32 + slot);
  fence_acq_rel();
  const uint64_t h2 = ld_relaxed(krow + 31);
  const uint64_t h0 = __shfl_sync(gmask, h, 0, kGetG);
  const bool bad = hdr_locked(h) || h2 != h || h != h0 || hdr_level(h) != 0 || hdr_epoch(h) != epoch ||
                   !(lo <= key && key < fence);
  if (group_sum<kGetG>(bad ? 1u : 0u, gmask) != 0) return false;
  ans = found ? v : 0;
  st = found ? kFound : kAbsent;
  return true;
}

// The GETs among requests [b0, b1) (at most 32; request q is list[q], or q
// without a list), four at a time by 8-lane groups.  Returns the bits q - b0
// of the requests left for the warp path: the writes, and the GETs whose
// leaf check failed.  op_override as in stm_kernel.
__device__ uint32_t get_pass(const DevTree& t, const uint32_t epoch, const uint64_t* __restrict__ keys,
                             const uint8_t* __restrict__ ops, const uint32_t op_override,
                             const uint32_t* __restrict__ list, const size_t b0, const size_t b1,
                             uint64_t* __restrict__ out_vals, uint8_t* __restrict__ out_st) {
  const uint32_t lane = lane_id();
  const uint32_t g = lane % kGetG, grp = lane / kGetG;
  const uint32_t gmask = group_mask<kGetG>(lane);
  uint32_t rest = 0;
  for (size_t b = b0; b < b1; b += 32 / kGetG) {
    const size_t q = b + grp;
    bool get = false;
    uint64_t key = 0;
    uint32_t r = 0;
    if (q < b1) {
      r = list ? list[q] : (uint32_t)q;
      key = keys[r];
      const uint32_t op = op_override <= 1 ? op_override : (uint32_t)ops[r];
      get = op == kOpGet && key != kKeyMax;
    }
    bool ok = false;
    uint64_t ans = 0;
    uint8_t st = kAbsent;
    if (get) ok = group_get(t, epoch, key, g, gmask, ans, st);
    if (ok && g == 0) {
      out_vals[r] = ans;
      out_st[r] = st;
    }
    const uint32_t need = __ballot_sync(kFull, g == 0 && q < b1 && !ok);
#pragma unroll
    for (int j = 0; j < 32 / kGetG; j++)
      if ((need >> (j * kGetG)) & 1u) rest |= 1u << (uint32_t)(b - b0 + (size_t)j);
  }
  return rest;
}

struct TxCounters {
  unsigned long long commits = 0, aborts = 0, exhausted = 0;
};

// One request, all 32 lanes: optimistic attempts, then the validated path.
__device__ __forceinline__ void run_request(const DevTree& t, const uint32_t epoch, const uint64_t key,
                                            const uint32_t op, const uint64_t val_in, const uint32_t retry_limit,
                                            uint64_t& ans, uint8_t& st, TxCounters& cnt, const LearnedDev* M) {
  const uint32_t lane = lane_id();
  ans = 0;
  st = kRejected;
  if (key == kKeyMax || op > 2) return;
  const bool ins = (op == kOpInsert);
  const bool del = (op == kOpDelete);
  const uint64_t val = ins ? val_in : 0;
  uint32_t attempts = 0, fails = 0;
  bool done = false;
  // optimistic attempts first; a split or repeated failed checks go to the
  // validated path below
  for (int f = 0; f < 4 && !done; f++) {
    attempts++;
    const int res = tx_fast(t, epoch, key, val, ins, del, ans, st, f == 0 ? M : nullptr);
    if (res == FAST_DONE) {
      if (ins || del) cnt.commits++;
      done = true;
    } else if (res == FAST_SLOW) {
      break;
    } else {
      cnt.aborts++;
    }
  }
  while (!done) {
    if (attempts++ >= retry_limit) {
      st = kRetryExhausted;
      ans = 0;
      cnt.exhausted++;
      if (lane == 0) atomicOr(&t.ctrl->error, kErrRetry);
      break;
    }
    const int res = tx_attempt(t, key, val, ins, del, ans, st);
    if (res == TX_DONE) {
      if (ins) cnt.commits++;
      break;
    }
    if (res == TX_AGAIN) {
      cnt.commits++;
      fails = 0;
      continue;
    }
    if (res == TX_NOCAP) {
      st = kNoCapacity;
      ans = 0;
      break;
    }
    cnt.aborts++;
    fails++;
    if (fails > 2) {
      // exponential backoff with a per-warp, per-attempt jitter so that
      // colliding warps do not retry in step
      const uint32_t jit = (uint32_t)(((key * 0x9E3779B97F4A7C15ull) >> 40) ^ (attempts * 0x85EBCA6Bu)) & 1023u;
      __nanosleep((32u << (fails < 8 ? fails : 8)) + jit);
    }
  }
}

__device__ __forceinline__ void flush_counters(const DevTree& t, const TxCounters& c) {
  if (lane_id() == 0) {
    if (c.commits) atomicAdd(&t.ctrl->commits, c.commits);
    if (c.aborts) atomicAdd(&t.ctrl->aborts, c.aborts);
    if (c.exhausted) atomicAdd(&t.ctrl->retry_exhausted, c.exhausted);
  }
}

__global__ void __launch_bounds__(256, 4) stm_kernel(DevTree t, const uint64_t* __restrict__ keys,
                                                     const uint64_t* __restrict__ vals, const uint8_t* __restrict__ ops,
                                                     uint32_t op_override, const uint32_t* __restrict__ list,
                                                     const uint32_t* __restrict__ n_dev, size_t n_host,
                                                     uint64_t* __restrict__ out_vals, uint8_t* __restrict__ out_st,
                                                     uint32_t retry_limit, LearnedDev lm, int use_learned,
                                                     const uint8_t* __restrict__ skip) {
  const uint32_t lane = lane_id();
  const size_t n = n_dev ? (size_t)*n_dev : n_host;
  const LearnedDev* M = use_learned ? &lm : nullptr;
  const size_t n_warps = ((size_t)gridDim.x * blockDim.x) >> 5;
  TxCounters cnt;
  const uint32_t epoch = t.ctrl->epoch;
  // each warp takes a contiguous run of requests (the reference gives each
  // warp 16 consecutive requests, bpt-gpustm-kernel.cu:41-56): neighbouring
  // keys of a sorted list then land in one warp, not in concurrent warps
  const size_t chunk = (n + n_warps - 1) / n_warps;
  const size_t q_begin = (((size_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5) * chunk;
  const size_t q_end = min(n, q_begin + chunk);
  // in windows of 32: the GETs four at a time (8 lanes each), then the
  // writes and any GET whose leaf check failed on the whole warp (requests of
  // a batch are concurrent transactions, so this order is as good as any)
  const bool all_ins = op_override == kOpInsert;
  for (size_t w0 = q_begin; w0 < q_end; w0 += 32) {
    const size_t w1 = min(q_end, w0 + 32);
    uint32_t rest = all_ins ? (w1 - w0 == 32 ? 0xffffffffu : (1u << (w1 - w0)) - 1u)
                            : get_pass(t, epoch, keys, ops, op_override, list, w0, w1, out_vals, out_st);
    while (rest) {
      const size_t q = w0 + (size_t)(__ffs(rest) - 1);
      rest &= rest - 1;
      const uint32_t r = list ? list[q] : (uint32_t)q;
      const uint32_t op = op_override <= 1 ? op_override : (uint32_t)ops[r];
      if (skip && op == kOpInsert && skip[r]) continue;  // a combined INSERT, answered already
      uint64_t ans;
      uint8_t st;
      run_request(t, epoch, keys[r], op, op == kOpInsert ? vals[r] : 0, retry_limit, ans, st, cnt, M);
      if (lane == 0) {
        out_vals[r] = ans;
        out_st[r] = st;
      }
    }
  }
  flush_counters(t, cnt);
}

// ----------------------------------------------------------- serving ----
// Persistent request loop of the server (bt_serve.cu).  Batches are published
// into a ring of descriptors; `tail` counts published batches and `cursor` is
// the oldest batch that still has unclaimed requests.  Every warp claims
// kServeChunk consecutive requests of the cursor batch, runs them (v39
// meaning: batches in flight together interleave; the chunk's GETs go first,
// four at a time, get_pass), and the warp that
// completes a batch writes its sequence number and the device clock to host
// memory.  A warp that finds no work sleeps; after idle_ns without work (or
// when stop is set) the kernel exits and the host relaunches it on demand.
// descriptor written by the copy engine while the kernel runs: coherent loads
__device__ __forceinline__ ServeDesc load_desc(const ServeDesc* p) {
  static_assert(sizeof(ServeDesc) == 48, "ServeDesc layout");
  const uint64_t* w = reinterpret_cast<const uint64_t*>(p);
  ServeDesc d;
  d.keys = reinterpret_cast<const uint64_t*>(ld_relaxed(w + 0));
  d.vals = reinterpret_cast<const uint64_t*>(ld_relaxed(w + 1));
  d.ops = reinterpret_cast<const uint8_t*>(ld_relaxed(w + 2));
  d.out_vals = reinterpret_cast<uint64_t*>(ld_relaxed(w + 3));
  d.out_st = reinterpret_cast<uint8_t*>(ld_relaxed(w + 4));
  const uint64_t ns = ld_relaxed(w + 5);
  d.n = (uint32_t)ns;
  d.seq = (uint32_t)(ns >> 32);
  return d;
}

__device__ __forceinline__ unsigned long long global_ns() {
  unsigned long long v;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(v));
  return v;
}

__global__ void __launch_bounds__(256, 4) serve_kernel(DevTree t, ServeDev S, uint32_t retry_limit, LearnedDev lm,
                                                       int use_learned) {
  const uint32_t lane = lane_id();
  const LearnedDev* M = use_learned ? &lm : nullptr;
  TxCounters cnt;
  const uint32_t epoch = t.ctrl->epoch;
  // Idle exit is decided on the whole kernel's activity, not the warp's own
  // (a warp that slept through a small batch claimed by others must not count
  // that time as idle), and it is all or nothing: the warp that sees the
  // timeout raises `exiting` and every warp leaves at its next turn, even if
  // work has arrived meanwhile.  Warps that left one by one would leave a
  // kernel of a few warps that new work keeps alive, so the host (which
  // relaunches only when the whole kernel has ended) would never restore the
  // full grid.  The graph clears `exiting` before each launch.
  const unsigned long long t_start = global_ns();
  unsigned long long my_mark = 0;
  for (;;) {
    uint32_t cur = 0, tail = 0, stop = 0, ex = 0;
    if (lane == 0) {
      ex = ld_relaxed32(S.exiting);
      tail = ld_acquire32(S.tail);
      cur = ld_relaxed32(S.cursor);
      stop = ld_relaxed32(S.stop);
    }
    if (__shfl_sync(kFull, ex, 0)) break;  // the kernel is ending: later work waits for the relaunch
    cur = __shfl_sync(kFull, cur, 0);
    tail = __shfl_sync(kFull, tail, 0);
    stop = __shfl_sync(kFull, stop, 0);
    if (cur >= tail) {
      if (stop) break;
      int leave = 0;
      if (lane == 0) {
        const unsigned long long now = global_ns();
        unsigned long long busy = ld_relaxed(reinterpret_cast<const uint64_t*>(S.last_busy));
        if (busy < t_start) busy = t_start;
        leave = now - busy > S.idle_ns;
        if (leave) atomicExch(S.exiting, 1u);
      }
      if (__shfl_sync(kFull, leave, 0)) break;
      __nanosleep(2000);
      continue;
    }
    if (lane == 0) {
      const unsigned long long now = global_ns();
      if (now - my_mark > 20000) {  // publish activity at most every 20 us per warp
        my_mark = now;
        atomicMax(S.last_busy, now);
      }
    }
    // the batch to claim from: the oldest one with unclaimed requests, or
    // (policy 1) the one with the fewest unclaimed requests among the
    // kServeWindow oldest, so that a large batch does not hold the small
    // ones behind it (shortest remaining work first)
    uint32_t pick = cur;
    if (S.policy == 1) {
      if (lane == 0) {
        uint32_t best = 0xFFFFFFFFu;
        const uint32_t lim = tail - cur > (uint32_t)kServeWindow ? cur + (uint32_t)kServeWindow : tail;
        for (uint32_t q = cur; q != lim; q++) {
          const uint32_t sq = q % S.cap;
          const uint64_t ns = ld_relaxed(reinterpret_cast<const uint64_t*>(S.desc + sq) + 5);
          const unsigned long long cw = ld_relaxed(reinterpret_cast<const uint64_t*>(S.claimed + sq));
          if ((uint32_t)(ns >> 32) != q || (uint32_t)(cw >> 32) != q) continue;  // not this batch's yet
          const uint32_t dn = (uint32_t)ns, cl = (uint32_t)cw;
          if (cl >= dn) {
            if (q == cur) atomicCAS(S.cursor, cur, cur + 1);  // the oldest is fully claimed
            continue;
          }
          if (dn - cl < best) {
            best = dn - cl;
            pick = q;
          }
        }
      }
      pick = __shfl_sync(kFull, pick, 0);
    }
    const uint32_t slot = pick % S.cap;
    // Claim kServeChunk requests with one atomicAdd on the slot's word
    // (batch seq << 32 | requests claimed); every claim succeeds, so thousands
    // of warps do not serialise on a compare-and-swap.  The returned tag names
    // the batch the claim landed in: normally `cur`; if the host has already
    // retired `cur` and reused the slot for a newer batch, the claim belongs to
    // that batch, and this warp runs exactly that range once its descriptor
    // has landed, so no claimed range is ever dropped or run twice.
    unsigned long long w = 0;
    if (lane == 0) {
      const uint32_t dseq = (uint32_t)(ld_relaxed(reinterpret_cast<const uint64_t*>(S.desc + slot) + 5) >> 32);
      if (dseq == pick) w = atomicAdd(S.claimed + slot, (unsigned long long)kServeChunk);
      else w = ~0ull;  // descriptor of `pick` not visible yet, or slot already reused
    }
    w = __shfl_sync(kFull, w, 0);
    if (w == ~0ull) {
      __nanosleep(200);
      continue;
    }
    const uint32_t tag = (uint32_t)(w >> 32);
    const uint32_t c = (uint32_t)w;
    ServeDesc d;
    bool have = true;
    if (lane == 0) {
      d = load_desc(S.desc + slot);
      // a claim in a newer batch: wait (bounded) for its descriptor
      uint32_t spins = 0;
      while (d.seq != tag && spins < (1u << 20)) {
        __nanosleep(256);
        spins++;
        d = load_desc(S.desc + slot);
      }
      if (d.seq != tag) {
        atomicOr(&t.ctrl->error, kErrSpin);
        have = false;
      }
    }
    have = __shfl_sync(kFull, have ? 1 : 0, 0);
    if (!have) continue;
    d.keys = (const uint64_t*)__shfl_sync(kFull, (unsigned long long)d.keys, 0);
    d.vals = (const uint64_t*)__shfl_sync(kFull, (unsigned long long)d.vals, 0);
    d.ops = (const uint8_t*)__shfl_sync(kFull, (unsigned long long)d.ops, 0);
    d.out_vals = (uint64_t*)__shfl_sync(kFull, (unsigned long long)d.out_vals, 0);
    d.out_st = (uint8_t*)__shfl_sync(kFull, (unsigned long long)d.out_st, 0);
    d.n = __shfl_sync(kFull, d.n, 0);
    d.seq = __shfl_sync(kFull, d.seq, 0);
    if (c >= d.n) {
      if (lane == 0 && tag == cur) atomicCAS(S.cursor, cur, cur + 1);
      continue;
    }
    if (c == 0 && lane == 0) S.host_tclaim[slot] = global_ns();  // the batch's first claim
    const uint32_t end = min(d.n, c + (uint32_t)kServeChunk);
    // GETs first, four at a time (8 lanes each); the writes and any GET whose
    // leaf check failed then run one at a time on the whole warp.  Requests
    // of a batch are concurrent transactions, so this order is as good as any.
    uint32_t rest = get_pass(t, epoch, d.keys, d.ops, 0xFF, nullptr, c, end, d.out_vals, d.out_st);
    while (rest) {
      const uint32_t q = c + (uint32_t)(__ffs(rest) - 1);
      rest &= rest - 1;
      uint64_t ans;
      uint8_t st;
      const uint32_t op = d.ops[q];
      run_request(t, epoch, d.keys[q], op, op == kOpInsert ? d.vals[q] : 0, retry_limit, ans, st, cnt, M);
      if (lane == 0) {
        d.out_vals[q] = ans;
        d.out_st[q] = st;
      }
    }
    if (lane == 0) {
      __threadfence();
      const uint32_t prev = atomicAdd(&S.done[slot], end - c);
      if (prev + (end - c) == d.n) {
        __threadfence_system();
        S.host_tend[slot] = global_ns();
        asm volatile("st.release.sys.global.u32 [%0], %1;" ::"l"(S.host_done + slot), "r"(d.seq) : "memory");
      }
    }
    __syncwarp();
  }
  flush_counters(t, cnt);
}

}  // namespace

cudaError_t launch_serve(Handle* h, const ServeDev& S, cudaStream_t s) {
  static int per_sm[64] = {};
  if (h->device < 64 && per_sm[h->device] == 0) {
    int b = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b, serve_kernel, 256, 0) != cudaSuccess || b < 1) b = 2;
    per_sm[h->device] = b;
  }
  const unsigned blocks = (unsigned)(h->sm_count * (h->device < 64 ? per_sm[h->device] : 2));
  LearnedDev lm{};
  const int use = learned_dev(h, &lm);
  h->pfx_valid = false;  // STM writes inner rows without their prefixes
  serve_kernel<<<blocks, 256, 0, s>>>(h->tree, S, h->retry_limit, lm, use);
  count_launch();
  return cudaGetLastError();
}

cudaError_t launch_stm(Handle* h, const uint64_t* keys, const uint64_t* vals, const uint8_t* ops, uint8_t op_override,
                       const uint32_t* list, const uint32_t* n_dev, size_t n, uint64_t* out_vals, uint8_t* out_st,
                       cudaStream_t s, const uint8_t* skip) {
  if (n == 0) return cudaSuccess;
  const int threads = 256;  // 8 warps
  // one resident wave: every warp runs at once, each on a contiguous run
  static int per_sm[64] = {};
  if (h->device < 64 && per_sm[h->device] == 0) {
    int b = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b, stm_kernel, threads, 0) != cudaSuccess || b < 1) b = 2;
    per_sm[h->device] = b;
  }
  size_t blocks = (n * 32 + threads - 1) / threads;
  const size_t cap = (size_t)h->sm_count * (h->device < 64 ? per_sm[h->device] : 2);
  if (blocks > cap) blocks = cap;
  LearnedDev lm{};
  const int use = learned_dev(h, &lm);
  h->pfx_valid = false;  // STM writes inner rows without their prefixes
  stm_kernel<<<(unsigned)blocks, threads, 0, s>>>(h->tree, keys, vals, ops, op_override, list, n_dev, n, out_vals,
                                                   out_st, h->retry_limit, lm, use, skip);
  count_launch();
  return cudaGetLastError();
}

// A BT_MODE_STM batch.  Its requests are concurrent transactions (the v39
// meaning), so any serial order of them is a valid outcome; this one puts
// every valid GET first.  Phase 1 answers the GETs with the batch lookup
// kernels over the pre-batch tree (learned or plain, as the sorted batches):
// no writer runs beside them, so they need none of the STM path's seqlock
// validation.  Phase 2 runs the rest (INSERT, DELETE, invalid requests) as
// STM transactions over their list, the INSERTs of one key combined
// (BT_OPT_STM_COMBINE).  The reference interleaves GETs and writes in one
// kernel (src/gpu-stm-tree-v39/bpt-gpustm-kernel.cu:14-256).
int batch_stm(Handle* h, const uint64_t* keys, const uint64_t* vals, const uint8_t* ops, uint64_t* out_vals,
              uint8_t* out_st, size_t n, cudaStream_t s) {
  if (n == 0) return 0;
  Work& w = h->w;
  if (n > w.cap) return -6;
  const bool learned = batch_learned(h, h->batch_descent >= 0 ? h->batch_descent : h->descent, s);
  if (stm_split(h, keys, ops, n, s) != 0) return -2;
  BatchCounts* c = w.counts;
  const cudaError_t e = learned
                            ? launch_learned_lookup(h, keys, w.get_list, &c->n_lookup, n, out_vals, out_st, s, w.ukeys,
                                                    true)
                            : launch_search(h, keys, w.get_list, &c->n_lookup, n, out_vals, out_st, s, w.ukeys);
  if (e != cudaSuccess) return -2;
  if (learned) learned_sample(h, s);
  const uint8_t* skip = nullptr;
  const uint64_t* run_vals = vals;
  if (h->stm_combine && stm_combine(h, keys, vals, ops, n, out_vals, out_st, s, &skip, &run_vals) != 0) return -2;
  if (launch_stm(h, keys, run_vals, ops, 0xFF, w.ins_list, &c->n_ins_req, n, out_vals, out_st, s, skip) !=
      cudaSuccess)
    return -2;
  if (h->stm_combine && stm_combine_fixup(h, ops, n, out_vals, out_st, s) != 0) return -2;
  return 0;
}

}  // namespace bt
