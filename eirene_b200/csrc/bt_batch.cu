// Sort-based batch merge (the reference's v38 front end and back end,
// src/gpu-stm-tree-v38/bpt-gpustm-kernel.cu:289-332 and
// src/gpu-stm-tree-v38/bpt-gpustm-kernel-aux.cuh:16-56), restated for B200:
//
//   sort (key, idx|op)        hand-written radix sort (bt_sort.cu)
//   tile pass 1 / 2 / 3       one segmented scan over the sorted requests
//                             replaces RunLengthEncode + ExclusiveSum +
//                             mergeMission; it is parallel per request, so a
//                             Zipf-hot key with 10^5 repeats costs no more than
//                             10^5 distinct keys (mergeMission walks each run
//                             with one thread).
//   search phase              lock-free grouped search over the unique GETs
//   insert phase              STM kernel over the unique INSERTs
//   writeback                 scatter answers to request order
//
// Meaning (identical to v38): within a run of equal keys in input order a
// request sees the pre-batch value until the first INSERT, then the value of
// the latest INSERT before it; the run reaches the tree as one INSERT (last
// value) or one GET.  The unique count never leaves the device (the reference
// copies it to the host and synchronises, v38 bpt-gpustm-kernel.cu:303-306).
#include <utility>

#include <cuda_runtime.h>

#include "bt_block.cuh"
#include "bt_common.cuh"
#include "bt_internal.h"

namespace bt {

struct TileSummary {
  uint64_t agg_v;
  uint64_t pre_v;
  uint64_t carry_v;
  uint32_t agg_f;
  uint32_t pre_f;
  uint32_t carry_f;
  uint32_t heads;
  uint32_t cont;  // bit0: tile holds the tail of a run begun in an earlier tile; bit1: that key is reserved
  uint32_t ins_local;
  uint32_t get_local;
  uint32_t del_local;
  uint32_t heads_before;
  uint32_t ins_before;
  uint32_t get_before;
  uint32_t del_before;
};

namespace {

constexpr int kThreads = 512;
constexpr int kItems = 8;
constexpr int kTile = kThreads * kItems;

inline size_t pass_tiles(size_t n) { return (n + kTile - 1) / kTile; }
constexpr uint32_t kIdxMask = 0x3FFFFFFFu;
constexpr uint32_t kResolved = 0xFFFFFFFFu;

struct Item {
  uint64_t k;
  uint32_t r;
  uint32_t op;
  bool head, tail, valid, wr, del;  // wr: INSERT or DELETE of a usable key
};

__device__ __forceinline__ void load_items(const uint64_t* __restrict__ sk, const uint32_t* __restrict__ sv,
                                           size_t n, size_t i0, Item (&it)[kItems]) {
  uint64_t prev = (i0 > 0 && i0 - 1 < n) ? sk[i0 - 1] : 0;
#pragma unroll
  for (int j = 0; j < kItems; j++) {
    const size_t i = i0 + j;
    it[j].valid = i < n;
    if (i < n) {
      it[j].k = sk[i];
      const uint32_t p = sv[i];
      it[j].r = p & kIdxMask;
      it[j].op = p >> 30;
      it[j].head = (i == 0) || (prev != it[j].k);
      prev = it[j].k;
    } else {
      it[j].k = 0;
      it[j].r = 0;
      it[j].op = 3;
      it[j].head = false;
    }
  }
#pragma unroll
  for (int j = 0; j < kItems; j++) {
    const size_t i = i0 + j;
    if (i < n) {
      const uint64_t nx = (j + 1 < kItems) ? it[j + 1].k : (i + 1 < n ? sk[i + 1] : 0);
      it[j].tail = (i + 1 == n) || (nx != it[j].k) || (j + 1 < kItems && !it[j + 1].valid);
      it[j].wr = (it[j].op == kOpInsert || it[j].op == kOpDelete) && it[j].k != kKeyMax;
      it[j].del = it[j].op == kOpDelete;
    } else {
      it[j].tail = false;
      it[j].wr = false;
      it[j].del = false;
    }
  }
}

__device__ __forceinline__ Seg item_seg(const Item& x, const uint64_t* __restrict__ vals) {
  Seg s;
  s.f = x.head ? 1u : 0u;
  s.v = 0;
  if (x.valid && x.wr) {
    s.f |= x.del ? 6u : 2u;
    s.v = x.del ? 0 : vals[x.r];
  }
  return s;
}

// pass 1: per tile aggregate, head count, locally determined tail counts and
// the state at the tail of the run continued from the previous tile
__global__ void __launch_bounds__(kThreads) merge_pass1(const uint64_t* __restrict__ sk,
                                                        const uint32_t* __restrict__ sv,
                                                        const uint64_t* __restrict__ vals, size_t n,
                                                        const uint32_t* __restrict__ n_dev,
                                                        TileSummary* __restrict__ tiles) {
  if (n_dev) n = min(n, (size_t)*n_dev);
  if ((size_t)blockIdx.x * kTile >= n) return;  // grid sized for the host bound
  __shared__ uint32_t wsf[32];
  __shared__ uint64_t wsv[32];
  __shared__ uint32_t ws[32];
  __shared__ uint64_t s_pre_v;
  __shared__ uint32_t s_pre_f, s_cont;
  if (threadIdx.x == 0) {
    s_cont = 0;
    s_pre_f = 0;
    s_pre_v = 0;
  }
  const size_t i0 = (size_t)blockIdx.x * kTile + (size_t)threadIdx.x * kItems;
  Item it[kItems];
  load_items(sk, sv, n, i0, it);
  Seg seg[kItems];
  Seg tagg{0, 0};
  uint32_t heads = 0;
#pragma unroll
  for (int j = 0; j < kItems; j++) {
    seg[j] = item_seg(it[j], vals);
    tagg = seg_combine(tagg, seg[j]);
    heads += it[j].head ? 1u : 0u;
  }
  Seg agg;
  Seg st = blk_exclusive_seg(tagg, Seg{0, 0}, wsf, wsv, &agg);
  uint32_t ins_l = 0, get_l = 0, del_l = 0;
#pragma unroll
  for (int j = 0; j < kItems; j++) {
    st = seg_combine(st, seg[j]);
    if (it[j].valid && it[j].tail) {
      if (st.f & 1u) {  // run began inside this tile
        if (it[j].k != kKeyMax) {
          if (st.f & 4u) del_l++;
          else if (st.f & 2u) ins_l++;
          else get_l++;
        }
      } else {  // tail of the run continued from the previous tile
        s_cont = 1u | (it[j].k == kKeyMax ? 2u : 0u);
        s_pre_f = st.f;
        s_pre_v = st.v;
      }
    }
  }
  uint32_t th, ti, tg, td;
  blk_exclusive_sum(heads, ws, &th);
  blk_exclusive_sum(ins_l, ws, &ti);
  blk_exclusive_sum(get_l, ws, &tg);
  blk_exclusive_sum(del_l, ws, &td);
  if (threadIdx.x == 0) {
    TileSummary& T = tiles[blockIdx.x];
    T.agg_f = agg.f;
    T.agg_v = agg.v;
    T.heads = th;
    T.ins_local = ti;
    T.get_local = tg;
    T.del_local = td;
    T.cont = s_cont;
    T.pre_f = s_pre_f;
    T.pre_v = s_pre_v;
  }
}

// pass 2 (one block): carries and prefix counts across tiles; writes totals
__global__ void __launch_bounds__(1024) merge_pass2(TileSummary* __restrict__ tiles, uint32_t n_tiles,
                                                    const uint32_t* __restrict__ n_dev,
                                                    BatchCounts* __restrict__ counts) {
  if (n_dev) n_tiles = min(n_tiles, (uint32_t)(((size_t)*n_dev + kTile - 1) / kTile));
  __shared__ uint32_t wsf[32];
  __shared__ uint64_t wsv[32];
  __shared__ uint32_t ws[32];
  const uint32_t per = (n_tiles + blockDim.x - 1) / blockDim.x;
  const uint32_t t0 = threadIdx.x * per;
  const uint32_t t1 = min(n_tiles, t0 + per);
  Seg a{0, 0};
  uint32_t hsum = 0;
  for (uint32_t t = t0; t < t1; t++) {
    a = seg_combine(a, Seg{tiles[t].agg_f, tiles[t].agg_v});
    hsum += tiles[t].heads;
  }
  Seg carry = blk_exclusive_seg(a, Seg{0, 0}, wsf, wsv, nullptr);
  uint32_t htot;
  uint32_t hb = blk_exclusive_sum(hsum, ws, &htot);
  uint32_t isum = 0, gsum = 0, dsum = 0;
  for (uint32_t t = t0; t < t1; t++) {
    TileSummary& T = tiles[t];
    T.carry_f = carry.f;
    T.carry_v = carry.v;
    T.heads_before = hb;
    hb += T.heads;
    uint32_t ic = T.ins_local, gc = T.get_local, dc = T.del_local;
    if ((T.cont & 1u) && !(T.cont & 2u)) {
      const Seg s = seg_combine(carry, Seg{T.pre_f, T.pre_v});
      if (s.f & 4u) dc++;
      else if (s.f & 2u) ic++;
      else gc++;
    }
    T.ins_before = ic;  // per-tile counts for now
    T.get_before = gc;
    T.del_before = dc;
    isum += ic;
    gsum += gc;
    dsum += dc;
    carry = seg_combine(carry, Seg{T.agg_f, T.agg_v});
  }
  uint32_t itot, gtot, dtot;
  uint32_t ib = blk_exclusive_sum(isum, ws, &itot);
  uint32_t gb = blk_exclusive_sum(gsum, ws, &gtot);
  uint32_t db = blk_exclusive_sum(dsum, ws, &dtot);
  for (uint32_t t = t0; t < t1; t++) {
    TileSummary& T = tiles[t];
    const uint32_t ic = T.ins_before, gc = T.get_before, dc = T.del_before;
    T.ins_before = ib;
    T.get_before = gb;
    T.del_before = db;
    ib += ic;
    gb += gc;
    db += dc;
  }
  if (threadIdx.x == 0) {
    counts->n_unique = htot;
    counts->n_ins = itot;
    counts->n_get = gtot;
    counts->n_del = dtot;
  }
}

// pass 3: per request resolution, unique ops and the two work lists
__global__ void __launch_bounds__(kThreads) merge_pass3(
    const uint64_t* __restrict__ sk, const uint32_t* __restrict__ sv, const uint64_t* __restrict__ vals, size_t n,
    const uint32_t* __restrict__ n_dev, const TileSummary* __restrict__ tiles, uint64_t* __restrict__ ukeys,
    uint64_t* __restrict__ uvals, uint32_t* __restrict__ ins_list, uint32_t* __restrict__ get_list,
    uint32_t* __restrict__ del_list, uint32_t* __restrict__ pend, uint64_t* __restrict__ out_vals,
    uint8_t* __restrict__ out_st) {
  if (n_dev) n = min(n, (size_t)*n_dev);
  if ((size_t)blockIdx.x * kTile >= n) return;
  __shared__ uint32_t wsf[32];
  __shared__ uint64_t wsv[32];
  __shared__ uint32_t ws[32];
  const TileSummary& T = tiles[blockIdx.x];
  const size_t i0 = (size_t)blockIdx.x * kTile + (size_t)threadIdx.x * kItems;
  Item it[kItems];
  load_items(sk, sv, n, i0, it);
  Seg seg[kItems];
  Seg tagg{0, 0};
  uint32_t heads = 0;
#pragma unroll
  for (int j = 0; j < kItems; j++) {
    seg[j] = item_seg(it[j], vals);
    tagg = seg_combine(tagg, seg[j]);
    heads += it[j].head ? 1u : 0u;
  }
  Seg st = blk_exclusive_seg(tagg, Seg{T.carry_f, T.carry_v}, wsf, wsv, nullptr);
  // tail kinds with the true carry
  uint32_t n_ins = 0, n_get = 0, n_del = 0;
  {
    Seg s = st;
#pragma unroll
    for (int j = 0; j < kItems; j++) {
      s = seg_combine(s, seg[j]);
      if (it[j].valid && it[j].tail && it[j].k != kKeyMax) {
        if (s.f & 4u) n_del++;
        else if (s.f & 2u) n_ins++;
        else n_get++;
      }
    }
  }
  uint32_t hpos = blk_exclusive_sum(heads, ws, nullptr) + T.heads_before;
  uint32_t ipos = blk_exclusive_sum(n_ins, ws, nullptr) + T.ins_before;
  uint32_t gpos = blk_exclusive_sum(n_get, ws, nullptr) + T.get_before;
  uint32_t dpos = blk_exclusive_sum(n_del, ws, nullptr) + T.del_before;
  // hpos counts heads strictly before this thread's first item
#pragma unroll
  for (int j = 0; j < kItems; j++) {
    if (!it[j].valid) break;
    const size_t i = i0 + j;
    if (it[j].head) hpos++;
    const uint32_t u = hpos - 1;  // unique id of this item's run
    const bool ok = it[j].k != kKeyMax && it[j].op <= 2u;
    if (!ok) {
      out_vals[it[j].r] = 0;
      out_st[it[j].r] = kRejected;
      pend[i] = kResolved;
    } else if (!it[j].head && (st.f & 2u)) {  // an earlier write of this same run
      const bool gone = (st.f & 4u) != 0;
      out_vals[it[j].r] = gone ? 0 : st.v;
      out_st[it[j].r] = gone ? kAbsent : kFound;
      pend[i] = kResolved;
    } else {
      pend[i] = u;
    }
    st = seg_combine(st, seg[j]);
    if (it[j].tail && it[j].k != kKeyMax) {
      ukeys[u] = it[j].k;
      uvals[u] = st.v;
      if (st.f & 4u) del_list[dpos++] = u;
      else if (st.f & 2u) ins_list[ipos++] = u;
      else get_list[gpos++] = u;
    }
  }
}

__global__ void writeback_kernel(const uint32_t* __restrict__ sv, const uint32_t* __restrict__ pend, size_t n,
                                 const uint32_t* __restrict__ n_dev, const uint64_t* __restrict__ uans,
                                 const uint8_t* __restrict__ uans_st, uint64_t* __restrict__ out_vals,
                                 uint8_t* __restrict__ out_st) {
  if (n_dev) n = min(n, (size_t)*n_dev);
  const size_t stride = (size_t)gridDim.x * blockDim.x;
  for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) {
    const uint32_t u = pend[i];
    if (u != kResolved) {
      const uint32_t r = sv[i] & kIdxMask;
      out_vals[r] = uans[u];
      out_st[r] = uans_st[u];
    }
  }
}

}  // namespace

int work_alloc(Work* w, size_t cap) {
  work_free(w);
  if (cap == 0) cap = 1;
  const size_t tiles = pass_tiles(cap);
  bool ok = true;
  auto A = [&](void** p, size_t bytes) {
    if (ok && cudaMalloc(p, bytes) != cudaSuccess) ok = false;
  };
  A((void**)&w->k_a, cap * 8);
  A((void**)&w->k_b, cap * 8);
  A((void**)&w->v_a, cap * 4);
  A((void**)&w->v_b, cap * 4);
  A((void**)&w->sort_scratch, sort_scratch_words(cap) * 4);
  A((void**)&w->ukeys, cap * 8);
  A((void**)&w->uvals, cap * 8);
  A((void**)&w->uans, cap * 8);
  A((void**)&w->uans_st, cap);
  A((void**)&w->ins_list, cap * 4);
  A((void**)&w->get_list, cap * 4);
  A((void**)&w->del_list, cap * 4);
  A((void**)&w->pend, cap * 4);
  A((void**)&w->tiles, tiles * sizeof(TileSummary));
  A((void**)&w->counts, sizeof(BatchCounts));
  A((void**)&w->m_path, cap * 32);
  A((void**)&w->m_vpos, cap * 8);
  A((void**)&w->m_leaf, cap * 4);
  A((void**)&w->m_isnew, cap * 4);
  A((void**)&w->m_pos, cap * 4);
  A((void**)&w->m_newk, cap * 8);
  A((void**)&w->m_newv, cap * 8);
  A((void**)&w->m_nq, cap * 4 + 64);
  A((void**)&w->m_nleaf, cap * 4);
  A((void**)&w->m_seg, cap * 4);
  A((void**)&w->d_leaf, cap * 4);
  A((void**)&w->d_slot, cap * 4);
  A((void**)&w->m_ent_a, cap * 16);
  A((void**)&w->m_ent_b, cap * 16);
  A((void**)&w->m_counts, 64);
  A(&w->m_sync, 8192);
  A((void**)&w->ins_ops, cap);
  {
    size_t tc = 1024;
    while (tc < 2 * cap) tc <<= 1;
    A(&w->f_tab, tc * 16);
    w->f_tab_cap = tc;
  }
  A((void**)&w->f_flags, cap * 4);
  A((void**)&w->f_pos, cap * 4);
  A((void**)&w->f_list, cap * 4);
  A((void**)&w->f_lk, cap * 8);
  A((void**)&w->f_tk, cap * 8);
  A((void**)&w->f_tv, cap * 4);
  A((void**)&w->lb_status, scan_lb_words(cap) * 8);
  A((void**)&w->lb_ctr, 8);
  ok = ok && cudaMemset(w->lb_status, 0, scan_lb_words(cap) * 8) == cudaSuccess &&
       cudaMemset(w->lb_ctr, 0, 8) == cudaSuccess;
  if (!ok) {
    work_free(w);
    return -3;
  }
  w->cap = cap;
  return 0;
}

// the fields of Work that make up a BatchSet
#define BT_SET_FIELDS(X) X(tiles) X(counts) X(f_list) X(f_lk) X(ukeys) X(uvals) X(ins_list) X(get_list) X(del_list) X(pend) \
  X(k_a) X(k_b) X(v_a) X(v_b)

void work_swap_set(Work* w) {
#define BT_SWAP(f) std::swap(w->f, w->alt.f);
  BT_SET_FIELDS(BT_SWAP)
#undef BT_SWAP
  w->alt_in = !w->alt_in;
}

int work_alt_alloc(Work* w) {
  if (w->alt.counts) return 0;
  const size_t cap = w->cap;
  BatchSet& a = w->alt;
  bool ok = cudaMalloc((void**)&a.tiles, pass_tiles(cap) * sizeof(TileSummary)) == cudaSuccess &&
            cudaMalloc((void**)&a.counts, sizeof(BatchCounts)) == cudaSuccess &&
            cudaMalloc((void**)&a.f_list, cap * 4) == cudaSuccess && cudaMalloc((void**)&a.f_lk, cap * 8) == cudaSuccess &&
            cudaMalloc((void**)&a.ukeys, cap * 8) == cudaSuccess && cudaMalloc((void**)&a.uvals, cap * 8) == cudaSuccess &&
            cudaMalloc((void**)&a.ins_list, cap * 4) == cudaSuccess &&
            cudaMalloc((void**)&a.get_list, cap * 4) == cudaSuccess &&
            cudaMalloc((void**)&a.del_list, cap * 4) == cudaSuccess &&
            cudaMalloc((void**)&a.pend, cap * 4) == cudaSuccess && cudaMalloc((void**)&a.k_a, cap * 8) == cudaSuccess &&
            cudaMalloc((void**)&a.k_b, cap * 8) == cudaSuccess && cudaMalloc((void**)&a.v_a, cap * 4) == cudaSuccess &&
            cudaMalloc((void**)&a.v_b, cap * 4) == cudaSuccess;
  if (!ok) {
#define BT_FREE_ALT(f) cudaFree(a.f);
    BT_SET_FIELDS(BT_FREE_ALT)
#undef BT_FREE_ALT
    a = BatchSet{};
    return -3;
  }
  return 0;
}

void work_free(Work* w) {
  if (w->alt_in) work_swap_set(w);  // the fields hold the first set again
  {
    BatchSet& a = w->alt;
#define BT_FREE_ALT(f) if (a.f) cudaFree(a.f);
    BT_SET_FIELDS(BT_FREE_ALT)
#undef BT_FREE_ALT
    a = BatchSet{};
  }
  void* ps[] = {w->k_a,      w->k_b,       w->v_a,       w->v_b,       w->sort_scratch, w->ukeys,   w->uvals,
                w->uans,     w->uans_st,   w->ins_list,  w->get_list,  w->del_list, w->pend,         w->tiles,   w->counts,
                w->m_path,   w->m_vpos,   w->m_leaf,    w->m_isnew,   w->m_pos,     w->m_newk,       w->m_newv,  w->m_nq,
                w->m_nleaf,  w->m_seg,     w->d_leaf,    w->d_slot,    w->m_ent_a,   w->m_ent_b,   w->m_counts,     w->m_sync,
                w->ins_ops,  w->f_tab, w->f_flags,
                w->f_pos,    w->f_list,    w->f_lk,      w->f_tk,      w->f_tv,      w->lb_status, w->lb_ctr};
  for (void* p : ps)
    if (p) cudaFree(p);
  *w = Work{};
}

static bool merge_usable(const Handle* h, int engine) {
  // the merge engine needs leaf_fill >= 16 and inner_fill >= 16: then a split
  // emits at most one separator per new key or entry, which bounds its buffers
  return engine == 1 && h->leaf_fill >= 16 && h->inner_fill >= 16;
}

// write phase shared by both front ends: the unique DELETE runs (w.del_list,
// count w.counts->n_del), then the unique INSERT runs of (w.ukeys, w.uvals,
// w.ins_list, count w.counts->n_ins) reach the tree.
static int insert_phase(Handle* h, size_t n, int engine, cudaStream_t s) {
  Work& w = h->w;
  // the DELETE runs first: their keys differ from the INSERT runs' keys
  if (delete_locate(h, n, s) != 0) return -2;
  if (delete_apply(h, n, s) != 0) return -2;
  if (merge_usable(h, engine)) return merge_engine(h, n, s) != 0 ? -2 : 0;
  const cudaError_t e =
      launch_stm(h, w.ukeys, w.uvals, nullptr, kOpInsert, w.ins_list, &w.counts->n_ins, n, w.uans, w.uans_st, s);
  return e == cudaSuccess ? 0 : -2;
}

static int wait_vals(Handle* h, cudaStream_t s) {
  return h->vals_wait && cudaStreamWaitEvent(s, h->vals_wait, 0) != cudaSuccess ? -2 : 0;
}

static int answers_ready(Handle* h, cudaStream_t s) {
  return h->ans_ready && cudaEventRecord(h->ans_ready, s) != cudaSuccess ? -2 : 0;
}

// The hash front end (bt_front.cu): only the requests coupled by a write of
// their key are sorted and merged; the rest are plain lookups of the
// pre-batch tree, answered in place.  Same meaning as the full-sort path.
//
// Streams (overlap on): `s` runs the front end, the touched requests' sort
// and merge passes, then the lookups; with the merge engine a high-priority
// side stream runs the two locates and the grouping of the new keys by leaf
// beside the lookups (the locates only read the pre-batch tree: a plain
// lookup may ask for a key that a later request of the batch writes).  `s`
// then waits for the side stream, writes the new values of existing keys,
// applies the DELETE runs, reserves the leaf pieces (a full node pool
// answers kNoCapacity here) and writes the touched answers back: every
// answer is final before the leaf merge.  With async_write the leaf
// and inner merge run on tree_stream, so the caller's stream goes on to the
// next batch, whose front end and sort need neither the tree nor the merge
// scratch; its first tree access waits for tree_ev.
//
// A hash-front-end batch in two parts.  The front part reads no tree: the
// classification, the touched requests' sort and (unless they wait for the
// values on the side stream) the merge passes.  The tree part does the
// rest.  A single batch runs them back to back on `s`; bt_execute_batches
// runs batch j + 1's front part on its own stream beside batch j's tree
// part, each batch with its set of the buffers the two parts share
// (Work::sets).
struct FrontPart {
  uint64_t* sk = nullptr;
  uint32_t* sv = nullptr;
  uint32_t n_tiles = 0;
  bool passes_done = false;
};

static int hashed_front(Handle* h, const uint64_t* keys, const uint64_t* vals, const uint8_t* ops, uint64_t* out_vals,
                        uint8_t* out_st, size_t n, cudaStream_t s, bool passes, FrontPart& fp,
                        cudaEvent_t vals_ready = nullptr) {
  Work& w = h->w;
  BatchCounts* c = w.counts;
  const uint32_t* n_touch = &c->n_touch;
  if (front_classify(h, keys, ops, n, s) != 0) return -2;
  // the touched requests' sort and merge passes need no tree: they run at
  // full width (beside the previous batch's deferred merge)
  // the merge sort while the touched counts are small (the count of a batch
  // that ran before: a hint, both sorts give the same order)
  bool merge = h->touch_sort == 1;
  if (h->touch_sort == 2 && h->touch_hint)
    merge = *reinterpret_cast<volatile const uint32_t*>(h->touch_hint) <= kMergeSortMax;
  const cudaError_t se =
      merge
          ? merge_sort_pairs(w.f_tk, w.f_tv, w.k_a, w.v_a, w.k_b, w.v_b, n, n_touch, h->sm_count, s, &fp.sk, &fp.sv)
          : radix_sort_pairs(w.f_tk, w.f_tv, nullptr, w.k_a, w.v_a, w.k_b, w.v_b, n, 0, 64, w.sort_scratch, s,
                             &fp.sk, &fp.sv, &h->tree.ctrl->error, n_touch, h->sort_threads_touch);
  if (se != cudaSuccess) return -2;
  fp.n_tiles = (uint32_t)pass_tiles(n);
  prof_mark(h, h->overlap != 0 ? kEvSortEnd : 1, s);
  if (passes) {
    if (vals_ready && cudaStreamWaitEvent(s, vals_ready, 0) != cudaSuccess) return -2;
    merge_pass1<<<fp.n_tiles, kThreads, 0, s>>>(fp.sk, fp.sv, vals, n, n_touch, w.tiles);
    count_launch();
    merge_pass2<<<1, 1024, 0, s>>>(w.tiles, fp.n_tiles, n_touch, c);
    count_launch();
    merge_pass3<<<fp.n_tiles, kThreads, 0, s>>>(fp.sk, fp.sv, vals, n, n_touch, w.tiles, w.ukeys, w.uvals,
                                                w.ins_list, w.get_list, w.del_list, w.pend, out_vals, out_st);
    count_launch();
    fp.passes_done = true;
  }
  return cudaGetLastError() == cudaSuccess ? 0 : -2;
}

static int hashed_tree(Handle* h, const uint64_t* keys, const uint64_t* vals, uint64_t* out_vals, uint8_t* out_st,
                       size_t n, int engine, cudaStream_t s, const FrontPart& fp) {
  Work& w = h->w;
  BatchCounts* c = w.counts;
  const uint32_t* n_touch = &c->n_touch;
  const bool ov = h->overlap != 0;
  const bool early = merge_usable(h, engine);
  const bool defer = early && h->async_write != 0;
  const bool learned = batch_learned(h, h->batch_descent >= 0 ? h->batch_descent : h->descent, s);
  // the locates (side stream) run beside the lookups (`s`); so do the merge
  // passes when the values are still being copied in (vals_wait): the
  // lookups do not need them
  cudaStream_t s2 = ov ? h->hi_stream : s;
  auto fork = [&]() {
    // a stale prefix table is rebuilt before the fork, so that the locates
    // (side stream) and the lookups (`s`) both come after the rebuild
    if (early && h->use_pfx && (tree_join(h, s) != cudaSuccess || ensure_pfx(h, s) != cudaSuccess)) return false;
    return cudaEventRecord(h->fork_ev, s) == cudaSuccess && cudaStreamWaitEvent(s2, h->fork_ev, 0) == cudaSuccess;
  };
  if (!fp.passes_done) {
    cudaStream_t sp = ov ? s2 : s;
    if ((ov && !fork()) || wait_vals(h, sp) != 0) return -2;
    merge_pass1<<<fp.n_tiles, kThreads, 0, sp>>>(fp.sk, fp.sv, vals, n, n_touch, w.tiles);
    count_launch();
    merge_pass2<<<1, 1024, 0, sp>>>(w.tiles, fp.n_tiles, n_touch, c);
    count_launch();
    merge_pass3<<<fp.n_tiles, kThreads, 0, sp>>>(fp.sk, fp.sv, vals, n, n_touch, w.tiles, w.ukeys, w.uvals,
                                                 w.ins_list, w.get_list, w.del_list, w.pend, out_vals, out_st);
    count_launch();
    if (cudaGetLastError() != cudaSuccess) return -2;
  } else if (ov && !fork()) {
    return -2;
  }
  if (early) {
    if (tree_join(h, s2) != cudaSuccess || delete_locate(h, n, s2) != 0 || merge_locate_phase(h, s2) != 0 ||
        merge_group_phase(h, n, s2) != 0)
      return -2;
  }
  prof_mark(h, 2, s2);
  if (ov && cudaEventRecord(h->join_ev, s2) != cudaSuccess) return -2;
  // plain lookups of the pre-batch tree; every touched run begins with a
  // write, so the merged batch has no GET runs (n_get is zero)
  if (tree_join(h, s) != cudaSuccess) return -2;
  if (ov) prof_mark(h, 1, s);
  cudaError_t e;
  h->lookup_reserve = ov ? h->overlap_reserve : 0;
  // the lookups read their keys compacted (w.f_lk[q], written by the front
  // end) instead of through the list (keys[f_list[q]]): one dependent load less
  if (learned)
    e = launch_learned_lookup(h, keys, w.f_list, &c->n_lookup, n, out_vals, out_st, s, w.f_lk, true);
  else
    e = launch_search(h, keys, w.f_list, &c->n_lookup, n, out_vals, out_st, s, w.f_lk);
  h->lookup_reserve = 0;
  if (e != cudaSuccess) return -2;
  if (learned) learned_sample(h, s);
  if (ov) {
    prof_mark(h, kEvLookupEnd, s);
    if (cudaStreamWaitEvent(s, h->join_ev, 0) != cudaSuccess) return -2;
  }
  prof_mark(h, 3, s);
  const unsigned wb_blocks = (unsigned)min((size_t)h->sm_count * 8, (n + 255) / 256);
  if (!early) {
    if (insert_phase(h, n, engine, s) != 0) return -2;
    prof_mark(h, 4, s);
    writeback_kernel<<<wb_blocks, 256, 0, s>>>(fp.sv, w.pend, n, n_touch, w.uans, w.uans_st, out_vals, out_st);
    count_launch();
    prof_mark(h, 5, s);
    return answers_ready(h, s) != 0 || cudaGetLastError() != cudaSuccess ? -2 : 0;
  }
  if (merge_update_phase(h, n, s) != 0 || delete_apply(h, n, s) != 0 || merge_reserve_phase(h, n, s) != 0)
    return -2;
  prof_mark(h, kEvWbStart, s);
  writeback_kernel<<<wb_blocks, 256, 0, s>>>(fp.sv, w.pend, n, n_touch, w.uans, w.uans_st, out_vals, out_st);
  count_launch();
  prof_mark(h, 4, s);
  if (answers_ready(h, s) != 0 || cudaGetLastError() != cudaSuccess) return -2;
  cudaStream_t t = s;
  if (defer) {
    t = h->tree_stream;
    if (cudaEventRecord(h->ans_ev, s) != cudaSuccess || cudaStreamWaitEvent(t, h->ans_ev, 0) != cudaSuccess)
      return -2;
  }
  if (merge_write_phase(h, t) != 0) return -2;
  prof_mark(h, 5, t);
  if (defer) {
    if (cudaEventRecord(h->tree_ev, t) != cudaSuccess) return -2;
    h->tree_pending = true;
  }
  return cudaGetLastError() == cudaSuccess ? 0 : -2;
}

static int batch_hashed(Handle* h, const uint64_t* keys, const uint64_t* vals, const uint8_t* ops,
                        uint64_t* out_vals, uint8_t* out_st, size_t n, int engine, cudaStream_t s) {
  const bool ov = h->overlap != 0;
  const bool pass_side = ov && (h->vals_wait != nullptr || h->vals_remote);
  prof_mark(h, 0, s);
  prof_set_layout(h, (ov ? kLayoutOverlap : 0) | (merge_usable(h, engine) ? kLayoutEarly : 0));
  FrontPart fp;
  if (hashed_front(h, keys, vals, ops, out_vals, out_st, n, s, !pass_side, fp) != 0) return -2;
  return hashed_tree(h, keys, vals, out_vals, out_st, n, engine, s, fp);
}

static int front_stream_init(Handle* h) {
  if (h->front_stream) return 0;
  bool ok = cudaStreamCreateWithFlags(&h->front_stream, cudaStreamNonBlocking) == cudaSuccess &&
            cudaEventCreateWithFlags(&h->pipe_ev, cudaEventDisableTiming) == cudaSuccess &&
            cudaEventCreateWithFlags(&h->chain_gate, cudaEventDisableTiming) == cudaSuccess;
  for (int p = 0; ok && p < 2; p++)
    ok = cudaEventCreateWithFlags(&h->front_done[p], cudaEventDisableTiming) == cudaSuccess &&
         cudaEventCreateWithFlags(&h->tree_done[p], cudaEventDisableTiming) == cudaSuccess;
  return ok ? 0 : -2;
}

// Several hash-front-end batches, their inputs all ready on `s`, in order:
// batch j + 1's front part (classification, sort, merge passes: no tree) on
// front_stream beside batch j's tree part on `s`, the two with alternate
// buffer sets.  A front part waits for the tree part that last used its
// set; a tree part waits for its own front part.  The answers and the tree
// are the batches' one by one.  Phases are not recorded (they would span
// two streams).
int batches_pipelined(Handle* h, size_t count, const uint64_t* const* keys, const uint64_t* const* vals,
                      const uint8_t* const* ops, uint64_t* const* out_vals, uint8_t* const* out_st, const size_t* n,
                      int engine, cudaStream_t s) {
  Work& w = h->w;
  if (count == 0) return 0;
  for (size_t j = 0; j < count; j++)
    if (n[j] == 0 || n[j] > w.cap || n[j] > kIdxMask) return -6;
  if (work_alt_alloc(&w) != 0) return -3;
  if (front_stream_init(h) != 0) return -2;
  cudaStream_t F = h->front_stream;
  const bool prof = h->prof;
  h->prof = false;
  auto use = [&](int p) {
    if ((int)w.alt_in != p) work_swap_set(&w);
  };
  int rc = 0;
  FrontPart fp[2];
  // the inputs are ready in `s`'s order at this point
  if (cudaEventRecord(h->pipe_ev, s) != cudaSuccess || cudaStreamWaitEvent(F, h->pipe_ev, 0) != cudaSuccess) rc = -2;
  for (size_t j = 0; j <= count && rc == 0; j++) {
    if (j < count) {
      const int p = (int)(j & 1);
      use(p);
      fp[p] = FrontPart{};
      if ((j >= 2 && cudaStreamWaitEvent(F, h->tree_done[p], 0) != cudaSuccess) ||
          hashed_front(h, keys[j], vals[j], ops[j], out_vals[j], out_st[j], n[j], F, true, fp[p]) != 0 ||
          cudaEventRecord(h->front_done[p], F) != cudaSuccess)
        rc = -2;
    }
    if (rc == 0 && j >= 1) {
      const size_t i = j - 1;
      const int q = (int)(i & 1);
      use(q);
      if (cudaStreamWaitEvent(s, h->front_done[q], 0) != cudaSuccess ||
          hashed_tree(h, keys[i], vals[i], out_vals[i], out_st[i], n[i], engine, s, fp[q]) != 0 ||
          cudaEventRecord(h->tree_done[q], s) != cudaSuccess)
        rc = -2;
    }
  }
  use(0);
  h->prof = prof;
  // whatever the front stream did is ordered before `s`'s later work
  if (cudaEventRecord(h->pipe_ev, F) != cudaSuccess || cudaStreamWaitEvent(s, h->pipe_ev, 0) != cudaSuccess) rc = -2;
  return rc;
}

// The front part of batch j (set j & 1) waits for chain_gate, recorded on
// `s` just before batch j - 1's tree part was queued: by then `s` holds
// batch j - 2's tree part, the last user of the set, and nothing else of
// the handle came after it (chain_open; every other entry point closes the
// chain).  The other front parts are before it on front_stream.  With
// `vals_late` (a value slot per request, copied after the keys) the merge
// passes go to the tree part, beside the lookups as in batch_hashed, so
// that the lookups need not wait for the values.
int batch_chained(Handle* h, const uint64_t* keys, const uint64_t* vals, const uint8_t* ops, uint64_t* out_vals,
                  uint8_t* out_st, size_t n, int engine, cudaStream_t s, cudaEvent_t in_ready,
                  cudaEvent_t vals_ready, bool vals_late) {
  Work& w = h->w;
  if (n == 0) return 0;
  if (n > w.cap || n > kIdxMask) return -6;
  const bool open = h->chain_open;
  h->chain_open = false;
  if (work_alt_alloc(&w) != 0) return -3;
  if (front_stream_init(h) != 0) return -2;
  cudaStream_t F = h->front_stream;
  const int p = h->chain_set ^= 1;
  const bool prof = h->prof;
  h->prof = false;
  auto use = [&](int q) {
    if ((int)w.alt_in != q) work_swap_set(&w);
  };
  int rc = 0;
  FrontPart fp;
  const bool pass_tree = vals_late && h->overlap != 0;
  use(p);
  if ((!open && cudaEventRecord(h->chain_gate, s) != cudaSuccess) ||
      cudaStreamWaitEvent(F, h->chain_gate, 0) != cudaSuccess || cudaStreamWaitEvent(F, in_ready, 0) != cudaSuccess ||
      hashed_front(h, keys, vals, ops, out_vals, out_st, n, F, !pass_tree, fp, vals_ready) != 0 ||
      cudaEventRecord(h->front_done[p], F) != cudaSuccess || cudaEventRecord(h->chain_gate, s) != cudaSuccess ||
      cudaStreamWaitEvent(s, h->front_done[p], 0) != cudaSuccess)
    rc = -2;
  if (rc == 0) {
    h->vals_wait = pass_tree ? vals_ready : nullptr;
    if (hashed_tree(h, keys, vals, out_vals, out_st, n, engine, s, fp) != 0) rc = -2;
    h->vals_wait = nullptr;
  }
  use(0);
  h->prof = prof;
  h->chain_open = rc == 0;
  return rc;
}

int batch_sorted(Handle* h, const uint64_t* keys, const uint64_t* vals, const uint8_t* ops, uint64_t* out_vals,
                 uint8_t* out_st, size_t n, int engine, cudaStream_t s) {
  if (n == 0) return 0;
  Work& w = h->w;
  if (n > w.cap || n > kIdxMask) return -6;
  if (h->front_end == 1) return batch_hashed(h, keys, vals, ops, out_vals, out_st, n, engine, s);
  if (tree_join(h, s) != cudaSuccess) return -2;
  const bool learned = batch_learned(h, h->batch_descent >= 0 ? h->batch_descent : h->descent, s);
  uint64_t* sk = nullptr;
  uint32_t* sv = nullptr;
  prof_mark(h, 0, s);
  if (radix_sort_pairs(keys, nullptr, ops, w.k_a, w.v_a, w.k_b, w.v_b, n, 0, 64, w.sort_scratch, s, &sk, &sv,
                       &h->tree.ctrl->error, nullptr, h->sort_threads) != cudaSuccess)
    return -2;
  const uint32_t n_tiles = (uint32_t)pass_tiles(n);
  prof_mark(h, 1, s);
  if (wait_vals(h, s) != 0) return -2;
  merge_pass1<<<n_tiles, kThreads, 0, s>>>(sk, sv, vals, n, nullptr, w.tiles);
  count_launch();
  merge_pass2<<<1, 1024, 0, s>>>(w.tiles, n_tiles, nullptr, w.counts);
  count_launch();
  merge_pass3<<<n_tiles, kThreads, 0, s>>>(sk, sv, vals, n, nullptr, w.tiles, w.ukeys, w.uvals, w.ins_list,
                                           w.get_list, w.del_list, w.pend, out_vals, out_st);
  count_launch();
  if (cudaGetLastError() != cudaSuccess) return -2;
  // search phase on the pre-batch tree, then the insert phase
  prof_mark(h, 2, s);
  cudaError_t e;
  if (learned)
    e = launch_learned_search(h, w.ukeys, w.get_list, &w.counts->n_get, n, w.uans, w.uans_st, s,
                              h->sorted_search != 0);
  else if (h->sorted_search)
    e = launch_search_sorted(h, w.ukeys, w.get_list, &w.counts->n_get, n, w.uans, w.uans_st, s);
  else
    e = launch_search(h, w.ukeys, w.get_list, &w.counts->n_get, n, w.uans, w.uans_st, s);
  if (e != cudaSuccess) return -2;
  if (learned) learned_sample(h, s);
  prof_mark(h, 3, s);
  if (insert_phase(h, n, engine, s) != 0) return -2;
  prof_mark(h, 4, s);
  const unsigned wb_blocks = (unsigned)min((size_t)h->sm_count * 8, (n + 255) / 256);
  writeback_kernel<<<wb_blocks, 256, 0, s>>>(sv, w.pend, n, nullptr, w.uans, w.uans_st, out_vals, out_st);
  count_launch();
  prof_mark(h, 5, s);
  if (answers_ready(h, s) != 0) return -2;
  if (cudaGetLastError() != cudaSuccess) return -2;
  return 0;
}

}  // namespace bt
