// Tree construction and the lock-free batched point search.
//
// Search: a group of G lanes serves one request (G = 4, 8, 16 or 32; the
// reference uses a whole warp, one key per lane, src/gpu-stm-tree-v39/
// bpt-gpustm-kernel-tree.cuh:61-118).  Each lane loads 32/G consecutive keys
// of the node with 16-byte vector loads, counts keys <= target, and the group
// sums the counts with xor-shuffles: that sum is the child slot (child i covers
// [key[i-1], key[i]), src/tree.h:7-19).  With G = 8 a warp carries four
// independent descents, four times the memory-level parallelism of the
// reference's warp-per-request layout.  This kernel runs only when no writer
// is active (the batch executor orders it before/after the insert phase), so
// it needs no version checks and may use the read-only cache path.
#include <cstdio>
#include <cuda_runtime.h>

#include "bt_block.cuh"
#include "bt_common.cuh"
#include "bt_internal.h"
#include "bt_search.cuh"

namespace bt {

namespace {

__global__ void reset_kernel(Ctrl* c, uint32_t epoch) {
  c->root = kNil;
  c->epoch = epoch;
  c->root_lock = 0;
  c->n_nodes = 0;
  c->error = 0;
  c->root_level = 0;
  c->n_keys = 0;
  c->commits = c->aborts = c->leaf_splits = c->inner_splits = c->new_roots = 0;
  c->retry_exhausted = c->learned_hits = c->learned_fallbacks = c->learned_probe_sum = 0;
}

// ---------------------------------------------------------------- build ----
__global__ void tail_flags_kernel(const uint64_t* __restrict__ sk, size_t n, uint32_t* __restrict__ flags) {
  size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) flags[i] = (i + 1 == n || sk[i + 1] != sk[i]) ? 1u : 0u;
}

__global__ void dedupe_kernel(const uint64_t* __restrict__ sk, const uint32_t* __restrict__ sidx,
                              const uint64_t* __restrict__ vals, const uint32_t* __restrict__ flags,
                              const uint32_t* __restrict__ pos, size_t n, uint64_t* __restrict__ uk,
                              uint64_t* __restrict__ uv) {
  size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n && flags[i]) {
    uint32_t p = pos[i];
    uk[p] = sk[i];
    uv[p] = vals[sidx[i]];
  }
}

// one warp per leaf; leaves get base or base+1 keys (the first `rem` get one more)
__global__ void build_leaves_kernel(DevTree t, const uint64_t* __restrict__ uk, const uint64_t* __restrict__ uv,
                                    size_t m, uint32_t nl, uint32_t epoch) {
  const uint32_t lane = threadIdx.x & 31;
  const size_t j = ((size_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  if (j >= nl) return;
  const size_t base = m / nl, rem = m % nl;
  const size_t k = base + (j < rem ? 1 : 0);
  const size_t start = j * base + (j < rem ? j : rem);
  uint64_t* kr = t.keys + j * 32;
  uint64_t* vr = t.vals + j * 32;
  if (lane < 31) {
    kr[lane] = lane < k ? uk[start + lane] : kKeyMax;
    vr[lane] = lane < k ? uv[start + lane] : 0;
  } else {
    kr[31] = make_hdr((uint32_t)k, 0, 0, epoch);
    vr[31] = (j + 1 < nl) ? uk[start + k] : kKeyMax;
  }
  if (lane == 0) t.low[j] = j == 0 ? 0 : uk[start];
}

// one warp per inner node of a level: node p groups children [c, c + k)
__global__ void build_inner_kernel(DevTree t, uint32_t first_child, uint32_t n_children, uint32_t first_node,
                                   uint32_t n_nodes_level, uint32_t level, uint32_t epoch) {
  const uint32_t lane = threadIdx.x & 31;
  const uint32_t p = (uint32_t)(((size_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5);
  if (p >= n_nodes_level) return;
  const uint32_t base = n_children / n_nodes_level, rem = n_children % n_nodes_level;
  const uint32_t k = base + (p < rem ? 1 : 0);
  const uint32_t c = first_child + p * base + (p < rem ? p : rem);
  const uint32_t id = first_node + p;
  uint64_t* kr = t.keys + (size_t)id * 32;
  uint64_t* vr = t.vals + (size_t)id * 32;
  // key slot i (i < k-1) = low fence of child i+1
  if (lane < 31) kr[lane] = (lane + 1 < k) ? t.low[c + lane + 1] : kKeyMax;
  else kr[31] = make_hdr(k - 1, level, 0, epoch);
  vr[lane] = lane < k ? (uint64_t)(c + lane) : 0;
  if (lane == 0) t.low[id] = t.low[c];
}

__global__ void set_root_kernel(Ctrl* c, uint32_t root, uint32_t root_level, uint32_t n_nodes, uint64_t n_keys) {
  c->root = root;
  c->root_level = root_level;
  c->n_nodes = n_nodes;
  c->n_keys = n_keys;
}

// --------------------------------------------------------------- search ----
template <int G, bool kLeafVals>
__global__ void __launch_bounds__(256) search_kernel(DevTree t, const uint64_t* __restrict__ qkeys,
                                                     const uint32_t* __restrict__ list,
                                                     const uint32_t* __restrict__ n_dev, size_t n_host,
                                                     uint64_t* __restrict__ out_vals, uint8_t* __restrict__ out_st) {
  const uint32_t lane = threadIdx.x & 31;
  const uint32_t g = lane % G;
  const uint32_t gmask = group_mask<G>(lane);
  const size_t n = n_dev ? (size_t)*n_dev : n_host;
  const uint32_t root = t.ctrl->root;
  const uint32_t root_level = t.ctrl->root_level;
  const size_t stride = ((size_t)gridDim.x * blockDim.x) / G;
  for (size_t q = ((size_t)blockIdx.x * blockDim.x + threadIdx.x) / G; q < n; q += stride) {
    const uint32_t r = list ? __ldg(list + q) : (uint32_t)q;
    const uint64_t key = __ldg(qkeys + r);
    uint8_t st = kAbsent;
    uint64_t ans = 0;
    if (key == kKeyMax) st = kRejected;
    else if (root != kNil) st = group_descend<G, kLeafVals>(t, root, root_level, key, g, gmask, ans);
    if (g == 0) {
      out_vals[r] = ans;
      out_st[r] = st;
    }
  }
}

// Two requests per group in lock step (group_descend2): requests q and
// q + stride of the grid-stride loop share a group.
template <int G, bool kLeafVals, bool kChild>
__global__ void __launch_bounds__(256) search2_kernel(DevTree t, const uint64_t* __restrict__ qkeys,
                                                      const uint32_t* __restrict__ list,
                                                      const uint32_t* __restrict__ n_dev, size_t n_host,
                                                      uint64_t* __restrict__ out_vals, uint8_t* __restrict__ out_st,
                                                      int use_pfx, const uint64_t* __restrict__ ckeys) {
  const uint32_t lane = threadIdx.x & 31;
  const uint32_t g = lane % G;
  const uint32_t gmask = group_mask<G>(lane);
  const size_t n = n_dev ? (size_t)*n_dev : n_host;
  const uint32_t root = t.ctrl->root;
  const uint32_t root_level = t.ctrl->root_level;
  const size_t groups = ((size_t)gridDim.x * blockDim.x) / G;
  for (size_t q = ((size_t)blockIdx.x * blockDim.x + threadIdx.x) / G; q < n; q += 2 * groups) {
    const size_t q2 = q + groups;
    const bool two = q2 < n;
    const uint32_t ra = list ? __ldg(list + q) : (uint32_t)q;
    const uint32_t rb = two ? (list ? __ldg(list + q2) : (uint32_t)q2) : ra;
    const uint64_t key_a = ckeys ? __ldg(ckeys + q) : __ldg(qkeys + ra);
    const uint64_t key_b = ckeys ? __ldg(ckeys + (two ? q2 : q)) : __ldg(qkeys + rb);
    uint8_t sa = kAbsent, sb = kAbsent;
    uint64_t aa = 0, ab = 0;
    if (root != kNil) {
      // a reserved key descends as key 0 (keeping the pair in lock step) and is reported as rejected
      group_descend2<G, kLeafVals, kChild>(t, root, root_level, key_a == kKeyMax ? 0 : key_a,
                                   key_b == kKeyMax ? 0 : key_b, g, gmask, aa, sa, ab, sb, use_pfx != 0);
    }
    if (key_a == kKeyMax) {
      sa = kRejected;
      aa = 0;
    }
    if (key_b == kKeyMax) {
      sb = kRejected;
      ab = 0;
    }
    if (g == 0) {
      out_vals[ra] = aa;
      out_st[ra] = sa;
      if (two) {
        out_vals[rb] = ab;
        out_st[rb] = sb;
      }
    }
  }
}

// Search over keys given in ascending order (the batch executor's unique
// GET list).  Each group walks a contiguous chunk of the list and keeps the
// path of its previous lookup: lane l of the group caches level l's node id
// and the exclusive upper bound of its key range.  A key restarts its descent
// at the lowest cached level whose range still holds it (keys ascend, so only
// the upper bound needs checking); a key in the previous leaf reuses the leaf
// row already in registers.  Requires root_level < G.
template <int G, bool kLeafVals>
__global__ void __launch_bounds__(256) search_sorted_kernel(DevTree t, const uint64_t* __restrict__ qkeys,
                                                            const uint32_t* __restrict__ list,
                                                            const uint32_t* __restrict__ n_dev, size_t n_host,
                                                            uint64_t* __restrict__ out_vals,
                                                            uint8_t* __restrict__ out_st) {
  constexpr int S = 32 / G;
  const uint32_t lane = threadIdx.x & 31;
  const uint32_t g = lane % G;
  const uint32_t gmask = group_mask<G>(lane);
  const size_t n = n_dev ? (size_t)*n_dev : n_host;
  const uint32_t root = t.ctrl->root;
  const uint32_t root_level = t.ctrl->root_level;
  const size_t n_groups = ((size_t)gridDim.x * blockDim.x) / G;
  const size_t gid = ((size_t)blockIdx.x * blockDim.x + threadIdx.x) / G;
  const size_t chunk = (n + n_groups - 1) / n_groups;
  const size_t q0 = gid * chunk;
  const size_t q1 = min(n, q0 + chunk);
  // path cache (lane g holds level g)
  uint32_t c_node = root;
  uint64_t c_hi = 0;       // exclusive upper bound; 0 with c_valid = false
  bool c_valid = (g == root_level);
  if (c_valid) c_hi = kKeyMax;  // the root covers everything
  uint64_t k[S];
  uint64_t v[S];
  uint32_t leaf = kNil;
  for (size_t q = q0; q < q1; q++) {
    const uint32_t r = list ? __ldg(list + q) : (uint32_t)q;
    const uint64_t key = __ldg(qkeys + r);
    uint8_t st = kAbsent;
    uint64_t ans = 0;
    if (key == kKeyMax) {
      st = kRejected;
    } else if (root != kNil) {
      if (root_level >= (uint32_t)G) {  // tree taller than the cache: plain descent
        st = group_descend<G, false>(t, root, root_level, key, g, gmask, ans);
        if (g == 0) {
          out_vals[r] = ans;
          out_st[r] = st;
        }
        continue;
      }
      // lowest cached level whose range holds the key
      const uint32_t hit = (__ballot_sync(gmask, c_valid && key < c_hi) >> (lane - g)) & ((1u << G) - 1u);
      uint32_t level = hit ? (uint32_t)(__ffs(hit) - 1) : root_level;
      uint32_t node = __shfl_sync(gmask, c_node, level, G);
      uint64_t hi = __shfl_sync(gmask, c_hi, level, G);
      if (!hit) {
        node = root;
        hi = kKeyMax;
      }
      // levels below `level` are now stale
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
          load_slots<S>(t.keys + row, k);
          if (level > 0 || kLeafVals) load_slots<S>(t.vals + row, v);
          if (g == G - 1) k[S - 1] = kKeyMax;
          uint32_t c = 0;
#pragma unroll
          for (int i = 0; i < S; i++) c += (k[i] <= key) ? 1u : 0u;
          cnt = group_sum<G>(c, gmask);
          if (level == 0) break;
          // child range upper bound: key[cnt] (padding is UINT64_MAX) capped by ours
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
      st = group_leaf_lookup<G, kLeafVals>(t, leaf, key, g, gmask, k, v, cnt, ans);
    }
    if (g == 0) {
      out_vals[r] = ans;
      out_st[r] = st;
    }
  }
}

// ---------------------------------------------------------- enumeration ----
__global__ void child_count_kernel(DevTree t, const uint32_t* __restrict__ nodes, size_t n, uint32_t* cnt,
                                   int leaf_sizes) {
  size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) {
    uint64_t h = t.keys[(size_t)nodes[i] * 32 + 31];
    cnt[i] = leaf_sizes ? hdr_size(h) : hdr_size(h) + 1;
  }
}

__global__ void child_write_kernel(DevTree t, const uint32_t* __restrict__ nodes, size_t n,
                                   const uint32_t* __restrict__ off, uint32_t* __restrict__ out) {
  const uint32_t lane = threadIdx.x & 31;
  const size_t i = ((size_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  if (i >= n) return;
  const uint32_t node = nodes[i];
  const uint32_t sz = hdr_size(t.keys[(size_t)node * 32 + 31]);
  if (lane <= sz) out[off[i] + lane] = (uint32_t)t.vals[(size_t)node * 32 + lane];
}

__global__ void leaf_dump_kernel(DevTree t, const uint32_t* __restrict__ leaves, size_t n,
                                 const uint32_t* __restrict__ off, uint64_t* __restrict__ ok,
                                 uint64_t* __restrict__ ov) {
  const uint32_t lane = threadIdx.x & 31;
  const size_t i = ((size_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  if (i >= n) return;
  const uint32_t node = leaves[i];
  const uint32_t sz = hdr_size(t.keys[(size_t)node * 32 + 31]);
  if (lane < sz) {
    size_t o = (size_t)off[i] + lane;
    if (ok) ok[o] = t.keys[(size_t)node * 32 + lane];
    if (ov) ov[o] = t.vals[(size_t)node * 32 + lane];
  }
}

inline unsigned blocks_for(size_t n, int per) { return (unsigned)((n + per - 1) / per); }

// ------------------------------------------------------------ top cache ----
// The upper levels of the tree, copied into shared memory by every block of
// the unsorted search: a request descends them there and continues from
// global memory below.  Built per search launch by one block (breadth-first
// from the root, whole levels while they fit kTopNodes, never the leaf
// level), so it always matches the tree that the search reads.
struct TopNode {
  uint64_t keys[31];   // separators; unused slots hold kKeyMax
  uint32_t child[32];  // next cached level: index into the cache; last cached level: node id
  uint32_t pad[2];
};
static_assert(sizeof(TopNode) == 384, "TopNode layout");

__global__ void __launch_bounds__(256) top_build_kernel(DevTree t, TopNode* __restrict__ top,
                                                       TopInfo* __restrict__ info) {
  __shared__ uint32_t ids[kTopNodes];
  __shared__ uint32_t kids[kTopNodes];  // per node: index of its first child in ids
  __shared__ uint32_t ws[32];
  __shared__ uint32_t s_lvl_start, s_lvl_end, s_levels, s_stop;
  const uint32_t root = t.ctrl->root;
  const uint32_t rl = t.ctrl->root_level;
  if (root == kNil || rl < 1) {
    if (threadIdx.x == 0) info->n_levels = 0;
    return;
  }
  if (threadIdx.x == 0) {
    ids[0] = root;
    s_lvl_start = 0;
    s_lvl_end = 1;
    s_levels = 1;
    s_stop = 0;
  }
  __syncthreads();
  // add whole levels while the next one is still an inner level and fits
  for (uint32_t level = rl; level >= 2; level--) {
    const uint32_t a = s_lvl_start, b = s_lvl_end;
    uint32_t total = 0;
    for (uint32_t base = a; base < b; base += blockDim.x) {
      const uint32_t i = base + threadIdx.x;
      const uint32_t c = i < b ? hdr_size(t.keys[(size_t)ids[i] * 32 + 31]) + 1 : 0u;
      uint32_t tot;
      const uint32_t ex = blk_exclusive_sum(c, ws, &tot);
      if (i < b) kids[i] = b + total + ex;
      total += tot;
    }
    __syncthreads();
    if (b + total > (uint32_t)kTopNodes) break;  // uniform: every thread has the same total
    for (uint32_t i = a + threadIdx.x / 32; i < b; i += blockDim.x / 32) {
      const uint32_t lane = threadIdx.x & 31;
      const uint32_t c = hdr_size(t.keys[(size_t)ids[i] * 32 + 31]) + 1;
      if (lane < c) ids[kids[i] + lane] = (uint32_t)t.vals[(size_t)ids[i] * 32 + lane];
    }
    __syncthreads();
    if (threadIdx.x == 0) {
      s_lvl_start = b;
      s_lvl_end = b + total;
      s_levels++;
    }
    __syncthreads();
  }
  const uint32_t n_nodes = s_lvl_end, last = s_lvl_start, n_levels = s_levels;
  // kids[] holds the child offsets of every level except the last cached one
  for (uint32_t i = threadIdx.x / 32; i < n_nodes; i += blockDim.x / 32) {
    const uint32_t lane = threadIdx.x & 31;
    const size_t row = (size_t)ids[i] * 32;
    const uint32_t c = hdr_size(t.keys[row + 31]) + 1;
    if (lane < 31) top[i].keys[lane] = t.keys[row + lane];  // slots past the size hold kKeyMax
    uint32_t ch = kNil;
    if (lane < c) ch = i >= last ? (uint32_t)t.vals[row + lane] : kids[i] + lane;
    top[i].child[lane] = ch;
  }
  if (threadIdx.x == 0) {
    info->n_nodes = n_nodes;
    info->n_levels = n_levels;
    info->below_level = rl - n_levels;
  }
}

template <int G, bool kLeafVals>
__global__ void __launch_bounds__(512) search_top_kernel(DevTree t, const TopNode* __restrict__ top,
                                                        const TopInfo* __restrict__ info,
                                                        const uint64_t* __restrict__ qkeys,
                                                        const uint32_t* __restrict__ list,
                                                        const uint32_t* __restrict__ n_dev, size_t n_host,
                                                        uint64_t* __restrict__ out_vals,
                                                        uint8_t* __restrict__ out_st) {
  constexpr int S = 32 / G;
  extern __shared__ __align__(16) unsigned char top_raw[];
  const TopNode* ts = reinterpret_cast<const TopNode*>(top_raw);
  const uint32_t n_levels = info->n_levels;
  const uint32_t n_nodes = n_levels ? info->n_nodes : 0;
  {
    const uint4* src = reinterpret_cast<const uint4*>(top);
    uint4* dst = reinterpret_cast<uint4*>(top_raw);
    const uint32_t words = n_nodes * (uint32_t)(sizeof(TopNode) / 16);
    for (uint32_t i = threadIdx.x; i < words; i += blockDim.x) dst[i] = src[i];
  }
  __syncthreads();
  const uint32_t lane = threadIdx.x & 31;
  const uint32_t g = lane % G;
  const uint32_t gmask = group_mask<G>(lane);
  const size_t n = n_dev ? (size_t)*n_dev : n_host;
  const uint32_t root = t.ctrl->root;
  const uint32_t root_level = t.ctrl->root_level;
  const uint32_t below = info->below_level;
  const size_t stride = ((size_t)gridDim.x * blockDim.x) / G;
  for (size_t q = ((size_t)blockIdx.x * blockDim.x + threadIdx.x) / G; q < n; q += stride) {
    const uint32_t r = list ? __ldg(list + q) : (uint32_t)q;
    const uint64_t key = __ldg(qkeys + r);
    uint8_t st = kAbsent;
    uint64_t ans = 0;
    if (key == kKeyMax) {
      st = kRejected;
    } else if (root != kNil) {
      uint32_t node = root, level = root_level;
      if (n_levels) {
        uint32_t idx = 0;
        for (uint32_t l = 0; l < n_levels; l++) {
          const TopNode& tn = ts[idx];
          uint32_t c = 0;
#pragma unroll
          for (int i = 0; i < S; i++) {
            const int slot = g * S + i;
            c += (slot < 31 && tn.keys[slot] <= key) ? 1u : 0u;
          }
          c = group_sum<G>(c, gmask);
          idx = tn.child[c];
        }
        node = idx;
        level = below;
      }
      st = group_descend<G, kLeafVals>(t, node, level, key, g, gmask, ans);
    }
    if (g == 0) {
      out_vals[r] = ans;
      out_st[r] = st;
    }
  }
}

// Range scan, one warp per query: descend to the leaf that holds `lo`, take
// the leaf's keys in [lo, hi] (lane i holds slot i; a ballot compacts them in
// key order), and continue at the leaf that starts at this leaf's right fence
// (found by a new descent: leaves carry no sibling pointer) until a leaf's
// fence passes `hi`.  Read-only; runs only when no writer is active.
__global__ void __launch_bounds__(256) range_kernel(DevTree t, const uint64_t* __restrict__ lo_keys,
                                                   const uint64_t* __restrict__ hi_keys, size_t n, uint32_t max_per,
                                                   uint64_t* __restrict__ out_keys, uint64_t* __restrict__ out_vals,
                                                   uint32_t* __restrict__ out_counts) {
  const uint32_t lane = threadIdx.x & 31;
  const uint32_t root = t.ctrl->root;
  const uint32_t root_level = t.ctrl->root_level;
  const uint64_t cap_nodes = t.cap;
  const size_t warps = ((size_t)gridDim.x * blockDim.x) >> 5;
  for (size_t q = ((size_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5; q < n; q += warps) {
    const uint64_t lo = __ldg(lo_keys + q), hi = __ldg(hi_keys + q);
    uint32_t count = 0;
    uint64_t from = lo;
    bool more = root != kNil && lo <= hi && lo != kKeyMax;  // UINT64_MAX is never a stored key
    for (uint64_t visited = 0; more && visited <= cap_nodes; visited++) {
      // descend to the leaf holding `from`
      uint32_t node = root;
      for (uint32_t level = root_level; level > 0; level--) {
        const uint64_t k = __ldg(t.keys + (size_t)node * 32 + lane);
        const uint32_t c = __popc(__ballot_sync(0xffffffffu, lane < 31 && k <= from));
        node = (uint32_t)__ldg(t.vals + (size_t)node * 32 + c);
      }
      const uint64_t k = __ldg(t.keys + (size_t)node * 32 + lane);
      const uint64_t v = __ldg(t.vals + (size_t)node * 32 + lane);
      const uint32_t size = hdr_size(__shfl_sync(0xffffffffu, k, 31));
      const uint64_t fence = __shfl_sync(0xffffffffu, v, 31);
      const bool in = lane < size && lane < 31 && k >= lo && k <= hi;
      const uint32_t m = __ballot_sync(0xffffffffu, in);
      if (in) {
        const uint32_t pos = count + __popc(m & ((1u << lane) - 1u));
        if (pos < max_per) {
          out_keys[q * max_per + pos] = k;
          out_vals[q * max_per + pos] = v;
        }
      }
      count += __popc(m);
      // the next leaf starts at the fence; stop when it lies past hi
      more = fence != kKeyMax && fence <= hi && fence > from;
      from = fence;
    }
    if (lane == 0) out_counts[q] = count;
  }
}


}  // namespace

int top_alloc(Handle* h) {
  if (h->top) return 0;
  if (cudaMalloc(&h->top, (size_t)kTopNodes * sizeof(TopNode) + 64) != cudaSuccess) return -3;
  h->top_info = reinterpret_cast<TopInfo*>(static_cast<char*>(h->top) + (size_t)kTopNodes * sizeof(TopNode));
  return 0;
}

// unsorted search with the top levels in shared memory
cudaError_t launch_search_top(Handle* h, const uint64_t* qkeys, const uint32_t* list, const uint32_t* n_dev,
                              size_t n, uint64_t* out_vals, uint8_t* out_st, cudaStream_t s) {
  if (n == 0) return cudaSuccess;
  if (top_alloc(h) != 0) return cudaErrorMemoryAllocation;
  TopNode* top = reinterpret_cast<TopNode*>(h->top);
  top_build_kernel<<<1, 256, 0, s>>>(h->tree, top, h->top_info);
  count_launch();
  const int threads = 512;
  const size_t smem = (size_t)kTopNodes * sizeof(TopNode);
  const int G = h->search_group;
  static int per_sm[64][5] = {};
  const int gi = G == 4 ? 0 : G == 16 ? 2 : G == 32 ? 3 : G == -8 ? 4 : 1;
  const void* kern;
  switch (gi) {
    case 0: kern = (const void*)search_top_kernel<4, false>; break;
    case 2: kern = (const void*)search_top_kernel<16, false>; break;
    case 3: kern = (const void*)search_top_kernel<32, false>; break;
    case 4: kern = (const void*)search_top_kernel<8, true>; break;
    default: kern = (const void*)search_top_kernel<8, false>; break;
  }
  const int dev = h->device;
  int per = 1;
  if (dev >= 0 && dev < 64 && per_sm[dev][gi]) {
    per = per_sm[dev][gi];
  } else {
    if (cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) != cudaSuccess)
      return cudaErrorInvalidValue;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, kern, threads, smem) != cudaSuccess || per < 1) per = 1;
    if (dev >= 0 && dev < 64) per_sm[dev][gi] = per;
  }
  const int lanes = G < 0 ? -G : G;
  size_t blocks = (n * (size_t)lanes + threads - 1) / threads;
  const size_t cap = (size_t)h->sm_count * per;
  if (blocks > cap) blocks = cap;
  if (blocks == 0) blocks = 1;
  DevTree tree = h->tree;
  const TopInfo* info = h->top_info;
  void* args[] = {&tree, &top, &info, (void*)&qkeys, (void*)&list, (void*)&n_dev, &n, &out_vals, &out_st};
  cudaError_t e = cudaLaunchKernel(kern, dim3((unsigned)blocks), dim3(threads), args, smem, s);
  count_launch();
  return e;
}

__global__ void clear_headers_kernel(DevTree t, uint32_t first, uint32_t last) {
  for (size_t i = (size_t)first + (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < last;
       i += (size_t)gridDim.x * blockDim.x)
    t.keys[i * 32 + 31] = 0;
}

cudaError_t clear_headers(Handle* h, uint32_t first, uint32_t last, cudaStream_t s) {
  if (first >= last) return cudaSuccess;
  const size_t n = last - first;
  const unsigned blocks = (unsigned)min((size_t)h->sm_count * 8, (n + 255) / 256);
  clear_headers_kernel<<<blocks, 256, 0, s>>>(h->tree, first, last);
  count_launch();
  return cudaGetLastError();
}

cudaError_t tree_reset(Handle* h, cudaStream_t s) {
  h->pfx_valid = false;  // the bulk loader writes inner rows without prefixes
  // The epoch has 15 bits (1 .. 0x7fff; 0 marks never-written rows).  When
  // it comes round to 1 again, rows written by the trees of the last cycle
  // may still carry that number: clear every row's header first, so that a
  // reader which reaches a row without a validated path (the optimistic STM
  // descent, the learned leaf guess) cannot take a row of an older tree for
  // one of the new tree.
  if (h->epoch == 0x7fffu) {
    const cudaError_t e = clear_headers(h, 0, h->tree.cap, s);
    if (e != cudaSuccess) return e;
  }
  h->epoch = (h->epoch % 0x7fffu) + 1;
  reset_kernel<<<1, 1, 0, s>>>(h->tree.ctrl, h->epoch);
  count_launch();
  return cudaGetLastError();
}

// Bulk loader: replaces the contents.  Same packing rule as the oracle
// (bto_bulk_build): ceil(m/leaf_fill) leaves of even size, inner levels of
// inner_fill+1 children per node, leaves first in id order.
int tree_bulk_build(Handle* h, const uint64_t* keys, const uint64_t* vals, size_t n, cudaStream_t s) {
  cudaError_t e = tree_reset(h, s);
  if (e != cudaSuccess) return -2;
  if (n == 0) return 0;
  if (n > 0xFFFFFFFFull / 2) return -1;
  // temporaries (stream ordered)
  uint64_t *ka = nullptr, *kb = nullptr, *uk = nullptr, *uv = nullptr;
  uint32_t *va = nullptr, *vb = nullptr, *flags = nullptr, *pos = nullptr, *scratch = nullptr, *tot = nullptr;
  size_t scw = sort_scratch_words(n);
  if (scan_scratch_words(n) > scw) scw = scan_scratch_words(n);
  bool ok = cudaMallocAsync(&ka, n * 8, s) == cudaSuccess && cudaMallocAsync(&kb, n * 8, s) == cudaSuccess &&
            cudaMallocAsync(&va, n * 4, s) == cudaSuccess && cudaMallocAsync(&vb, n * 4, s) == cudaSuccess &&
            cudaMallocAsync(&scratch, scw * 4, s) == cudaSuccess && cudaMallocAsync(&tot, 64, s) == cudaSuccess;
  int rc = 0;
  uint64_t* sk = nullptr;
  uint32_t* si = nullptr;
  uint64_t last_key = 0;
  uint32_t m32 = 0;
  if (!ok) { rc = -3; goto done; }
  if (radix_sort_pairs(keys, nullptr, nullptr, ka, va, kb, vb, n, 0, 64, scratch, s, &sk, &si, &h->tree.ctrl->error) !=
      cudaSuccess) {
    rc = -2;
    goto done;
  }
  // reuse the other ping-pong buffers for flags / positions / unique pairs
  flags = (si == va) ? vb : va;
  uk = (sk == ka) ? kb : ka;
  if (cudaMallocAsync(&pos, n * 4, s) != cudaSuccess || cudaMallocAsync(&uv, n * 8, s) != cudaSuccess) {
    rc = -3;
    goto done;
  }
  tail_flags_kernel<<<blocks_for(n, 256), 256, 0, s>>>(sk, n, flags);
  count_launch();
  if (scan_exclusive_u32(flags, pos, n, tot, scratch, s) != cudaSuccess) { rc = -2; goto done; }
  dedupe_kernel<<<blocks_for(n, 256), 256, 0, s>>>(sk, si, vals, flags, pos, n, uk, uv);
  count_launch();
  cudaMemcpyAsync(&m32, tot, 4, cudaMemcpyDeviceToHost, s);
  cudaMemcpyAsync(&last_key, sk + (n - 1), 8, cudaMemcpyDeviceToHost, s);
  if (cudaStreamSynchronize(s) != cudaSuccess) { rc = -2; goto done; }
  if (last_key == kKeyMax) { rc = -5; goto done; }
  {
    const size_t m = m32;
    const uint32_t lf = h->leaf_fill, per = h->inner_fill + 1;
    const uint32_t nl = (uint32_t)((m + lf - 1) / lf);
    // count nodes first (capacity check)
    uint64_t total = nl;
    uint32_t cnt = nl, height = 1;
    while (cnt > 1) {
      cnt = (cnt + per - 1) / per;
      total += cnt;
      height++;
    }
    if (total > h->tree.cap) { rc = -4; goto done; }
    build_leaves_kernel<<<blocks_for((size_t)nl * 32, 256), 256, 0, s>>>(h->tree, uk, uv, m, nl, h->epoch);
    count_launch();
    uint32_t first_child = 0, n_children = nl, next = nl, level = 1;
    while (n_children > 1) {
      uint32_t nn = (n_children + per - 1) / per;
      build_inner_kernel<<<blocks_for((size_t)nn * 32, 256), 256, 0, s>>>(h->tree, first_child, n_children, next,
                                                                          nn, level, h->epoch);
      count_launch();
      first_child = next;
      next += nn;
      n_children = nn;
      level++;
    }
    set_root_kernel<<<1, 1, 0, s>>>(h->tree.ctrl, first_child, height - 1, (uint32_t)total, (uint64_t)m);
    count_launch();
    if (cudaGetLastError() != cudaSuccess) rc = -2;
  }
done:
  cudaFreeAsync(ka, s);
  cudaFreeAsync(kb, s);
  cudaFreeAsync(va, s);
  cudaFreeAsync(vb, s);
  cudaFreeAsync(scratch, s);
  cudaFreeAsync(tot, s);
  if (pos) cudaFreeAsync(pos, s);
  if (uv) cudaFreeAsync(uv, s);
  if (cudaStreamSynchronize(s) != cudaSuccess && rc == 0) rc = -2;
  return rc;
}

// Same bulk build with the scratch supplied by the caller (nothing allocated
// here); used by bt_bulk_build_static.  Packing rule identical to
// tree_bulk_build above.
int tree_bulk_build_scratch(Handle* h, const uint64_t* keys, const uint64_t* vals, size_t n, cudaStream_t s,
                            const BuildScratch& sc) {
  if (n > sc.cap) return -6;
  if (tree_reset(h, s) != cudaSuccess) return -2;
  if (n == 0) return cudaStreamSynchronize(s) == cudaSuccess ? 0 : -2;
  uint64_t* sk = nullptr;
  uint32_t* si = nullptr;
  if (radix_sort_pairs(keys, nullptr, nullptr, sc.ka, sc.va, sc.kb, sc.vb, n, 0, 64, sc.sort_scratch, s, &sk, &si, &h->tree.ctrl->error) !=
      cudaSuccess)
    return -2;
  uint32_t* flags = (si == sc.va) ? sc.vb : sc.va;
  uint64_t* uk = (sk == sc.ka) ? sc.kb : sc.ka;
  tail_flags_kernel<<<blocks_for(n, 256), 256, 0, s>>>(sk, n, flags);
  count_launch();
  if (scan_exclusive_u32(flags, sc.pos, n, sc.tot, sc.sort_scratch, s) != cudaSuccess) return -2;
  dedupe_kernel<<<blocks_for(n, 256), 256, 0, s>>>(sk, si, vals, flags, sc.pos, n, uk, sc.uv);
  count_launch();
  uint32_t m32 = 0;
  uint64_t last_key = 0;
  if (cudaMemcpyAsync(&m32, sc.tot, 4, cudaMemcpyDeviceToHost, s) != cudaSuccess ||
      cudaMemcpyAsync(&last_key, sk + (n - 1), 8, cudaMemcpyDeviceToHost, s) != cudaSuccess ||
      cudaStreamSynchronize(s) != cudaSuccess)
    return -2;
  if (last_key == kKeyMax) return -5;
  const size_t m = m32;
  const uint32_t lf = h->leaf_fill, per = h->inner_fill + 1;
  const uint32_t nl = (uint32_t)((m + lf - 1) / lf);
  uint64_t total = nl;
  uint32_t cnt = nl, height = 1;
  while (cnt > 1) {
    cnt = (cnt + per - 1) / per;
    total += cnt;
    height++;
  }
  if (total > h->tree.cap) return -4;
  build_leaves_kernel<<<blocks_for((size_t)nl * 32, 256), 256, 0, s>>>(h->tree, uk, sc.uv, m, nl, h->epoch);
  count_launch();
  uint32_t first_child = 0, n_children = nl, next = nl, level = 1;
  while (n_children > 1) {
    const uint32_t nn = (n_children + per - 1) / per;
    build_inner_kernel<<<blocks_for((size_t)nn * 32, 256), 256, 0, s>>>(h->tree, first_child, n_children, next, nn,
                                                                        level, h->epoch);
    count_launch();
    first_child = next;
    next += nn;
    n_children = nn;
    level++;
  }
  set_root_kernel<<<1, 1, 0, s>>>(h->tree.ctrl, first_child, height - 1, (uint32_t)total, (uint64_t)m);
  count_launch();
  if (cudaGetLastError() != cudaSuccess) return -2;
  return cudaStreamSynchronize(s) == cudaSuccess ? 0 : -2;
}

cudaError_t launch_search_sorted(Handle* h, const uint64_t* qkeys, const uint32_t* list, const uint32_t* n_dev,
                                 size_t n, uint64_t* out_vals, uint8_t* out_st, cudaStream_t s) {
  if (n == 0) return cudaSuccess;
  // one resident wave of groups; each group takes a contiguous chunk
  const int threads = 256;
  static int per_sm[64][2] = {};
  const int lv = h->sorted_leaf_vals ? 1 : 0;
  if (h->device < 64 && per_sm[h->device][lv] == 0) {
    int b = 0;
    cudaError_t e = lv ? cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b, search_sorted_kernel<8, true>, threads, 0)
                       : cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b, search_sorted_kernel<8, false>, threads, 0);
    if (e != cudaSuccess || b < 1) b = 4;
    per_sm[h->device][lv] = b;
  }
  const size_t blocks = (size_t)h->sm_count * (h->device < 64 ? per_sm[h->device][lv] : 4);
  if (lv) search_sorted_kernel<8, true><<<(unsigned)blocks, threads, 0, s>>>(h->tree, qkeys, list, n_dev, n, out_vals, out_st);
  else search_sorted_kernel<8, false><<<(unsigned)blocks, threads, 0, s>>>(h->tree, qkeys, list, n_dev, n, out_vals, out_st);
  count_launch();
  return cudaGetLastError();
}

// Prefix rows of every inner node from its keys: one warp per 32 nodes reads
// their headers (one sector each), then writes the rows of the inner ones.
__global__ void __launch_bounds__(256) pfx_rebuild_kernel(DevTree t) {
  const uint32_t lane = threadIdx.x & 31;
  const uint32_t n_nodes = min(t.ctrl->n_nodes, t.cap);
  const uint32_t warps = (gridDim.x * blockDim.x) >> 5;
  for (uint32_t b = ((blockIdx.x * blockDim.x + threadIdx.x) >> 5) * 32; b < n_nodes; b += warps * 32) {
    const uint32_t mine = b + lane;
    const bool inner = mine < n_nodes && hdr_level(t.keys[(size_t)mine * 32 + 31]) > 0;
    uint32_t todo = __ballot_sync(0xffffffffu, inner);
    while (todo) {
      const uint32_t nd = b + (uint32_t)(__ffs(todo) - 1);
      todo &= todo - 1;
      const uint64_t k = t.keys[(size_t)nd * 32 + lane];
      t.pfx[(size_t)nd * 32 + lane] = lane < 31 ? (uint32_t)(k >> 32) : 0xffffffffu;
    }
  }
}

cudaError_t ensure_pfx(Handle* h, cudaStream_t s) {
  if (h->pfx_valid) return cudaSuccess;
  pfx_rebuild_kernel<<<(unsigned)h->sm_count * 8, 256, 0, s>>>(h->tree);
  count_launch();
  h->pfx_valid = true;
  return cudaGetLastError();
}

cudaError_t launch_search(Handle* h, const uint64_t* qkeys, const uint32_t* list, const uint32_t* n_dev, size_t n,
                          uint64_t* out_vals, uint8_t* out_st, cudaStream_t s, const uint64_t* ckeys) {
  if (n == 0) return cudaSuccess;
  if (h->search_pairs && (h->search_group == 8 || h->search_group == 4 || h->search_group == 16)) {
    const int threads = 256;
    const int G = h->search_group;
    size_t blocks = ((n + 1) / 2 * (size_t)G + threads - 1) / threads;
    size_t cap = (size_t)h->sm_count * 8 * 4;
    if (h->lookup_reserve > 0) {
      // a resident, grid-striding launch that leaves `lookup_reserve` block
      // slots free for kernels running beside it (the overlapped sort)
      static int per_sm[64][3] = {};
      const int gi = G == 4 ? 0 : G == 16 ? 2 : 1;
      const int dev = h->device;
      int per = (dev >= 0 && dev < 64) ? per_sm[dev][gi] : 0;
      if (per == 0) {
        const void* k = G == 4 ? (const void*)search2_kernel<4, false, true>
                        : G == 16 ? (const void*)search2_kernel<16, false, true>
                                  : (const void*)search2_kernel<8, false, true>;
        if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, k, threads, 0) != cudaSuccess || per < 1) per = 1;
        if (dev >= 0 && dev < 64) per_sm[dev][gi] = per;
      }
      const size_t resident = (size_t)h->sm_count * per;
      cap = resident > (size_t)h->lookup_reserve + h->sm_count ? resident - h->lookup_reserve : h->sm_count;
    }
    if (blocks > cap) blocks = cap;
    if (blocks == 0) blocks = 1;
    const bool child = h->search_pairs == 2;
    // the separators' prefixes (child-id form only)
    const int use_pfx = child && h->use_pfx ? 1 : 0;
    if (use_pfx) {
      const cudaError_t pe = ensure_pfx(h, s);
      if (pe != cudaSuccess) return pe;
    }
#define BT_S2(GG, CC) search2_kernel<GG, false, CC><<<(unsigned)blocks, threads, 0, s>>>(h->tree, qkeys, list, n_dev, n, out_vals, out_st, use_pfx, list ? ckeys : nullptr)
    if (G == 4) { if (child) BT_S2(4, true); else BT_S2(4, false); }
    else if (G == 16) { if (child) BT_S2(16, true); else BT_S2(16, false); }
    else { if (child) BT_S2(8, true); else BT_S2(8, false); }
#undef BT_S2
    count_launch();
    return cudaGetLastError();
  }
  if (h->top_cache) return launch_search_top(h, qkeys, list, n_dev, n, out_vals, out_st, s);
  const int threads = 256;
  const int G = h->search_group;
  // enough groups to cover the requests, capped at a few waves of resident blocks
  size_t groups_needed = n;
  size_t blocks = (groups_needed * G + threads - 1) / threads;
  size_t cap = (size_t)h->sm_count * 8 * 4;
  if (blocks > cap) blocks = cap;
  if (blocks == 0) blocks = 1;
  switch (G) {
    case 4: search_kernel<4, false><<<(unsigned)blocks, threads, 0, s>>>(h->tree, qkeys, list, n_dev, n, out_vals, out_st); break;
    case 16: search_kernel<16, false><<<(unsigned)blocks, threads, 0, s>>>(h->tree, qkeys, list, n_dev, n, out_vals, out_st); break;
    case 32: search_kernel<32, false><<<(unsigned)blocks, threads, 0, s>>>(h->tree, qkeys, list, n_dev, n, out_vals, out_st); break;
    case -8: search_kernel<8, true><<<(unsigned)blocks, threads, 0, s>>>(h->tree, qkeys, list, n_dev, n, out_vals, out_st); break;
    default: search_kernel<8, false><<<(unsigned)blocks, threads, 0, s>>>(h->tree, qkeys, list, n_dev, n, out_vals, out_st); break;
  }
  count_launch();
  return cudaGetLastError();
}

cudaError_t launch_range(Handle* h, const uint64_t* lo, const uint64_t* hi, size_t n, uint32_t max_per,
                         uint64_t* out_keys, uint64_t* out_vals, uint32_t* out_counts, cudaStream_t s) {
  if (n == 0) return cudaSuccess;
  size_t blocks = (n * 32 + 255) / 256;
  const size_t cap = (size_t)h->sm_count * 16;
  if (blocks > cap) blocks = cap;
  range_kernel<<<(unsigned)blocks, 256, 0, s>>>(h->tree, lo, hi, n, max_per, out_keys, out_vals, out_counts);
  count_launch();
  return cudaGetLastError();
}

// grown with a quarter of headroom: the tree grows a little with every batch,
// and a reallocation (cudaFree synchronises the device) on every refit or
// dump stalled the batches queued behind it
static int ensure_enum(Handle* h, size_t n) {
  if (n <= h->enum_cap) return 0;
  n += n / 4 + 4096;
  cudaFree(h->enum_a);
  cudaFree(h->enum_b);
  cudaFree(h->enum_cnt);
  cudaFree(h->enum_scan_scratch);
  h->enum_a = h->enum_b = h->enum_cnt = h->enum_scan_scratch = nullptr;
  h->enum_cap = 0;
  size_t c = n + 64;
  if (cudaMalloc(&h->enum_a, c * 4) != cudaSuccess || cudaMalloc(&h->enum_b, c * 4) != cudaSuccess ||
      cudaMalloc(&h->enum_cnt, (c + 1) * 4) != cudaSuccess ||
      cudaMalloc(&h->enum_scan_scratch, (scan_scratch_words(c) + 1) * 4) != cudaSuccess)
    return -3;
  h->enum_cap = c;
  return 0;
}

int enumerate_leaves(Handle* h, cudaStream_t s, uint32_t** leaf_ids, size_t* n_leaves) {
  Ctrl c;
  if (cudaMemcpyAsync(&c, h->tree.ctrl, sizeof(Ctrl), cudaMemcpyDeviceToHost, s) != cudaSuccess) return -2;
  if (cudaStreamSynchronize(s) != cudaSuccess) return -2;
  *n_leaves = 0;
  *leaf_ids = nullptr;
  h->n_levels = 0;
  if (c.root == kNil) return 0;
  h->n_levels = c.root_level + 1;
  if (h->n_levels <= 48) h->level_counts[c.root_level] = 1;
  if (ensure_enum(h, c.n_nodes + 1) != 0) return -3;
  uint32_t* cur = h->enum_a;
  uint32_t* nxt = h->enum_b;
  cudaMemcpyAsync(cur, &c.root, 4, cudaMemcpyHostToDevice, s);
  size_t n = 1;
  uint32_t* tot = h->enum_cnt + h->enum_cap;  // last word
  for (uint32_t l = c.root_level; l > 0; l--) {
    child_count_kernel<<<blocks_for(n, 256), 256, 0, s>>>(h->tree, cur, n, h->enum_cnt, 0);
    count_launch();
    if (scan_exclusive_u32(h->enum_cnt, h->enum_cnt, n, tot, h->enum_scan_scratch, s) != cudaSuccess) return -2;
    child_write_kernel<<<blocks_for(n * 32, 256), 256, 0, s>>>(h->tree, cur, n, h->enum_cnt, nxt);
    count_launch();
    uint32_t m = 0;
    cudaMemcpyAsync(&m, tot, 4, cudaMemcpyDeviceToHost, s);
    if (cudaStreamSynchronize(s) != cudaSuccess) return -2;
    n = m;
    if (l - 1 < 48) h->level_counts[l - 1] = m;
    uint32_t* t = cur;
    cur = nxt;
    nxt = t;
  }
  *leaf_ids = cur;
  *n_leaves = n;
  return 0;
}

cudaError_t leaf_sizes_device(Handle* h, const uint32_t* leaves, size_t n, uint32_t* out, cudaStream_t s) {
  if (n == 0) return cudaSuccess;
  child_count_kernel<<<blocks_for(n, 256), 256, 0, s>>>(h->tree, leaves, n, out, 1);
  count_launch();
  return cudaGetLastError();
}

int tree_dump(Handle* h, uint64_t* out_keys, uint64_t* out_vals, size_t cap, size_t* n_out, cudaStream_t s) {
  uint32_t* leaves = nullptr;
  size_t nl = 0;
  int rc = enumerate_leaves(h, s, &leaves, &nl);
  if (rc) return rc;
  *n_out = 0;
  if (nl == 0) return 0;
  // leaves live in one enum buffer; use the other for sizes
  uint32_t* sizes = (leaves == h->enum_a) ? h->enum_b : h->enum_a;
  uint32_t* tot = h->enum_cnt + h->enum_cap;
  child_count_kernel<<<blocks_for(nl, 256), 256, 0, s>>>(h->tree, leaves, nl, sizes, 1);
  count_launch();
  if (scan_exclusive_u32(sizes, sizes, nl, tot, h->enum_scan_scratch, s) != cudaSuccess) return -2;
  uint32_t total = 0;
  cudaMemcpyAsync(&total, tot, 4, cudaMemcpyDeviceToHost, s);
  if (cudaStreamSynchronize(s) != cudaSuccess) return -2;
  *n_out = total;
  if (total > cap) return -4;
  leaf_dump_kernel<<<blocks_for(nl * 32, 256), 256, 0, s>>>(h->tree, leaves, nl, sizes, out_keys, out_vals);
  count_launch();
  if (cudaStreamSynchronize(s) != cudaSuccess) return -2;
  return 0;
}

}  // namespace bt
