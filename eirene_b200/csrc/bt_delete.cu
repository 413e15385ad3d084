// Delete phase of a sorted batch (op code DELETE = 2, src/input-helper.h:16,
// declared by the reference and implemented by none of its versions).
//
// Input: the unique keys whose run ends with a DELETE (w.del_list, ascending
// keys, count on the device).  Two kernels:
//   del_locate_kernel  one 8-lane group per key descends to its leaf and
//                      records the leaf and the key's slot (or none), and
//                      answers the run's first request with the key's
//                      pre-batch value;
//   del_apply_kernel   one warp per leaf (equal leaves are adjacent because
//                      the keys ascend) removes all of that leaf's found keys
//                      at once: a ballot over the row keeps the others in
//                      order and the header gets the new size.
// Leaves shrink in place: no merge with siblings; an emptied leaf stays and
// its separators keep routing (searches in it find nothing, inserts refill
// it).  The locate may run beside lookups of other keys (it writes no node);
// the apply runs before the insert phase with no other kernel on the tree.  HBM traffic per deleted key: the descent (288 B at the leaf)
// and, per touched leaf, one 512 B row read and written.
#include <cuda_runtime.h>

#include "bt_common.cuh"
#include "bt_internal.h"
#include "bt_search.cuh"

namespace bt {

namespace {

constexpr int kG = 8;
constexpr int kS = 32 / kG;
constexpr uint32_t kNoSlot = 0xFFFFFFFFu;

__global__ void __launch_bounds__(256) del_locate_kernel(DevTree t, const uint64_t* __restrict__ ukeys,
                                                         const uint32_t* __restrict__ del_list,
                                                         const uint32_t* __restrict__ n_dev,
                                                         uint32_t* __restrict__ dleaf, uint32_t* __restrict__ dslot,
                                                         uint64_t* __restrict__ uans, uint8_t* __restrict__ uans_st) {
  const uint32_t lane = threadIdx.x & 31;
  const uint32_t g = lane % kG;
  const uint32_t gmask = group_mask<kG>(lane);
  const size_t n = *n_dev;
  const uint32_t root = t.ctrl->root;
  const uint32_t root_level = t.ctrl->root_level;
  const size_t stride = ((size_t)gridDim.x * blockDim.x) / kG;
  for (size_t i = ((size_t)blockIdx.x * blockDim.x + threadIdx.x) / kG; i < n; i += stride) {
    const uint32_t u = del_list[i];
    const uint64_t key = ukeys[u];
    uint32_t node = root, slot = kNoSlot;
    uint64_t old = 0;
    if (root != kNil) {
      uint64_t k[kS];
      uint32_t cnt = 0;
      for (uint32_t level = root_level;; level--) {
        load_slots<kS>(t.keys + (size_t)node * 32 + g * kS, k);
        if (g == kG - 1) k[kS - 1] = kKeyMax;  // slot 31 holds the header
        uint32_t c = 0;
#pragma unroll
        for (int x = 0; x < kS; x++) c += (k[x] <= key) ? 1u : 0u;
        cnt = group_sum<kG>(c, gmask);
        if (level == 0) break;
        node = (uint32_t)__ldg(t.vals + (size_t)node * 32 + cnt);
      }
      const uint32_t s = cnt > 0 ? cnt - 1 : 0;
      const uint64_t kk = __shfl_sync(gmask, pick<kS>(k, s % kS), s / kS, kG);
      if (cnt > 0 && kk == key) {
        slot = s;
        old = __ldg(t.vals + (size_t)node * 32 + s);
      }
    } else {
      node = kNil;
    }
    if (g == 0) {
      dleaf[i] = node;
      dslot[i] = slot;
      uans[u] = slot != kNoSlot ? old : 0;
      uans_st[u] = slot != kNoSlot ? kFound : kAbsent;
    }
  }
}

__global__ void __launch_bounds__(256) del_apply_kernel(DevTree t, const uint32_t* __restrict__ n_dev,
                                                        const uint32_t* __restrict__ dleaf,
                                                        const uint32_t* __restrict__ dslot) {
  const uint32_t lane = threadIdx.x & 31;
  const size_t n = *n_dev;
  const size_t warps = ((size_t)gridDim.x * blockDim.x) >> 5;
  unsigned long long removed = 0;
  for (size_t i = ((size_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5; i < n; i += warps) {
    const uint32_t leaf = dleaf[i];
    if (leaf == kNil || (i > 0 && dleaf[i - 1] == leaf)) continue;  // not the first entry of its leaf
    // slots to remove: every found entry of this leaf (entries of a leaf are adjacent)
    uint32_t gone = 0;
    for (size_t j = i;; j += 32) {
      const size_t x = j + lane;
      const bool mine = x < n && dleaf[x] == leaf;
      const uint32_t sl = mine ? dslot[x] : kNoSlot;
      uint32_t bit = (mine && sl != kNoSlot) ? (1u << sl) : 0u;
      bit = __reduce_or_sync(0xffffffffu, bit);
      gone |= bit;
      if (__ballot_sync(0xffffffffu, mine) != 0xffffffffu) break;
    }
    if (!gone) continue;
    uint64_t* kr = t.keys + (size_t)leaf * 32;
    uint64_t* vr = t.vals + (size_t)leaf * 32;
    const uint64_t k = kr[lane];
    const uint64_t v = vr[lane];
    const uint64_t h = __shfl_sync(0xffffffffu, k, 31);
    const uint32_t sz = hdr_size(h);
    const bool keep = lane < sz && !((gone >> lane) & 1u);
    const uint32_t keepm = __ballot_sync(0xffffffffu, keep);
    const uint32_t nsz = __popc(keepm);
    const uint32_t pos = __popc(keepm & ((1u << lane) - 1u));
    __syncwarp();
    if (keep) {
      kr[pos] = k;
      vr[pos] = v;
    }
    __syncwarp();
    if (lane >= nsz && lane < 31) {
      kr[lane] = kKeyMax;
      vr[lane] = 0;
    }
    if (lane == 31) kr[31] = make_hdr(nsz, 0, hdr_version(h) + 1, hdr_epoch(h));
    removed += sz - nsz;
  }
  if (lane == 0 && removed) atomicAdd(&t.ctrl->n_keys, (unsigned long long)0 - removed);
}

}  // namespace

// The batch's DELETE runs (before its inserts), in two launches: the locate
// reads the tree only, the apply removes the keys.  n_upper bounds the device
// count w.counts->n_del.
int delete_locate(Handle* h, size_t n_upper, cudaStream_t s) {
  Work& w = h->w;
  const unsigned blocks = (unsigned)min((size_t)h->sm_count * 8, (n_upper * kG + 255) / 256 + 1);
  del_locate_kernel<<<blocks, 256, 0, s>>>(h->tree, w.ukeys, w.del_list, &w.counts->n_del, w.d_leaf, w.d_slot,
                                           w.uans, w.uans_st);
  count_launch();
  return cudaGetLastError() == cudaSuccess ? 0 : -2;
}

int delete_apply(Handle* h, size_t n_upper, cudaStream_t s) {
  Work& w = h->w;
  del_apply_kernel<<<(unsigned)min((size_t)h->sm_count * 8, (n_upper * 32 + 255) / 256 + 1), 256, 0, s>>>(
      h->tree, &w.counts->n_del, w.d_leaf, w.d_slot);
  count_launch();
  return cudaGetLastError() == cudaSuccess ? 0 : -2;
}

}  // namespace bt
