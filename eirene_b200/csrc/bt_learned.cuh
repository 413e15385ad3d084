// Learned leaf predictor: layout of the model tables and the device-side
// leaf prediction, shared by the lookup kernels (bt_learned.cu) and the STM
// fast path (bt_stm.cu).
#pragma once
#include "bt_common.cuh"
#include "bt_search.cuh"

namespace bt {

struct LeafEnt {
  uint64_t low;
  uint64_t id;
};

// Segment line, 16 B: predicted slot = a + slope * (key - base).  A segment
// with no usable line (no training leaf, or a maximum error above the
// window) has a = NaN, so its keys skip the probe and go to the fallback.
struct SegParam {
  uint64_t base;
  float a;
  float slope;
};

constexpr int kHidden = 32;
constexpr int kParams = 3 * kHidden + 1;  // w1[32] b1[32] w2[32] b2
constexpr uint32_t kErrNone = 0xFFFFFFFFu;

// the key mapped to [0, 1] over the training key range (float arithmetic:
// training and lookups evaluate the same expression)
__device__ __forceinline__ float norm_x(uint64_t key, uint64_t kmin, float inv_range) {
  if (key <= kmin) return 0.f;
  const float x = __ull2float_rn(key - kmin) * inv_range;
  return x >= 1.f ? 1.f : x;
}

__device__ __forceinline__ uint32_t seg_of_y(float y, uint32_t n_seg) {
  float f = y * (float)n_seg;
  if (!(f > 0.f)) return 0;
  if (f >= (float)(n_seg - 1)) return n_seg - 1;
  return (uint32_t)f;
}

// slot predicted by a segment line, in the exact arithmetic the lookup uses;
// the offset from the segment's base as a signed 64-bit value (a key more
// than 2^63 away from it wraps: a wrong prediction, which the probe rejects)
__device__ __forceinline__ float seg_predict(const SegParam& sp, uint64_t key) {
  const float d = __ll2float_rn((long long)(key - sp.base));
  return fmaf(sp.slope, d, sp.a);
}

// one 16-byte load of segment j's line
__device__ __forceinline__ SegParam load_seg(const SegParam* seg, uint32_t j) {
  const ulonglong2 w = __ldg(reinterpret_cast<const ulonglong2*>(seg + j));
  SegParam sp;
  sp.base = w.x;
  sp.a = __uint_as_float((uint32_t)w.y);
  sp.slope = __uint_as_float((uint32_t)(w.y >> 32));
  return sp;
}

// stage 1 for one request served by a group of G lanes: lane g evaluates the
// hidden units g, g + G, ...; the group sums the output with xor-shuffles
template <int G>
__device__ __forceinline__ float mlp_group(const float* p, float x, uint32_t g, uint32_t gmask) {
  float y = 0.f;
#pragma unroll
  for (int jj = 0; jj < kHidden / G; jj++) {
    const int j = g + jj * G;
    const float h = fmaf(p[j], x, p[kHidden + j]);
    if (h > 0.f) y = fmaf(p[2 * kHidden + j], h, y);
  }
#pragma unroll
  for (int o = G / 2; o >= 1; o >>= 1) y += __shfl_xor_sync(gmask, y, o, G);
  return y + p[3 * kHidden];
}

// The adaptive gate (BT_OPT_LEARNED_POLICY 1 and 2): a judge kernel after
// each learned lookup launch compares the hit and fallback counters with
// the last judged ones; once a window of at least kGateWindow lookups missed
// more than 1 in kGateMissDen, `stale` stays set until the model is fitted
// again, and the learned kernels hand every request to the plain descent.
constexpr unsigned long long kGateWindow = 65536;
constexpr unsigned long long kGateMissDen = 20;  // 5 %
struct LearnedGate {
  unsigned long long base_hits, base_falls;
  uint32_t stale;
  uint32_t have_base;
};

struct LearnedDev {
  const LeafEnt* tab;
  const SegParam* seg;
  const float* params;
  uint64_t kmin;
  float inv_range;
  uint32_t n_leaves;
  uint32_t n_seg;
  uint32_t window;
  const LearnedGate* gate;  // nullptr: always use the model (policy 0)
  uint64_t* miss_keys;      // the misses' keys, beside their request indices
};

// Predicted leaf for `key`: stage 1 (MLP) -> segment -> line -> one probe of
// the G leaf-table entries around the predicted slot.  Returns the leaf's node
// id, or kNil when the probe does not bracket the key (caller falls back).
template <int G>
__device__ __forceinline__ uint32_t learned_leaf(const LearnedDev& M, const float* p, uint64_t key, uint32_t g,
                                                 uint32_t gmask, uint32_t& dist) {
  const float y = mlp_group<G>(p, norm_x(key, M.kmin, M.inv_range), g, gmask);
  const SegParam sp = load_seg(M.seg, seg_of_y(y, M.n_seg));
  if (sp.a != sp.a) return kNil;  // segment without a usable line
  const float pred = seg_predict(sp, key);
  const int L = (int)M.n_leaves;
  int pc = (pred > 0.f) ? (pred < (float)(L - 1) ? __float2int_rn(pred) : L - 1) : 0;
  // probe the G entries [p0, p0 + G) and the one above them
  int p0 = pc - (G / 2 - 1);
  p0 = p0 > L - G ? L - G : p0;
  p0 = p0 < 0 ? 0 : p0;
  const int e = p0 + (int)g;
  // the leaf table is read by every lookup: keep it in L2
  const uint64_t keep = l2_keep();
  ulonglong2 ent = make_ulonglong2(kKeyMax, 0);
  if (e <= L) ent = ldg2_hint(reinterpret_cast<const ulonglong2*>(M.tab) + e, keep);
  uint64_t above = kKeyMax;
  if (g == 0 && p0 + G <= L) above = ldg_hint(&M.tab[p0 + G].low, keep);
  above = __shfl_sync(gmask, above, 0, G);
  const uint32_t c = group_sum<G>(ent.x <= key ? 1u : 0u, gmask);
  const uint32_t node = (uint32_t)__shfl_sync(gmask, ent.y, (c + G - 1) % G, G);
  if (c >= 1 && (c < (uint32_t)G || above > key)) {
    const int slot = p0 + (int)c - 1;
    dist = (uint32_t)(pc > slot ? pc - slot : slot - pc);
    return node;
  }
  return kNil;
}

}  // namespace bt
