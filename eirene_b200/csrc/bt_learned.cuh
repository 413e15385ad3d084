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

struct SegParam {
  uint64_t base;
  float inv_span;
  float a;
  float b;
  uint32_t err;
};

constexpr int kHidden = 32;
constexpr int kParams = 3 * kHidden + 1;  // w1[32] b1[32] w2[32] b2
constexpr uint32_t kErrNone = 0xFFFFFFFFu;

__device__ __forceinline__ float norm_x(uint64_t key, uint64_t kmin, double inv_range) {
  if (key <= kmin) return 0.f;
  const double x = (double)(key - kmin) * inv_range;
  return x >= 1.0 ? 1.f : (float)x;
}

__device__ __forceinline__ uint32_t seg_of_y(float y, uint32_t n_seg) {
  float f = y * (float)n_seg;
  if (!(f > 0.f)) return 0;
  if (f >= (float)(n_seg - 1)) return n_seg - 1;
  return (uint32_t)f;
}

// slot predicted by a segment line, in the exact arithmetic the lookup uses
__device__ __forceinline__ float seg_predict(const SegParam& sp, uint64_t key) {
  const float d = key >= sp.base ? (float)(key - sp.base) : -(float)(sp.base - key);
  return fmaf(sp.b, d * sp.inv_span, sp.a);
}

struct LearnedDev {
  const LeafEnt* tab;
  const SegParam* seg;
  const float* params;
  uint64_t kmin;
  double inv_range;
  uint32_t n_leaves;
  uint32_t n_seg;
  uint32_t window;
};

// Predicted leaf for `key`: stage 1 (MLP) -> segment -> line -> one probe of
// the G leaf-table entries around the predicted slot.  Returns the leaf's node
// id, or kNil when the probe does not bracket the key (caller falls back).
template <int G>
__device__ __forceinline__ uint32_t learned_leaf(const LearnedDev& M, const float* p, uint64_t key, uint32_t g,
                                                 uint32_t gmask, uint32_t& dist) {
  const float x = norm_x(key, M.kmin, M.inv_range);
  float y = 0.f;
#pragma unroll
  for (int jj = 0; jj < kHidden / G; jj++) {
    const int j = g + jj * G;
    const float h = fmaf(p[j], x, p[kHidden + j]);
    if (h > 0.f) y = fmaf(p[2 * kHidden + j], h, y);
  }
#pragma unroll
  for (int o = G / 2; o >= 1; o >>= 1) y += __shfl_xor_sync(gmask, y, o, G);
  y += p[3 * kHidden];
  const uint64_t* w = reinterpret_cast<const uint64_t*>(M.seg + seg_of_y(y, M.n_seg));
  SegParam sp;
  sp.base = __ldg(w);
  const uint64_t w1 = __ldg(w + 1), w2 = __ldg(w + 2);
  sp.inv_span = __uint_as_float((uint32_t)w1);
  sp.a = __uint_as_float((uint32_t)(w1 >> 32));
  sp.b = __uint_as_float((uint32_t)w2);
  if ((uint32_t)(w2 >> 32) == kErrNone) return kNil;  // segment without a model
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
