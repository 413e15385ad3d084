// Learned leaf predictor (no counterpart in the reference; its nearest
// structure is v35's sorted leaf array, src/gpu-stm-tree-v35/bpt-gpustm.h:58-61,
// src/gpu-stm-tree-v35/bpt-gpustm-kernel.cu:135-152).
//
// Two-stage model over the tree's own (leaf low key -> leaf slot) pairs, in
// the style of a recursive model index (Kraska et al., "The Case for Learned
// Index Structures", SIGMOD 2018):
//   stage 1: a 1 -> 32 (ReLU) -> 1 FP32 MLP maps the normalised key to the
//            leaf CDF and picks one of n_segments segments;
//   stage 2: per segment, a least-squares line key -> slot, with the maximum
//            error over its training leaves.
// A lookup predicts slot p, reads the window [p-err-1, p+err+1] of the leaf
// table, finds the last leaf whose low fence is <= key, checks the leaf's own
// right fence, and answers from that leaf.  Any failed check (error above the
// window limit, key outside the window, a leaf split since training) falls
// back to the plain root descent, so results are the plain tree's results.
//
// Training is done on the GPU by the kernels below: MLP forward + backward
// (per-block partial gradients, reduced in a fixed order so the gradient is
// deterministic), Adam update; the step is captured once in a CUDA graph and
// replayed.  Segment fits use per-run warp aggregation and double atomics.
#include <cooperative_groups.h>
#include <cmath>
#include <cstring>
#include <vector>

#include <cuda_runtime.h>

#include "bt_common.cuh"
#include "bt_internal.h"
#include "bt_learned.cuh"
#include "bt_search.cuh"

namespace bt {

struct SegAcc {
  unsigned long long kmin;
  unsigned long long kmax;
  unsigned int count;
  unsigned int pad;
  double su, suu, sy, suy;
};

namespace {

constexpr int kGradBlocks = 148;
constexpr int kGradThreads = 256;
constexpr int kPartStride = kParams + 1;  // + loss


__device__ __forceinline__ float mlp_fwd(const float* p, float x) {
  float y = p[3 * kHidden];
#pragma unroll
  for (int j = 0; j < kHidden; j++) {
    const float h = fmaf(p[j], x, p[kHidden + j]);
    if (h > 0.f) y = fmaf(p[2 * kHidden + j], h, y);
  }
  return y;
}



// ---------------------------------------------------------------- tables ----
__global__ void leaf_table_kernel(DevTree t, const uint32_t* __restrict__ ids, size_t L, LeafEnt* __restrict__ tab) {
  const size_t s = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (s < L) {
    const uint32_t id = ids[s];
    tab[s].low = t.low[id];
    tab[s].id = id;
  } else if (s == L) {
    tab[s].low = kKeyMax;
    tab[s].id = 0;
  }
}

__global__ void train_samples_kernel(const LeafEnt* __restrict__ tab, size_t L, size_t M, uint64_t kmin,
                                     float inv_range, float* __restrict__ xs, float* __restrict__ ys) {
  const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= M) return;
  const size_t s = 1 + (i * (L - 1)) / M;
  xs[i] = norm_x(tab[s].low, kmin, inv_range);
  ys[i] = (float)((double)s / (double)L);
}

// --------------------------------------------------------------- training ----
// MSE over (x, y): per-block partial gradients [block][kPartStride]
__global__ void __launch_bounds__(kGradThreads) mlp_grad_kernel(const float* __restrict__ params,
                                                                const float* __restrict__ xs,
                                                                const float* __restrict__ ys, size_t M,
                                                                float* __restrict__ partial) {
  __shared__ float p[kParams];
  __shared__ float red[kGradThreads / 32][kPartStride];
  for (int i = threadIdx.x; i < kParams; i += blockDim.x) p[i] = params[i];
  __syncthreads();
  float g[kPartStride];
#pragma unroll
  for (int i = 0; i < kPartStride; i++) g[i] = 0.f;
  const float inv_m = 1.0f / (float)M;
  const size_t stride = (size_t)gridDim.x * blockDim.x;
  for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < M; i += stride) {
    const float x = xs[i];
    float h[kHidden];
    float y = p[3 * kHidden];
#pragma unroll
    for (int j = 0; j < kHidden; j++) {
      const float a = fmaf(p[j], x, p[kHidden + j]);
      h[j] = a > 0.f ? a : 0.f;
      y = fmaf(p[2 * kHidden + j], h[j], y);
    }
    const float d = y - ys[i];
    const float go = 2.f * d * inv_m;
    g[kParams] += d * d * inv_m;
    g[3 * kHidden] += go;
#pragma unroll
    for (int j = 0; j < kHidden; j++) {
      g[2 * kHidden + j] = fmaf(go, h[j], g[2 * kHidden + j]);
      if (h[j] > 0.f) {
        const float gh = go * p[2 * kHidden + j];
        g[j] = fmaf(gh, x, g[j]);
        g[kHidden + j] += gh;
      }
    }
  }
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
  for (int i = 0; i < kPartStride; i++) {
    float v = g[i];
#pragma unroll
    for (int o = 16; o >= 1; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    if (lane == 0) red[warp][i] = v;
  }
  __syncthreads();
  for (int i = threadIdx.x; i < kPartStride; i += blockDim.x) {
    float v = 0.f;
    for (int w = 0; w < kGradThreads / 32; w++) v += red[w][i];
    partial[(size_t)blockIdx.x * kPartStride + i] = v;
  }
}

// fixed-order reduction of the partials, then (optionally) one Adam step
__global__ void mlp_reduce_adam_kernel(float* __restrict__ params, const float* __restrict__ partial, int blocks,
                                       float* __restrict__ m1, float* __restrict__ m2, int* __restrict__ step,
                                       float lr, float* __restrict__ grad_out, float* __restrict__ loss_out,
                                       int update) {
  const int i = threadIdx.x;
  __shared__ int t_s;
  if (i == 0) t_s = update ? ++(*step) : *step;
  __syncthreads();
  if (i >= kPartStride) return;
  float gsum = 0.f;
  for (int b = 0; b < blocks; b++) gsum += partial[(size_t)b * kPartStride + i];
  if (i == kParams) {
    if (loss_out) *loss_out = gsum;
    return;
  }
  if (grad_out) grad_out[i] = gsum;
  if (!update) return;
  const float b1 = 0.9f, b2 = 0.999f, eps = 1e-8f;
  const float a = b1 * m1[i] + (1.f - b1) * gsum;
  const float v = b2 * m2[i] + (1.f - b2) * gsum * gsum;
  m1[i] = a;
  m2[i] = v;
  const float t = (float)t_s;
  const float ah = a / (1.f - powf(b1, t));
  const float vh = v / (1.f - powf(b2, t));
  params[i] -= lr * ah / (sqrtf(vh) + eps);
}

// --------------------------------------------------------------- segments ----
// Each thread walks a contiguous chunk of leaves and flushes one atomic per
// run of equal segment ids.
constexpr int kChunk = 32;

__global__ void seg_init_kernel(SegAcc* __restrict__ acc, uint32_t n_seg, unsigned int* __restrict__ bad) {
  const uint32_t j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j < n_seg) {
    SegAcc a{};
    a.kmin = ~0ull;
    acc[j] = a;
  }
  if (j == 0) *bad = 0;
}

__global__ void seg_assign_kernel(const LeafEnt* __restrict__ tab, size_t L, const float* __restrict__ params,
                                  uint64_t kmin, float inv_range, uint32_t n_seg, uint32_t* __restrict__ seg_of,
                                  SegAcc* __restrict__ acc) {
  __shared__ float p[kParams];
  for (int i = threadIdx.x; i < kParams; i += blockDim.x) p[i] = params[i];
  __syncthreads();
  const size_t c0 = ((size_t)blockIdx.x * blockDim.x + threadIdx.x) * kChunk;
  if (c0 >= L) return;
  const size_t c1 = min(L, c0 + kChunk);
  uint32_t cur = kErrNone;
  unsigned long long lo = 0, hi = 0;
  unsigned int cnt = 0;
  for (size_t s = c0; s < c1; s++) {
    const uint64_t key = tab[s].low;
    const uint32_t j = seg_of_y(mlp_fwd(p, norm_x(key, kmin, inv_range)), n_seg);
    seg_of[s] = j;
    if (j != cur) {
      if (cnt) {
        atomicMin(&acc[cur].kmin, lo);
        atomicMax(&acc[cur].kmax, hi);
        atomicAdd(&acc[cur].count, cnt);
      }
      cur = j;
      lo = hi = key;
      cnt = 0;
    }
    lo = key < lo ? key : lo;
    hi = key > hi ? key : hi;
    cnt++;
  }
  if (cnt) {
    atomicMin(&acc[cur].kmin, lo);
    atomicMax(&acc[cur].kmax, hi);
    atomicAdd(&acc[cur].count, cnt);
  }
}

__global__ void seg_sums_kernel(const LeafEnt* __restrict__ tab, size_t L, const uint32_t* __restrict__ seg_of,
                                SegAcc* __restrict__ acc) {
  const size_t c0 = ((size_t)blockIdx.x * blockDim.x + threadIdx.x) * kChunk;
  if (c0 >= L) return;
  const size_t c1 = min(L, c0 + kChunk);
  uint32_t cur = kErrNone;
  double su = 0, suu = 0, sy = 0, suy = 0, inv = 1;
  uint64_t base = 0;
  for (size_t s = c0; s < c1; s++) {
    const uint32_t j = seg_of[s];
    if (j != cur) {
      if (cur != kErrNone) {
        atomicAdd(&acc[cur].su, su);
        atomicAdd(&acc[cur].suu, suu);
        atomicAdd(&acc[cur].sy, sy);
        atomicAdd(&acc[cur].suy, suy);
      }
      cur = j;
      su = suu = sy = suy = 0;
      base = acc[j].kmin;
      const uint64_t span = acc[j].kmax - acc[j].kmin;
      inv = span ? 1.0 / (double)span : 1.0;
    }
    const double u = (double)(tab[s].low - base) * inv;
    const double y = (double)s;
    su += u;
    suu += u * u;
    sy += y;
    suy += u * y;
  }
  if (cur != kErrNone) {
    atomicAdd(&acc[cur].su, su);
    atomicAdd(&acc[cur].suu, suu);
    atomicAdd(&acc[cur].sy, sy);
    atomicAdd(&acc[cur].suy, suy);
  }
}

// least-squares line per segment over u = (key - kmin) / span in [0, 1]
// (well conditioned in double), stored as a slope per key unit
__global__ void seg_solve_kernel(const SegAcc* __restrict__ acc, uint32_t n_seg, SegParam* __restrict__ sp,
                                 uint32_t* __restrict__ seg_err) {
  const uint32_t j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= n_seg) return;
  const SegAcc A = acc[j];
  SegParam P;
  P.base = A.count ? A.kmin : 0;
  const uint64_t span = A.count ? A.kmax - A.kmin : 1;
  const double inv_span = 1.0 / (double)(span ? span : 1);
  const double n = (double)A.count;
  double b = 0, a = 0;
  if (A.count >= 2) {
    const double den = n * A.suu - A.su * A.su;
    b = den > 1e-12 ? (n * A.suy - A.su * A.sy) / den : 0.0;
    a = (A.sy - b * A.su) / n;
  } else if (A.count == 1) {
    a = A.sy;
  }
  P.a = (float)a;
  P.slope = (float)(b * inv_span);
  sp[j] = P;
  seg_err[j] = A.count ? 0u : kErrNone;
}

__global__ void seg_err_kernel(const LeafEnt* __restrict__ tab, size_t L, const uint32_t* __restrict__ seg_of,
                               const SegParam* __restrict__ sp, uint32_t* __restrict__ seg_err) {
  const size_t c0 = ((size_t)blockIdx.x * blockDim.x + threadIdx.x) * kChunk;
  if (c0 >= L) return;
  const size_t c1 = min(L, c0 + kChunk);
  uint32_t cur = kErrNone, emax = 0;
  SegParam P{};
  for (size_t s = c0; s < c1; s++) {
    const uint32_t j = seg_of[s];
    if (j != cur) {
      if (cur != kErrNone) atomicMax(&seg_err[cur], emax);
      cur = j;
      emax = 0;
      P = sp[j];
    }
    const float p = seg_predict(P, tab[s].low);
    const float d = fabsf(floorf(p + 0.5f) - (float)s);
    const uint32_t e = d > 4.0e9f ? 0xFFFFFFF0u : (uint32_t)d;
    emax = e > emax ? e : emax;
  }
  if (cur != kErrNone) atomicMax(&seg_err[cur], emax);
}

// segments without training leaves or with a maximum error above the window
// get a = NaN (their keys go to the fallback without a probe) and are counted
__global__ void seg_finish_kernel(SegParam* __restrict__ sp, const uint32_t* __restrict__ seg_err, uint32_t n_seg,
                                  uint32_t window, unsigned int* __restrict__ bad) {
  const uint32_t j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j < n_seg && seg_err[j] > window) {
    sp[j].a = __int_as_float(0x7fc00000);
    atomicAdd(bad, 1u);
  }
}

// ----------------------------------------------------------------- lookup ----
// kSorted: keys arrive in ascending order (the batch's unique GETs); each
// group walks a contiguous chunk and reuses the previous leaf while the key
// stays below its fence.  Otherwise a grid-stride loop over any keys.
template <int G, bool kSorted>
__global__ void __launch_bounds__(256, 6) learned_search_kernel(DevTree t, LearnedDev M,
                                                                const uint64_t* __restrict__ qkeys,
                                                                const uint32_t* __restrict__ list,
                                                                const uint32_t* __restrict__ n_dev, size_t n_host,
                                                                uint64_t* __restrict__ out_vals,
                                                                uint8_t* __restrict__ out_st) {
  constexpr int S = 32 / G;
  __shared__ float p[kParams];
  for (int i = threadIdx.x; i < kParams; i += blockDim.x) p[i] = M.params[i];
  __syncthreads();
  const uint32_t lane = threadIdx.x & 31;
  const uint32_t g = lane % G;
  const uint32_t gmask = group_mask<G>(lane);
  const size_t n = n_dev ? (size_t)*n_dev : n_host;
  const uint32_t root = t.ctrl->root;
  const uint32_t root_level = t.ctrl->root_level;
  const size_t n_groups = ((size_t)gridDim.x * blockDim.x) / G;
  const size_t gid = ((size_t)blockIdx.x * blockDim.x + threadIdx.x) / G;
  size_t q, q_end, stride;
  if (kSorted) {
    const size_t chunk = (n + n_groups - 1) / n_groups;
    q = gid * chunk;
    q_end = min(n, q + chunk);
    stride = 1;
  } else {
    q = gid;
    q_end = n;
    stride = n_groups;
  }
  unsigned long long hits = 0, falls = 0, probe = 0;
  uint32_t leaf = kNil;
  uint64_t fence = 0;
  uint64_t k[S];
  const uint64_t stream = l2_stream();
  for (; q < q_end; q += stride) {
    const uint32_t r = list ? __ldg(list + q) : (uint32_t)q;
    const uint64_t key = __ldg(qkeys + r);
    uint8_t st = kAbsent;
    uint64_t ans = 0;
    if (key == kKeyMax) {
      st = kRejected;
    } else if (root != kNil) {
      bool have = kSorted && leaf != kNil && key < fence;  // same leaf as the previous key
      if (!have) {
        uint32_t dist = 0;
        const uint32_t node = learned_leaf<G>(M, p, key, g, gmask, dist);
        if (node != kNil) {
          // a leaf row is read once per lookup: let it leave L2 first
          load_slots_hint<S>(t.keys + (size_t)node * 32 + g * S, k, stream);
          fence = __shfl_sync(gmask, g == G - 1 ? ldg_hint(t.vals + (size_t)node * 32 + 31, stream) : 0, G - 1, G);
          if (g == G - 1) k[S - 1] = kKeyMax;
          leaf = node;
          have = key < fence;  // the leaf may have split since training
          if (have) {
            hits++;
            probe += dist;
          }
        }
      }
      if (have) {
        uint32_t c = 0;
#pragma unroll
        for (int i = 0; i < S; i++) c += (k[i] <= key) ? 1u : 0u;
        c = group_sum<G>(c, gmask);
        st = group_leaf_lookup_hint<G>(t, leaf, key, g, gmask, k, c, stream, ans);
      } else {
        falls++;
        leaf = kNil;
        st = group_descend<G, false>(t, root, root_level, key, g, gmask, ans);
      }
    }
    if (g == 0) {
      out_vals[r] = ans;
      out_st[r] = st;
    }
  }
  if (g == 0 && (hits | falls)) {
    atomicAdd(&t.ctrl->learned_hits, hits);
    atomicAdd(&t.ctrl->learned_fallbacks, falls);
    atomicAdd(&t.ctrl->learned_probe_sum, probe);
  }
}

// Unsorted learned lookup.  G lanes serve a request and R requests share a
// group in lock step (every step issues the loads of all R before using any),
// so a warp keeps 32 / G * R lookups in flight.  Per request the dependent
// chain is: stage 1 in registers -> the segment's 16 B line -> one probe of
// W = G * E leaf-table entries around the predicted slot -> the leaf's key row
// -> the value.  The leaf is right when the probe brackets the key between
// two training-time low fences (low fences never change) and either some key
// of the leaf is above the key or the key is below the leaf's live right
// fence (loaded only in that case: a leaf may have split since training).
// Everything else - no usable line, a key outside the probe, a split leaf -
// is appended to `miss` and answered by the plain descent afterwards, so no
// warp waits on another group's fallback.
// A miss joins the miss list with one atomic per group of lanes that miss
// together: with one atomic per miss, a tree whose leaves moved since
// training (a fifth of the lookups missing) serialised millions of atomics
// on the list's one counter.
__device__ __forceinline__ void append_miss(uint32_t* __restrict__ miss, uint64_t* __restrict__ miss_keys,
                                            uint32_t* __restrict__ n_miss, uint32_t r, uint64_t key) {
  const cooperative_groups::coalesced_group c = cooperative_groups::coalesced_threads();
  uint32_t base = 0;
  if (c.thread_rank() == 0) base = atomicAdd(n_miss, (uint32_t)c.size());
  base = c.shfl(base, 0);
  miss[base + c.thread_rank()] = r;
  miss_keys[base + c.thread_rank()] = key;
}

// A stale gate: the launch skips the model and lists every request as a miss
// (request index and key), so the plain descent answers them all.  Returns
// true when it did (the caller returns).
__device__ __forceinline__ bool gate_pass_all(const LearnedDev& M, const uint64_t* __restrict__ qkeys,
                                              const uint32_t* __restrict__ list, const uint64_t* __restrict__ ckeys,
                                              size_t n, uint32_t* __restrict__ miss, uint32_t* __restrict__ n_miss) {
  if (!M.gate || !M.gate->stale) return false;
  const size_t stride = (size_t)gridDim.x * blockDim.x;
  for (size_t q = (size_t)blockIdx.x * blockDim.x + threadIdx.x; q < n; q += stride) {
    const uint32_t r = list ? list[q] : (uint32_t)q;
    miss[q] = r;
    M.miss_keys[q] = ckeys ? ckeys[q] : qkeys[r];
  }
  if (blockIdx.x == 0 && threadIdx.x == 0) *n_miss = (uint32_t)n;
  return true;
}

__global__ void learned_judge_kernel(const Ctrl* __restrict__ ctrl, LearnedGate* __restrict__ g) {
  const unsigned long long hits = ctrl->learned_hits, falls = ctrl->learned_fallbacks;
  if (!g->have_base || hits < g->base_hits || falls < g->base_falls) {  // first look, or counters reset
    g->base_hits = hits;
    g->base_falls = falls;
    g->have_base = 1;
    return;
  }
  const unsigned long long dh = hits - g->base_hits, df = falls - g->base_falls;
  if (dh + df < kGateWindow) return;  // the window grows
  if (df * kGateMissDen > dh + df) g->stale = 1;
  g->base_hits = hits;
  g->base_falls = falls;
}

template <int G, int R>
__global__ void __launch_bounds__(256) learned_lookup_kernel(DevTree t, LearnedDev M,
                                                             const uint64_t* __restrict__ qkeys,
                                                             const uint32_t* __restrict__ list,
                                                             const uint32_t* __restrict__ n_dev, size_t n_host,
                                                             uint64_t* __restrict__ out_vals,
                                                             uint8_t* __restrict__ out_st,
                                                             uint32_t* __restrict__ miss,
                                                             uint32_t* __restrict__ n_miss,
                                                             const uint64_t* __restrict__ ckeys) {
  constexpr int S = 32 / G;              // key slots per lane
  constexpr int E = G >= 8 ? 1 : 8 / G;  // leaf-table entries per lane
  constexpr int W = G * E;               // probe width
  __shared__ float p[kParams];
  for (int i = threadIdx.x; i < kParams; i += blockDim.x) p[i] = M.params[i];
  __syncthreads();
  const uint32_t lane = threadIdx.x & 31;
  const uint32_t g = lane % G;
  const uint32_t gmask = group_mask<G>(lane);
  const size_t n = n_dev ? (size_t)*n_dev : n_host;
  if (gate_pass_all(M, qkeys, list, ckeys, n, miss, n_miss)) return;
  const size_t groups = ((size_t)gridDim.x * blockDim.x) / G;
  const int L = (int)M.n_leaves;
  const int p_hi = L + 1 - W > 0 ? L + 1 - W : 0;  // the table holds L + 1 entries (sentinel last)
  const uint64_t keep = l2_keep(), stream = l2_stream();
  unsigned long long hits = 0, falls = 0, probe = 0;
  for (size_t q0 = ((size_t)blockIdx.x * blockDim.x + threadIdx.x) / G; q0 < n; q0 += R * groups) {
    uint32_t r[R];
    uint64_t key[R];
    bool live[R], ok[R];
    float y[R];
#pragma unroll
    for (int j = 0; j < R; j++) {
      const size_t q = q0 + (size_t)j * groups;
      live[j] = q < n;
      r[j] = live[j] ? (list ? __ldg(list + q) : (uint32_t)q) : 0;
      key[j] = live[j] ? (ckeys ? __ldg(ckeys + q) : __ldg(qkeys + r[j])) : 0;
      ok[j] = live[j] && key[j] != kKeyMax;
      y[j] = mlp_group<G>(p, norm_x(key[j], M.kmin, M.inv_range), g, gmask);
    }
    // the segments' lines (4096 x 16 B: L1 / L2 resident)
    SegParam sp[R];
#pragma unroll
    for (int j = 0; j < R; j++) sp[j] = load_seg(M.seg, seg_of_y(y[j], M.n_seg));
    int p0[R], pc[R];
    ulonglong2 ent[R][E];
#pragma unroll
    for (int j = 0; j < R; j++) {
      const float pred = seg_predict(sp[j], key[j]);
      ok[j] = ok[j] && sp[j].a == sp[j].a;  // NaN: no usable line
      pc[j] = (pred > 0.f) ? (pred < (float)(L - 1) ? __float2int_rn(pred) : L - 1) : 0;
      int b = pc[j] - (W / 2 - 1);
      b = b > p_hi ? p_hi : b;
      p0[j] = b < 0 ? 0 : b;
#pragma unroll
      for (int e = 0; e < E; e++) {
        const int idx = p0[j] + e * G + (int)g;  // interleaved: each load covers W / E contiguous entries
        ent[j][e] = make_ulonglong2(kKeyMax, 0);
        // the leaf table is read by every lookup: keep it in L2
        if (ok[j] && idx <= L) ent[j][e] = ldg2_hint(reinterpret_cast<const ulonglong2*>(M.tab) + idx, keep);
      }
    }
    uint32_t node[R], pslot[R];
#pragma unroll
    for (int j = 0; j < R; j++) {
      uint32_t c = 0;
#pragma unroll
      for (int e = 0; e < E; e++) c += ent[j][e].x <= key[j] ? 1u : 0u;
      c = group_sum<G>(c, gmask);
      // bracketed: tab[slot].low <= key < tab[slot + 1].low inside the probe
      ok[j] = ok[j] && c >= 1 && c < (uint32_t)W;
      const uint32_t i = c >= 1 ? c - 1 : 0;
      uint64_t id = ent[j][0].y;
#pragma unroll
      for (int e = 1; e < E; e++)
        if (i / G == (uint32_t)e) id = ent[j][e].y;
      node[j] = (uint32_t)__shfl_sync(gmask, id, i % G, G);
      pslot[j] = (uint32_t)p0[j] + i;
    }
    // the leaves' key rows (read once per lookup: let them leave L2 first)
    uint64_t k[R][S];
#pragma unroll
    for (int j = 0; j < R; j++) {
      if (ok[j]) load_row_il<G>(t.keys + (size_t)node[j] * 32, g, k[j], stream);
      else {
#pragma unroll
        for (int i = 0; i < S; i++) k[j][i] = kKeyMax;
      }
    }
    uint32_t slot[R];
    bool found[R], need_fence[R];
#pragma unroll
    for (int j = 0; j < R; j++) {
      const uint64_t hdr = __shfl_sync(gmask, k[j][S - 1], G - 1, G);
      if (g == G - 1) k[j][S - 1] = kKeyMax;  // slot 31 holds the header
      uint32_t c = 0;
#pragma unroll
      for (int i = 0; i < S; i++) c += (k[j][i] <= key[j]) ? 1u : 0u;
      c = group_sum<G>(c, gmask);
      slot[j] = c > 0 ? c - 1 : 0;
      const uint64_t kk = __shfl_sync(gmask, pick<S>(k[j], il_elem<G>(slot[j])), il_lane<G>(slot[j]), G);
      ok[j] = ok[j] && hdr_level(hdr) == 0;
      found[j] = c > 0 && kk == key[j];
      // a key at or above the leaf's largest key: only the right fence tells
      // whether the leaf still covers it
      need_fence[j] = !found[j] && c >= hdr_size(hdr);
    }
    uint64_t v[R];
#pragma unroll
    for (int j = 0; j < R; j++) {
      v[j] = 0;
      if (g == 0 && ok[j] && (found[j] || need_fence[j]))
        v[j] = ldg_hint(t.vals + (size_t)node[j] * 32 + (found[j] ? slot[j] : 31), stream);
    }
#pragma unroll
    for (int j = 0; j < R; j++) {
      if (g != 0 || !live[j]) continue;
      if (key[j] == kKeyMax) {
        out_vals[r[j]] = 0;
        out_st[r[j]] = kRejected;
      } else if (ok[j] && (!need_fence[j] || key[j] < v[j])) {
        out_vals[r[j]] = found[j] ? v[j] : 0;
        out_st[r[j]] = found[j] ? kFound : kAbsent;
        hits++;
        probe += (uint32_t)(pc[j] > (int)pslot[j] ? pc[j] - (int)pslot[j] : (int)pslot[j] - pc[j]);
      } else {
        falls++;
        append_miss(miss, M.miss_keys, n_miss, r[j], key[j]);
      }
    }
  }
  // one atomic per warp for the counters
#pragma unroll
  for (int o = 16; o >= 1; o >>= 1) {
    hits += __shfl_xor_sync(0xffffffffu, hits, o);
    falls += __shfl_xor_sync(0xffffffffu, falls, o);
    probe += __shfl_xor_sync(0xffffffffu, probe, o);
  }
  if (lane == 0 && (hits | falls)) {
    atomicAdd(&t.ctrl->learned_hits, hits);
    atomicAdd(&t.ctrl->learned_fallbacks, falls);
    atomicAdd(&t.ctrl->learned_probe_sum, probe);
  }
}

// Software-pipelined learned lookup.  The dependent chain of one lookup has
// five memory rounds: list entry -> request key -> segment line and leaf-
// table probe -> leaf key row -> value (or right fence).  A group of G lanes
// carries up to five requests, one per round, and each loop iteration issues
// the loads of every round at once and consumes them in the next iteration,
// so a group finishes one lookup per memory latency instead of one per chain
// while holding the registers of about one request (the key row of one, the
// probe entries of one, ...).  Results and misses as learned_lookup_kernel.
// kCompact: the listed requests' keys come compacted (ckeys[q]), loaded in
// the same round as the list entry: four rounds instead of five.
// 256-thread blocks without a register cap: capping registers to fit more
// warps (64 per thread, or 72 at 128 threads) made the compiler hold fewer
// rounds of loads in flight, and the kernel got 1.5x slower
constexpr int kPipeThreads = 256;
template <int G, bool kCompact>
__global__ void __launch_bounds__(kPipeThreads) learned_pipe_kernel(DevTree t, LearnedDev M,
                                                           const uint64_t* __restrict__ qkeys,
                                                           const uint32_t* __restrict__ list,
                                                           const uint32_t* __restrict__ n_dev, size_t n_host,
                                                           uint64_t* __restrict__ out_vals,
                                                           uint8_t* __restrict__ out_st,
                                                           uint32_t* __restrict__ miss,
                                                           uint32_t* __restrict__ n_miss,
                                                           const uint64_t* __restrict__ ckeys) {
  constexpr int S = 32 / G;
  constexpr int E = G >= 8 ? 1 : 8 / G;
  constexpr int W = G * E;
  __shared__ float p[kParams];
  for (int i = threadIdx.x; i < kParams; i += blockDim.x) p[i] = M.params[i];
  __syncthreads();
  const uint32_t lane = threadIdx.x & 31;
  const uint32_t g = lane % G;
  const uint32_t gmask = group_mask<G>(lane);
  const size_t n = n_dev ? (size_t)*n_dev : n_host;
  if (gate_pass_all(M, qkeys, list, ckeys, n, miss, n_miss)) return;
  const size_t groups = ((size_t)gridDim.x * blockDim.x) / G;
  const int L = (int)M.n_leaves;
  const int p_hi = L + 1 - W > 0 ? L + 1 - W : 0;
  const uint64_t keep = l2_keep(), stream = l2_stream();
  uint32_t hits = 0, falls = 0, probe = 0;
  size_t q = ((size_t)blockIdx.x * blockDim.x + threadIdx.x) / G;
  // stage registers: B list entry loaded, C key loaded, D probe loaded,
  // E key row loaded, F value / fence loaded
  bool vB = false, vC = false, vD = false, vE = false, vF = false;
  uint32_t rB = 0, rC = 0, rD = 0, rE = 0, rF = 0;
  uint64_t kC = 0, kD = 0, kE = 0, kF = 0;
  bool okD = false, okE = false, okF = false;
  int p0D = 0, pcD = 0;
  uint32_t nodeE = 0, distE = 0, distF = 0;
  ulonglong2 entD[E];
  uint64_t rowE[S];
  uint64_t valF = 0;
  bool foundF = false, needF = false;
#pragma unroll
  for (int e = 0; e < E; e++) entD[e] = make_ulonglong2(kKeyMax, 0);
#pragma unroll
  for (int i = 0; i < S; i++) rowE[i] = kKeyMax;
  while (vB || vC || vD || vE || vF || q < n) {
    // F: answer, or hand the request to the plain descent
    if (vF && g == 0) {
      if (kF == kKeyMax) {
        out_vals[rF] = 0;
        out_st[rF] = kRejected;
      } else if (okF && (!needF || kF < valF)) {
        out_vals[rF] = foundF ? valF : 0;
        out_st[rF] = foundF ? kFound : kAbsent;
        hits++;
        probe += distF;
      } else {
        falls++;
        append_miss(miss, M.miss_keys, n_miss, rF, kF);
      }
    }
    // E -> F: rank the key in its leaf row; load the value or the right fence
    vF = vE;
    if (vE) {
      const uint64_t hdr = __shfl_sync(gmask, rowE[S - 1], G - 1, G);
      if (g == G - 1) rowE[S - 1] = kKeyMax;  // slot 31 holds the header
      // (shuffle sums: a redux.sync or a ballot per group mask, eight
      // distinct masks per warp, measured 1.5x slower here)
      uint32_t c = 0, eq = 0;
#pragma unroll
      for (int i = 0; i < S; i++) {
        c += (rowE[i] <= kE) ? 1u : 0u;
        eq |= (rowE[i] == kE) ? 1u : 0u;
      }
      c = group_sum<G>(c, gmask);
      const bool found = group_sum<G>(eq, gmask) != 0;
      okF = okE && hdr_level(hdr) == 0;
      foundF = found;
      needF = !foundF && c >= hdr_size(hdr);
      rF = rE;
      kF = kE;
      distF = distE;
      valF = 0;
      if (g == 0 && okF && (foundF || needF))
        valF = ldg_hint(t.vals + (size_t)nodeE * 32 + (foundF ? c - 1 : 31), stream);
    }
    // D -> E: the probe brackets the key; load the leaf's key row
    vE = vD;
    if (vD) {
      uint32_t c = 0;
#pragma unroll
      for (int e = 0; e < E; e++) c += entD[e].x <= kD ? 1u : 0u;
      c = group_sum<G>(c, gmask);
      okE = okD && c >= 1 && c < (uint32_t)W;
      const uint32_t i = c >= 1 ? c - 1 : 0;
      uint64_t id = entD[0].y;
#pragma unroll
      for (int e = 1; e < E; e++)
        if (i / G == (uint32_t)e) id = entD[e].y;
      nodeE = (uint32_t)__shfl_sync(gmask, id, i % G, G);
      const int slot = p0D + (int)i;
      distE = (uint32_t)(pcD > slot ? pcD - slot : slot - pcD);
      rE = rD;
      kE = kD;
      if (okE) load_row_il<G>(t.keys + (size_t)nodeE * 32, g, rowE, stream);
      else {
#pragma unroll
        for (int s = 0; s < S; s++) rowE[s] = kKeyMax;
      }
    }
    // C -> D: stage 1, the segment's line (L1), the leaf-table probe
    vD = vC;
    if (vC) {
      const float y = mlp_group<G>(p, norm_x(kC, M.kmin, M.inv_range), g, gmask);
      const SegParam sp = load_seg(M.seg, seg_of_y(y, M.n_seg));
      const float pred = seg_predict(sp, kC);
      okD = kC != kKeyMax && sp.a == sp.a;
      pcD = (pred > 0.f) ? (pred < (float)(L - 1) ? __float2int_rn(pred) : L - 1) : 0;
      int b = pcD - (W / 2 - 1);
      b = b > p_hi ? p_hi : b;
      p0D = b < 0 ? 0 : b;
      rD = rC;
      kD = kC;
#pragma unroll
      for (int e = 0; e < E; e++) {
        const int idx = p0D + e * G + (int)g;
        entD[e] = make_ulonglong2(kKeyMax, 0);
        if (okD && idx <= L) entD[e] = ldg2_hint(reinterpret_cast<const ulonglong2*>(M.tab) + idx, keep);
      }
    }
    if (kCompact) {
      // A -> C: the next request's list entry and key, side by side
      vC = q < n;
      if (vC) {
        rC = __ldg(list + q);
        kC = __ldg(ckeys + q);
        q += groups;
      }
    } else {
      // B -> C: the request's key
      vC = vB;
      if (vB) {
        rC = rB;
        kC = __ldg(qkeys + rB);
      }
      // A -> B: the next request's list entry
      vB = q < n;
      if (vB) {
        rB = list ? __ldg(list + q) : (uint32_t)q;
        q += groups;
      }
    }
  }
  hits = __reduce_add_sync(0xffffffffu, hits);
  falls = __reduce_add_sync(0xffffffffu, falls);
  probe = __reduce_add_sync(0xffffffffu, probe);
  if (lane == 0 && (hits | falls)) {
    atomicAdd(&t.ctrl->learned_hits, (unsigned long long)hits);
    atomicAdd(&t.ctrl->learned_fallbacks, (unsigned long long)falls);
    atomicAdd(&t.ctrl->learned_probe_sum, (unsigned long long)probe);
  }
}

inline unsigned nblk(size_t n, int per) { return (unsigned)((n + per - 1) / per); }

}  // namespace

// ------------------------------------------------------------------ host ----
void learned_free(Learned* L) {
  cudaFree(L->leaf_low);
  cudaFree(L->mlp);
  cudaFree(L->mlp_grad);
  cudaFree(L->seg);
  cudaFree(L->seg_scratch);
  cudaFree(L->seg_of);
  L->seg_of = nullptr;
  cudaFree(L->miss);
  cudaFree(L->miss_keys);
  cudaFree(L->gate);
  L->miss_keys = nullptr;
  L->gate = nullptr;
  if (L->host_words) cudaFreeHost(L->host_words);
  L->host_words = nullptr;
  L->miss = nullptr;
  L->n_miss = nullptr;
  L->miss_cap = 0;
  L->trained = false;
  L->leaf_low = nullptr;
  L->mlp = nullptr;
  L->mlp_grad = nullptr;
  L->seg = nullptr;
  L->seg_scratch = nullptr;
  L->leaf_cap = 0;
  L->seg_cap = 0;
  L->valid = false;
}

// ---- adaptive use in the batches (BT_OPT_LEARNED_POLICY) ----
// The model is trained on the leaves as they are; a batch's inserts split
// leaves, and a lookup whose predicted leaf has split since the fit falls
// back to the plain descent (one learned kernel's work wasted).  On a tree
// that the batches grow fast against its size (2^23 keys and 2^22-request
// 95/5 batches: 28 % fallbacks over 25 batches; any 50/50 mix) the learned
// form then loses to the plain one.  So the device judges the miss rate
// after every learned lookup launch (learned_judge_kernel) and, once it is
// stale, the learned kernels pass every request to the plain descent until
// the model is fitted again (LearnedGate): the decision is in stream order,
// however far the host has queued batches ahead.  Policy 2 also refits on
// its own: the host reads the gate through a page-locked word copied on a
// side stream after the lookups (read only once its copy has completed, so
// no batch waits for it) and refits kRefitAfter batches after the last fit.
constexpr uint32_t kRefitAfter = 8;

void learned_policy_free(Learned* L) {
  if (L->sample_stream) cudaStreamSynchronize(L->sample_stream);
  if (L->sample) cudaFreeHost(L->sample);
  if (L->sample_ev) cudaEventDestroy(L->sample_ev);
  if (L->lookups_ev) cudaEventDestroy(L->lookups_ev);
  if (L->sample_stream) cudaStreamDestroy(L->sample_stream);
  L->sample = nullptr;
  L->sample_ev = L->lookups_ev = nullptr;
  L->sample_stream = nullptr;
  L->pending = false;
}

static void learned_fitted(Learned& L) {
  L.stale = false;
  L.batches = 0;
}

bool batch_learned(Handle* h, int desc, cudaStream_t s) {
  Learned& L = h->L;
  if (desc != 1 || !L.valid) return false;
  if (L.policy != 2) return true;
  L.batches++;
  if (L.pending && cudaEventQuery(L.sample_ev) == cudaSuccess) {
    L.pending = false;
    if (L.sample[0] != 0) L.stale = true;  // the gate closed
  }
  cudaGetLastError();  // a copy not done yet (cudaErrorNotReady) is not an error
  if (L.stale && L.batches >= kRefitAfter) {
    // the refit reads the leaves: after the previous batch's deferred merge
    if (tree_join(h, s) != cudaSuccess || learned_retrain(h, s, true) != 0) return false;
  }
  return true;
}

void learned_sample(Handle* h, cudaStream_t s) {
  Learned& L = h->L;
  if (L.policy != 2 || L.pending || !L.gate) return;
  if (!L.sample) {
    if (cudaHostAlloc(&L.sample, 16, cudaHostAllocDefault) != cudaSuccess) {
      L.sample = nullptr;
      cudaGetLastError();
      return;
    }
    L.sample[0] = 0;
    if (cudaEventCreateWithFlags(&L.sample_ev, cudaEventDisableTiming) != cudaSuccess ||
        cudaEventCreateWithFlags(&L.lookups_ev, cudaEventDisableTiming) != cudaSuccess ||
        cudaStreamCreateWithFlags(&L.sample_stream, cudaStreamNonBlocking) != cudaSuccess) {
      learned_policy_free(&L);
      cudaGetLastError();
      return;
    }
  }
  // the gate word, on a side stream behind the lookups: the batch's own stream does not wait
  L.sample[0] = 0;
  if (cudaEventRecord(L.lookups_ev, s) != cudaSuccess || cudaStreamWaitEvent(L.sample_stream, L.lookups_ev, 0) != cudaSuccess ||
      cudaMemcpyAsync(L.sample, &L.gate->stale, 4, cudaMemcpyDeviceToHost, L.sample_stream) != cudaSuccess ||
      cudaEventRecord(L.sample_ev, L.sample_stream) != cudaSuccess) {
    cudaGetLastError();
    return;
  }
  L.pending = true;
}

// device scratch layout inside Learned:
//   leaf_low  -> LeafEnt tab[leaf_cap + 1] (reused as the leaf table)
//   mlp       -> params[97], m1[97], m2[97], step (int), loss, grad[97]
//   mlp_grad  -> partial gradients [kGradBlocks][kPartStride] then xs[M], ys[M]
//   seg       -> SegParam[n_seg] (as raw bytes)
//   seg_scratch -> SegAcc[n_seg], seg_err[n_seg], counter (256 B)
//   seg_of    -> [leaf_cap] segment of each leaf
//   miss      -> [miss_cap] requests the learned lookup left to the plain descent, then their count
static constexpr size_t kTrainMax = 65536;

// The model's own buffers (stage 1, segment lines) and the per-leaf arrays
// (leaf table, segment of each leaf) grow independently: a refit on a grown
// tree reallocates only the latter and keeps the trained stage 1.
static int learned_reserve(Learned* L, size_t n_leaves, uint32_t n_seg) {
  if (n_seg > L->seg_cap || !L->mlp) {
    learned_free(L);
    const size_t sc = n_seg;
    bool ok = cudaMalloc(&L->mlp, 512 * sizeof(float)) == cudaSuccess &&
              cudaMalloc(&L->mlp_grad, (kGradBlocks * kPartStride + 2 * kTrainMax) * sizeof(float)) == cudaSuccess &&
              cudaMalloc(&L->seg, sc * sizeof(SegParam)) == cudaSuccess &&
              cudaMalloc(&L->seg_scratch, sc * (sizeof(SegAcc) + 4) + 256) == cudaSuccess;
    if (!ok) {
      learned_free(L);
      return -3;
    }
    L->seg_cap = sc;
  }
  if (n_leaves + 1 > L->leaf_cap) {
    cudaFree(L->leaf_low);
    cudaFree(L->seg_of);
    L->leaf_low = nullptr;
    L->seg_of = nullptr;
    L->leaf_cap = 0;
    const size_t lc = n_leaves + n_leaves / 4 + 1024;
    if (cudaMalloc(&L->leaf_low, (lc + 1) * sizeof(LeafEnt)) != cudaSuccess ||
        cudaMalloc(&L->seg_of, lc * 4) != cudaSuccess) {
      learned_free(L);
      return -3;
    }
    L->leaf_cap = lc;
  }
  if (!L->host_words) {
    if (cudaHostAlloc(&L->host_words, 64, cudaHostAllocDefault) != cudaSuccess) {
      L->host_words = nullptr;
      return -3;
    }
    std::memset(L->host_words, 0, 64);
  }
  return 0;
}

static int miss_reserve(Learned* L, size_t cap) {
  if (!L->gate) {
    if (cudaMalloc(&L->gate, sizeof(LearnedGate)) != cudaSuccess) {
      L->gate = nullptr;
      return -3;
    }
    if (cudaMemset(L->gate, 0, sizeof(LearnedGate)) != cudaSuccess) return -3;
  }
  if (cap <= L->miss_cap) return 0;
  cudaFree(L->miss);
  cudaFree(L->miss_keys);
  L->miss = nullptr;
  L->miss_keys = nullptr;
  L->miss_cap = 0;
  if (cudaMalloc(&L->miss, (cap + 64) * 4) != cudaSuccess || cudaMalloc(&L->miss_keys, cap * 8) != cudaSuccess)
    return -3;
  L->n_miss = L->miss + cap;
  L->miss_cap = cap;
  return 0;
}

static void init_params(std::vector<float>& p, int stage1_mlp) {
  p.assign(kParams, 0.f);
  if (stage1_mlp) {
    // hinge basis with knots spread over [0, 1): y = x initially
    for (int j = 0; j < kHidden; j++) {
      p[j] = 1.f;
      p[kHidden + j] = -(float)j / (float)kHidden;
    }
    p[2 * kHidden + 0] = 1.f;
  } else {
    p[0] = 1.f;
    p[2 * kHidden] = 1.f;  // y = relu(x) = x: the linear root model
  }
}

// Full training (refit = false): leaf table, key range, stage 1 from its
// initial parameters for train_steps Adam steps, stage 2.  Refit (refit =
// true, after a full training): the leaf table and the segment lines follow
// the current leaves, stage 1 and its key normalisation are kept, with
// refit_steps warm-started Adam steps on the new table (default none).
int learned_retrain(Handle* h, cudaStream_t s, bool refit) {
  Learned& L = h->L;
  refit = refit && L.trained;
  L.valid = false;
  uint32_t* ids = nullptr;
  size_t nl = 0;
  int rc = enumerate_leaves(h, s, &ids, &nl);
  if (rc) return rc;
  if (nl < 2) return -7;
  // segments: as configured, else one per 64 leaves (a power of two, at
  // least 4096), fixed at the full training so that refits keep stage 1.
  // Measured on a 2^26-key tree grown by 16 M merged inserts (3.4 M leaves
  // of 16-31 keys, so leaf position drifts from linear in the key): 4096
  // segments miss the 8-entry probe for 22 % of the lookups, 16384 for
  // 2.9 %, 65536 for 0.8 % (0.4 % on the bulk-built tree either way)
  if (!refit) {
    uint32_t a = 4096;
    while (a < (nl + 63) / 64 && a < (1u << 20)) a <<= 1;
    L.n_segments = L.seg_config ? L.seg_config : a;
  }
  const uint32_t n_seg = L.n_segments;
  if (refit && n_seg > L.seg_cap) refit = false;
  if (!refit) L.trained = false;
  if (learned_reserve(&L, nl, n_seg)) return -3;
  if (miss_reserve(&L, h->w.cap > 65536 ? h->w.cap : 65536)) return -3;
  LeafEnt* tab = reinterpret_cast<LeafEnt*>(L.leaf_low);
  leaf_table_kernel<<<nblk(nl + 1, 256), 256, 0, s>>>(h->tree, ids, nl, tab);
  count_launch();
  if (!refit) {
    // key range over leaf lows 1 .. nl-1
    uint64_t kk[2];
    cudaMemcpyAsync(&kk[0], &tab[1].low, 8, cudaMemcpyDeviceToHost, s);
    cudaMemcpyAsync(&kk[1], &tab[nl - 1].low, 8, cudaMemcpyDeviceToHost, s);
    if (cudaStreamSynchronize(s) != cudaSuccess) return -2;
    L.kmin = kk[0];
    L.kmax = kk[1] > kk[0] ? kk[1] : kk[0] + 1;
  }
  const float inv_range = (float)(1.0 / (double)(L.kmax - L.kmin));
  L.n_leaves = (uint32_t)nl;
  // ---- stage 1
  float* params = L.mlp;
  float* m1 = params + 128;
  float* m2 = params + 256;
  int* step = reinterpret_cast<int*>(params + 384);
  float* loss = params + 385;
  float* partial = L.mlp_grad;
  float* xs = partial + kGradBlocks * kPartStride;
  float* ys = xs + kTrainMax;
  if (!refit) {
    std::vector<float> p0;
    init_params(p0, L.stage1);
    cudaMemcpyAsync(params, p0.data(), kParams * sizeof(float), cudaMemcpyHostToDevice, s);
  }
  cudaMemsetAsync(m1, 0, 2 * 128 * sizeof(float) + 2 * sizeof(float), s);
  const size_t M = (nl - 1) < kTrainMax ? (nl - 1) : kTrainMax;
  const uint32_t steps = refit ? L.refit_steps : L.train_steps;
  if (L.stage1 && steps > 0) {
    train_samples_kernel<<<nblk(M, 256), 256, 0, s>>>(tab, nl, M, L.kmin, inv_range, xs, ys);
    count_launch();
    // capture one training step and replay it
    cudaStream_t cs = h->internal_stream;
    cudaEvent_t ready;
    cudaEventCreateWithFlags(&ready, cudaEventDisableTiming);
    cudaEventRecord(ready, s);
    cudaStreamWaitEvent(cs, ready, 0);
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    bool ok = cudaStreamBeginCapture(cs, cudaStreamCaptureModeThreadLocal) == cudaSuccess;
    if (ok) {
      mlp_grad_kernel<<<kGradBlocks, kGradThreads, 0, cs>>>(params, xs, ys, M, partial);
      mlp_reduce_adam_kernel<<<1, 128, 0, cs>>>(params, partial, kGradBlocks, m1, m2, step, L.lr, nullptr, loss, 1);
      ok = cudaStreamEndCapture(cs, &graph) == cudaSuccess;
    }
    ok = ok && cudaGraphInstantiate(&exec, graph, 0) == cudaSuccess;
    for (uint32_t it = 0; ok && it < steps; it++) {
      ok = cudaGraphLaunch(exec, cs) == cudaSuccess;
      count_launch(2);
    }
    if (exec) cudaGraphExecDestroy(exec);
    if (graph) cudaGraphDestroy(graph);
    cudaEventRecord(ready, cs);
    cudaStreamWaitEvent(s, ready, 0);
    cudaEventDestroy(ready);
    if (!ok) return -2;
    cudaMemcpyAsync(L.host_words, loss, 4, cudaMemcpyDeviceToHost, s);
  }
  // ---- stage 2
  SegAcc* acc = reinterpret_cast<SegAcc*>(L.seg_scratch);
  uint32_t* seg_err = reinterpret_cast<uint32_t*>(acc + L.seg_cap);
  unsigned int* bad = seg_err + L.seg_cap;
  uint32_t* seg_of = L.seg_of;
  {
    seg_init_kernel<<<nblk(n_seg, 256), 256, 0, s>>>(acc, n_seg, bad);
    const size_t threads = (nl + kChunk - 1) / kChunk;
    seg_assign_kernel<<<nblk(threads, 256), 256, 0, s>>>(tab, nl, params, L.kmin, inv_range, n_seg, seg_of, acc);
    seg_sums_kernel<<<nblk(threads, 256), 256, 0, s>>>(tab, nl, seg_of, acc);
    seg_solve_kernel<<<nblk(n_seg, 256), 256, 0, s>>>(acc, n_seg, reinterpret_cast<SegParam*>(L.seg), seg_err);
    seg_err_kernel<<<nblk(threads, 256), 256, 0, s>>>(tab, nl, seg_of, reinterpret_cast<SegParam*>(L.seg), seg_err);
    seg_finish_kernel<<<nblk(n_seg, 256), 256, 0, s>>>(reinterpret_cast<SegParam*>(L.seg), seg_err, n_seg, L.window,
                                                       bad);
    count_launch(6);
    // diagnostics leave through page-locked host words, read by learned_info
    // after a synchronisation: a refit never waits for the device here
    cudaMemcpyAsync(L.host_words + 1, bad, 4, cudaMemcpyDeviceToHost, s);
  }
  if (cudaGetLastError() != cudaSuccess) return -2;
  if (!refit) {
    if (cudaStreamSynchronize(s) != cudaSuccess) return -2;
    L.trained = true;
  }
  L.refits += refit ? 1 : 0;
  L.valid = true;
  learned_fitted(L);
  // the gate opens again: the new fit is judged afresh
  if (cudaMemsetAsync(L.gate, 0, sizeof(LearnedGate), s) != cudaSuccess) return -2;
  return 0;
}

static LearnedDev dev_view(const Learned& L) {
  LearnedDev M;
  M.tab = reinterpret_cast<const LeafEnt*>(L.leaf_low);
  M.seg = reinterpret_cast<const SegParam*>(L.seg);
  M.params = L.mlp;
  M.kmin = L.kmin;
  M.inv_range = (float)(1.0 / (double)(L.kmax - L.kmin));
  M.n_leaves = L.n_leaves;
  M.n_seg = L.n_segments;
  M.window = L.window;
  M.gate = L.policy != 0 ? L.gate : nullptr;
  M.miss_keys = L.miss_keys;
  return M;
}

// R = 1 or 2: learned_lookup_kernel<G, R>; R = 0: learned_pipe_kernel<G, C>
template <int G, int R, bool C>
static cudaError_t lookup_launch(Handle* h, const LearnedDev& M, const uint64_t* qkeys, const uint32_t* list,
                                 const uint32_t* n_dev, size_t n, uint64_t* out_vals, uint8_t* out_st, cudaStream_t s,
                                 const uint64_t* ckeys) {
  const void* kfn =
      R == 0 ? (const void*)learned_pipe_kernel<G, C> : (const void*)learned_lookup_kernel<G, R ? R : 1>;
  const int threads = R == 0 ? kPipeThreads : 256;
  // a resident, grid-striding launch that leaves `lookup_reserve` block slots
  // free for kernels running beside it (the batch's overlapped locates)
  static int per_sm[64] = {};
  const int dev = h->device;
  int per = (dev >= 0 && dev < 64) ? per_sm[dev] : 0;
  if (per == 0) {
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, kfn, threads, 0) != cudaSuccess || per < 1)
      per = 1;
    if (dev >= 0 && dev < 64) per_sm[dev] = per;
  }
  const size_t resident = (size_t)h->sm_count * per;
  // lookup_reserve counts 256-thread block slots
  const size_t reserve = (size_t)h->lookup_reserve * 256 / threads;
  const size_t cap = resident > reserve + h->sm_count ? resident - reserve : (size_t)h->sm_count;
  // the pipelined form wants several requests per group to fill its rounds
  const size_t per_group = R == 0 ? 8 : R;
  size_t blocks = ((n + per_group - 1) / per_group * (size_t)G + threads - 1) / threads;
  if (blocks > cap) blocks = cap;
  if (blocks == 0) blocks = 1;
  if (R == 0)
    learned_pipe_kernel<G, C><<<(unsigned)blocks, threads, 0, s>>>(h->tree, M, qkeys, list, n_dev, n, out_vals, out_st,
                                                               h->L.miss, h->L.n_miss, ckeys);
  else
    learned_lookup_kernel<G, R ? R : 1><<<(unsigned)blocks, 256, 0, s>>>(h->tree, M, qkeys, list, n_dev, n, out_vals,
                                                                          out_st, h->L.miss, h->L.n_miss, ckeys);
  count_launch();
  return cudaGetLastError();
}

// gated: the batch paths' lookups, which the adaptive gate may hand to the
// plain descent (bt_search_batch keeps bt_set_descent's choice)
cudaError_t launch_learned_lookup(Handle* h, const uint64_t* qkeys, const uint32_t* list, const uint32_t* n_dev,
                                  size_t n, uint64_t* out_vals, uint8_t* out_st, cudaStream_t s,
                                  const uint64_t* ckeys, bool gated) {
  if (!list) ckeys = nullptr;
  if (n == 0) return cudaSuccess;
  Learned& L = h->L;
  if (n > L.miss_cap) {
    // the batch path never gets here (n <= max_batch <= miss_cap); a larger
    // bt_search_batch runs in pieces
    if (list || n_dev) return cudaErrorInvalidValue;
    for (size_t off = 0; off < n; off += L.miss_cap) {
      const size_t m = n - off < L.miss_cap ? n - off : L.miss_cap;
      const cudaError_t e = launch_learned_lookup(h, qkeys + off, nullptr, nullptr, m, out_vals + off, out_st + off, s);
      if (e != cudaSuccess) return e;
    }
    return cudaSuccess;
  }
  LearnedDev M = dev_view(L);
  if (!gated) M.gate = nullptr;
  if (cudaMemsetAsync(L.n_miss, 0, 4, s) != cudaSuccess) return cudaGetLastError();
  cudaError_t e;
  const int G = h->learned_group, R = h->learned_mode;
#define BT_LL(GG, RR)                                                                         \
  (ckeys ? lookup_launch<GG, RR, true>(h, M, qkeys, list, n_dev, n, out_vals, out_st, s, ckeys) \
         : lookup_launch<GG, RR, false>(h, M, qkeys, list, n_dev, n, out_vals, out_st, s, nullptr))
  if (G == 8) e = R == 3 ? BT_LL(8, 0) : R == 2 ? BT_LL(8, 2) : BT_LL(8, 1);
  else if (G == 2) e = R == 3 ? BT_LL(2, 0) : BT_LL(2, 1);
  else if (G == 16) e = R == 3 ? BT_LL(16, 0) : BT_LL(16, 1);
  else if (G == 32) e = BT_LL(32, 1);
  else e = R == 3 ? BT_LL(4, 0) : R == 2 ? BT_LL(4, 2) : BT_LL(4, 1);
#undef BT_LL
  if (e != cudaSuccess) return e;
  // the misses: plain descent over the miss list (keys compacted beside it),
  // one resident wave
  const int saved = h->lookup_reserve;
  h->lookup_reserve = saved > 1 ? saved : 1;
  e = launch_search(h, qkeys, L.miss, L.n_miss, n, out_vals, out_st, s, L.miss_keys);
  h->lookup_reserve = saved;
  if (e != cudaSuccess || !M.gate) return e;
  learned_judge_kernel<<<1, 1, 0, s>>>(h->tree.ctrl, L.gate);
  count_launch();
  return cudaGetLastError();
}

cudaError_t launch_learned_search(Handle* h, const uint64_t* qkeys, const uint32_t* list, const uint32_t* n_dev,
                                  size_t n, uint64_t* out_vals, uint8_t* out_st, cudaStream_t s, bool sorted) {
  if (n == 0) return cudaSuccess;
  const LearnedDev M = dev_view(h->L);
  const int threads = 256;
  const int G = h->learned_group;
  size_t blocks;
  if (sorted) {
    blocks = (size_t)h->sm_count * 6;  // one resident wave (6 blocks per SM at 256 threads)
  } else {
    blocks = (n * (size_t)G + threads - 1) / threads;
    const size_t cap = (size_t)h->sm_count * 8 * 4;
    if (blocks > cap) blocks = cap;
  }
#define BT_LSK(GG, SS) learned_search_kernel<GG, SS><<<(unsigned)blocks, threads, 0, s>>>(h->tree, M, qkeys, list, n_dev, n, out_vals, out_st)
  if (sorted) {
    if (G == 16) BT_LSK(16, true);
    else if (G == 32) BT_LSK(32, true);
    else BT_LSK(8, true);
  } else {
    if (G == 16) BT_LSK(16, false);
    else if (G == 32) BT_LSK(32, false);
    else BT_LSK(8, false);
  }
#undef BT_LSK
  count_launch();
  return cudaGetLastError();
}

int learned_dev(Handle* h, LearnedDev* M) {
  Learned& L = h->L;
  if (!(h->descent == 1 && L.valid)) return 0;
  *M = dev_view(L);
  return 1;
}

// gradient of the MSE of the MLP over (x, y) on the device (diagnostics / tests)
int learned_mlp_grad(Handle* h, const float* params, const float* x, const float* y, size_t n, float* grad_out,
                     float* loss_out, cudaStream_t s) {
  if (learned_reserve(&h->L, 1, h->L.n_segments ? h->L.n_segments : 1)) return -3;
  float* partial = h->L.mlp_grad;
  mlp_grad_kernel<<<kGradBlocks, kGradThreads, 0, s>>>(params, x, y, n, partial);
  mlp_reduce_adam_kernel<<<1, 128, 0, s>>>(const_cast<float*>(params), partial, kGradBlocks, nullptr, nullptr,
                                          reinterpret_cast<int*>(h->L.mlp + 384), 0.f, grad_out, loss_out, 0);
  count_launch(2);
  return cudaGetLastError() == cudaSuccess ? 0 : -2;
}

}  // namespace bt
