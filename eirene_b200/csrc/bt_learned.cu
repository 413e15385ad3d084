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
                                     double inv_range, float* __restrict__ xs, float* __restrict__ ys) {
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

__global__ void seg_assign_kernel(const LeafEnt* __restrict__ tab, size_t L, const float* __restrict__ params,
                                  uint64_t kmin, double inv_range, uint32_t n_seg, uint32_t* __restrict__ seg_of,
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

__global__ void seg_solve_kernel(const SegAcc* __restrict__ acc, uint32_t n_seg, SegParam* __restrict__ sp) {
  const uint32_t j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= n_seg) return;
  const SegAcc A = acc[j];
  SegParam P;
  P.base = A.count ? A.kmin : 0;
  const uint64_t span = A.count ? A.kmax - A.kmin : 1;
  P.inv_span = (float)(1.0 / (double)(span ? span : 1));
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
  P.b = (float)b;
  P.err = A.count ? 0u : kErrNone;
  sp[j] = P;
}

__global__ void seg_err_kernel(const LeafEnt* __restrict__ tab, size_t L, const uint32_t* __restrict__ seg_of,
                               SegParam* __restrict__ sp) {
  const size_t c0 = ((size_t)blockIdx.x * blockDim.x + threadIdx.x) * kChunk;
  if (c0 >= L) return;
  const size_t c1 = min(L, c0 + kChunk);
  uint32_t cur = kErrNone, emax = 0;
  SegParam P{};
  for (size_t s = c0; s < c1; s++) {
    const uint32_t j = seg_of[s];
    if (j != cur) {
      if (cur != kErrNone) atomicMax(&sp[cur].err, emax);
      cur = j;
      emax = 0;
      P = sp[j];
    }
    const float p = seg_predict(P, tab[s].low);
    const float d = fabsf(floorf(p + 0.5f) - (float)s);
    const uint32_t e = d > 4.0e9f ? 0xFFFFFFF0u : (uint32_t)d;
    emax = e > emax ? e : emax;
  }
  if (cur != kErrNone) atomicMax(&sp[cur].err, emax);
}

__global__ void seg_count_bad_kernel(const SegParam* __restrict__ sp, uint32_t n_seg, uint32_t window,
                                     unsigned int* __restrict__ bad) {
  const uint32_t j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j < n_seg && sp[j].err > window) atomicAdd(bad, 1u);
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

inline unsigned nblk(size_t n, int per) { return (unsigned)((n + per - 1) / per); }

}  // namespace

// ------------------------------------------------------------------ host ----
void learned_free(Learned* L) {
  cudaFree(L->leaf_low);
  cudaFree(L->mlp);
  cudaFree(L->mlp_grad);
  cudaFree(L->seg);
  cudaFree(L->seg_scratch);
  L->leaf_low = nullptr;
  L->mlp = nullptr;
  L->mlp_grad = nullptr;
  L->seg = nullptr;
  L->seg_scratch = nullptr;
  L->leaf_cap = 0;
  L->seg_cap = 0;
  L->valid = false;
}

// device scratch layout inside Learned:
//   leaf_low  -> LeafEnt tab[leaf_cap + 1] (reused as the leaf table)
//   mlp       -> params[97], m1[97], m2[97], step (int), loss, grad[97]
//   mlp_grad  -> partial gradients [kGradBlocks][kPartStride] then xs[M], ys[M]
//   seg       -> SegParam[n_seg] (as raw bytes)
//   seg_scratch -> SegAcc[n_seg], seg_of[leaf_cap], counter
static constexpr size_t kTrainMax = 65536;

static int learned_reserve(Learned* L, size_t n_leaves, uint32_t n_seg) {
  if (n_leaves + 1 > L->leaf_cap || n_seg > L->seg_cap) {
    learned_free(L);
    const size_t lc = n_leaves + n_leaves / 4 + 1024;
    const size_t sc = n_seg;
    bool ok = cudaMalloc(&L->leaf_low, (lc + 1) * sizeof(LeafEnt)) == cudaSuccess &&
              cudaMalloc(&L->mlp, 512 * sizeof(float)) == cudaSuccess &&
              cudaMalloc(&L->mlp_grad, (kGradBlocks * kPartStride + 2 * kTrainMax) * sizeof(float)) == cudaSuccess &&
              cudaMalloc(&L->seg, sc * sizeof(SegParam)) == cudaSuccess &&
              cudaMalloc(&L->seg_scratch, sc * sizeof(SegAcc) + lc * 4 + 256) == cudaSuccess;
    if (!ok) {
      learned_free(L);
      return -3;
    }
    L->leaf_cap = lc;
    L->seg_cap = sc;
  }
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

int learned_retrain(Handle* h, cudaStream_t s) {
  Learned& L = h->L;
  L.valid = false;
  uint32_t* ids = nullptr;
  size_t nl = 0;
  int rc = enumerate_leaves(h, s, &ids, &nl);
  if (rc) return rc;
  if (nl < 2) return -7;
  const uint32_t n_seg = L.n_segments;
  if (learned_reserve(&L, nl, n_seg)) return -3;
  LeafEnt* tab = reinterpret_cast<LeafEnt*>(L.leaf_low);
  leaf_table_kernel<<<nblk(nl + 1, 256), 256, 0, s>>>(h->tree, ids, nl, tab);
  count_launch();
  // key range over leaf lows 1 .. nl-1
  uint64_t kk[2];
  cudaMemcpyAsync(&kk[0], &tab[1].low, 8, cudaMemcpyDeviceToHost, s);
  cudaMemcpyAsync(&kk[1], &tab[nl - 1].low, 8, cudaMemcpyDeviceToHost, s);
  if (cudaStreamSynchronize(s) != cudaSuccess) return -2;
  L.kmin = kk[0];
  L.kmax = kk[1] > kk[0] ? kk[1] : kk[0] + 1;
  const double inv_range = 1.0 / (double)(L.kmax - L.kmin);
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
  std::vector<float> p0;
  init_params(p0, L.stage1);
  cudaMemcpyAsync(params, p0.data(), kParams * sizeof(float), cudaMemcpyHostToDevice, s);
  cudaMemsetAsync(m1, 0, 2 * 128 * sizeof(float) + 2 * sizeof(float), s);
  const size_t M = (nl - 1) < kTrainMax ? (nl - 1) : kTrainMax;
  train_samples_kernel<<<nblk(M, 256), 256, 0, s>>>(tab, nl, M, L.kmin, inv_range, xs, ys);
  count_launch();
  if (L.stage1 && L.train_steps > 0) {
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
    for (uint32_t it = 0; ok && it < L.train_steps; it++) {
      ok = cudaGraphLaunch(exec, cs) == cudaSuccess;
      count_launch(2);
    }
    if (exec) cudaGraphExecDestroy(exec);
    if (graph) cudaGraphDestroy(graph);
    cudaEventRecord(ready, cs);
    cudaStreamWaitEvent(s, ready, 0);
    cudaEventDestroy(ready);
    if (!ok) return -2;
    float lv = 0;
    cudaMemcpyAsync(&lv, loss, 4, cudaMemcpyDeviceToHost, s);
    if (cudaStreamSynchronize(s) != cudaSuccess) return -2;
    L.last_loss = lv;
  }
  // ---- stage 2
  SegAcc* acc = reinterpret_cast<SegAcc*>(L.seg_scratch);
  uint32_t* seg_of = reinterpret_cast<uint32_t*>(reinterpret_cast<char*>(L.seg_scratch) + n_seg * sizeof(SegAcc));
  unsigned int* bad = seg_of + L.leaf_cap;
  {
    std::vector<SegAcc> init(n_seg);
    for (auto& a : init) {
      std::memset(&a, 0, sizeof(a));
      a.kmin = ~0ull;
    }
    cudaMemcpyAsync(acc, init.data(), n_seg * sizeof(SegAcc), cudaMemcpyHostToDevice, s);
    cudaMemsetAsync(bad, 0, 4, s);
    const size_t threads = (nl + kChunk - 1) / kChunk;
    seg_assign_kernel<<<nblk(threads, 256), 256, 0, s>>>(tab, nl, params, L.kmin, inv_range, n_seg, seg_of, acc);
    seg_sums_kernel<<<nblk(threads, 256), 256, 0, s>>>(tab, nl, seg_of, acc);
    seg_solve_kernel<<<nblk(n_seg, 256), 256, 0, s>>>(acc, n_seg, reinterpret_cast<SegParam*>(L.seg));
    seg_err_kernel<<<nblk(threads, 256), 256, 0, s>>>(tab, nl, seg_of, reinterpret_cast<SegParam*>(L.seg));
    seg_count_bad_kernel<<<nblk(n_seg, 256), 256, 0, s>>>(reinterpret_cast<SegParam*>(L.seg), n_seg, L.window, bad);
    count_launch(5);
    unsigned int nb = 0;
    cudaMemcpyAsync(&nb, bad, 4, cudaMemcpyDeviceToHost, s);
    if (cudaStreamSynchronize(s) != cudaSuccess) return -2;
    L.seg_fallback = nb;
  }
  if (cudaGetLastError() != cudaSuccess) return -2;
  L.valid = true;
  return 0;
}

cudaError_t launch_learned_search(Handle* h, const uint64_t* qkeys, const uint32_t* list, const uint32_t* n_dev,
                                  size_t n, uint64_t* out_vals, uint8_t* out_st, cudaStream_t s, bool sorted) {
  if (n == 0) return cudaSuccess;
  Learned& L = h->L;
  LearnedDev M;
  M.tab = reinterpret_cast<const LeafEnt*>(L.leaf_low);
  M.seg = reinterpret_cast<const SegParam*>(L.seg);
  M.params = L.mlp;
  M.kmin = L.kmin;
  M.inv_range = 1.0 / (double)(L.kmax - L.kmin);
  M.n_leaves = L.n_leaves;
  M.n_seg = L.n_segments;
  M.window = L.window;
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
  M->tab = reinterpret_cast<const LeafEnt*>(L.leaf_low);
  M->seg = reinterpret_cast<const SegParam*>(L.seg);
  M->params = L.mlp;
  M->kmin = L.kmin;
  M->inv_range = 1.0 / (double)(L.kmax - L.kmin);
  M->n_leaves = L.n_leaves;
  M->n_seg = L.n_segments;
  M->window = L.window;
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
