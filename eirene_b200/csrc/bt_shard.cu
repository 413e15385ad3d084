// Routing for a key-range-sharded tree: one tree per GPU, shard s owning the
// keys in [splitter[s-1], splitter[s]).  A batch is partitioned by owner
// (stable: requests keep their input order inside each shard's run), the
// runs are exchanged between GPUs by the caller's all-to-all, each GPU runs
// its runs as one batch, and the answers come back by the reverse exchange
// and are scattered to input order here.  The reference is single-GPU only
// (one GPU_STM_Tree, src/gpu-stm-tree-v39/bpt-gpustm.cpp:14-28); routing
// has no counterpart there.
//
// bt_route_batch: shard ids (upper bound over the splitters, which sit in
// shared memory) -> one stable 8-bit radix pass over the ids with the
// request index as payload -> gather into owner order + per-shard counts.
// HBM traffic per request: 8 B key read + 8 B id write, the radix pass
// (8 + 8 B read, 8 + 4 B write), the gather (4 B perm + 8 + 8 + 1 B
// reads, 8 + 8 + 1 + 4 B writes).
#include <cuda_runtime.h>

#include "../../include/eirene_b200.h"
#include "bt_common.cuh"
#include "bt_internal.h"

namespace {

constexpr int kThreads = 256;

__global__ void __launch_bounds__(kThreads) shard_id_kernel(const uint64_t* __restrict__ keys, size_t n,
                                                            const uint64_t* __restrict__ splitters,
                                                            int n_split, uint64_t* __restrict__ ids) {
  __shared__ uint64_t spl[BT_MAX_SHARDS];
  for (int i = threadIdx.x; i < n_split; i += blockDim.x) spl[i] = splitters[i];
  __syncthreads();
  for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
    const uint64_t k = keys[i];
    int lo = 0, hi = n_split;  // first splitter greater than k
    while (lo < hi) {
      const int mid = (lo + hi) >> 1;
      if (spl[mid] <= k) lo = mid + 1;
      else hi = mid;
    }
    ids[i] = (uint64_t)lo;
  }
}

__global__ void __launch_bounds__(kThreads) route_gather_kernel(
    const uint32_t* __restrict__ perm, size_t n, const uint64_t* __restrict__ keys,
    const uint64_t* __restrict__ vals, const uint8_t* __restrict__ ops, uint64_t* __restrict__ out_keys,
    uint64_t* __restrict__ out_vals, uint8_t* __restrict__ out_ops, uint32_t* __restrict__ out_perm) {
  for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
    const uint32_t j = perm[i];
    out_keys[i] = keys[j];
    if (vals) out_vals[i] = vals[j];
    if (ops) out_ops[i] = ops[j];
    out_perm[i] = j;
  }
}

// counts[s] = lower_bound(s + 1) - lower_bound(s) over the sorted ids
__global__ void shard_count_kernel(const uint64_t* __restrict__ sorted_ids, size_t n, int n_shards,
                                   uint64_t* __restrict__ counts) {
  const int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= n_shards) return;
  auto lower = [&](uint64_t v) {
    size_t lo = 0, hi = n;
    while (lo < hi) {
      const size_t mid = (lo + hi) >> 1;
      if (sorted_ids[mid] < v) lo = mid + 1;
      else hi = mid;
    }
    return lo;
  };
  counts[s] = (uint64_t)(lower((uint64_t)s + 1) - lower((uint64_t)s));
}

__global__ void __launch_bounds__(kThreads) unroute_kernel(const uint32_t* __restrict__ perm, size_t n,
                                                           const uint64_t* __restrict__ in_vals,
                                                           const uint8_t* __restrict__ in_st,
                                                           uint64_t* __restrict__ out_vals,
                                                           uint8_t* __restrict__ out_st) {
  for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
    const uint32_t j = perm[i];
    out_vals[j] = in_vals[i];
    out_st[j] = in_st[i];
  }
}

unsigned grid_for(size_t n, int sm_count) {
  const size_t want = (n + kThreads - 1) / kThreads;
  const size_t cap = (size_t)sm_count * 8;
  return (unsigned)(want < cap ? (want ? want : 1) : cap);
}

}  // namespace

namespace bt {

int route_batch(Handle* h, const uint64_t* splitters, int n_shards, const uint64_t* keys, const uint64_t* vals,
                const uint8_t* ops, size_t n, uint64_t* out_keys, uint64_t* out_vals, uint8_t* out_ops,
                uint32_t* out_perm, uint64_t* out_counts, cudaStream_t s) {
  Work& w = h->w;
  const int n_split = n_shards - 1;
  if (n == 0) return cudaMemsetAsync(out_counts, 0, (size_t)n_shards * 8, s) == cudaSuccess ? BT_OK : BT_ERR_CUDA;
  // batches up to the handle's capacity use its work buffers; larger inputs
  // (a bulk build's keys) take stream-ordered temporaries for this call
  uint64_t *ids = w.ukeys, *ka = w.k_a, *kb = w.k_b;
  uint32_t *va = w.v_a, *vb = w.v_b, *scratch = w.sort_scratch;
  const bool tmp = n > w.cap;
  if (tmp) {
    void* p[6] = {};
    const size_t sz[6] = {n * 8, n * 8, n * 8, n * 4, n * 4, sort_scratch_words(n) * 4};
    for (int i = 0; i < 6; i++) {
      if (cudaMallocAsync(&p[i], sz[i], s) != cudaSuccess) {
        for (int j = 0; j < i; j++) cudaFreeAsync(p[j], s);
        return BT_ERR_NO_MEMORY;
      }
    }
    ids = (uint64_t*)p[0];
    ka = (uint64_t*)p[1];
    kb = (uint64_t*)p[2];
    va = (uint32_t*)p[3];
    vb = (uint32_t*)p[4];
    scratch = (uint32_t*)p[5];
  }
  int rc = BT_OK;
  const unsigned g = grid_for(n, h->sm_count);
  shard_id_kernel<<<g, kThreads, 0, s>>>(keys, n, splitters, n_split, ids);
  count_launch();
  uint64_t* sk = nullptr;
  uint32_t* perm = nullptr;
  // one stable pass over the low 8 bits (n_shards <= 256) with the index as payload
  if (cudaGetLastError() != cudaSuccess ||
      radix_sort_pairs(ids, nullptr, nullptr, ka, va, kb, vb, n, 0, 8, scratch, s, &sk, &perm,
                       &h->tree.ctrl->error) != cudaSuccess) {
    rc = BT_ERR_CUDA;
  } else {
    route_gather_kernel<<<g, kThreads, 0, s>>>(perm, n, keys, vals, ops, out_keys, out_vals, out_ops, out_perm);
    count_launch();
    shard_count_kernel<<<(n_shards + 255) / 256, 256, 0, s>>>(sk, n, n_shards, out_counts);
    count_launch();
    if (cudaGetLastError() != cudaSuccess) rc = BT_ERR_CUDA;
  }
  if (tmp) {
    cudaFreeAsync(ids, s);
    cudaFreeAsync(ka, s);
    cudaFreeAsync(kb, s);
    cudaFreeAsync(va, s);
    cudaFreeAsync(vb, s);
    cudaFreeAsync(scratch, s);
  }
  return rc;
}

int unroute_results(Handle* h, const uint32_t* perm, const uint64_t* in_vals, const uint8_t* in_st, size_t n,
                    uint64_t* out_vals, uint8_t* out_st, cudaStream_t s) {
  if (n == 0) return BT_OK;
  unroute_kernel<<<grid_for(n, h->sm_count), kThreads, 0, s>>>(perm, n, in_vals, in_st, out_vals, out_st);
  count_launch();
  return cudaGetLastError() == cudaSuccess ? BT_OK : BT_ERR_CUDA;
}

}  // namespace bt
