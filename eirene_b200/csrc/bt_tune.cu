// Autotuner: times the candidate lookup configurations on the live tree with
// a caller-supplied sample of keys and keeps the fastest.  Tuned: lanes per
// request of the unsorted plain and learned searches, the sorted search's
// leaf-value load, and which descent serves the batch GET phase.  Lookups
// only: the tree is not modified.  Node fanout (32, fixed by the node layout)
// and the sort tile (4096) are compile-time constants.
#include <cuda_runtime.h>

#include "bt_common.cuh"
#include "bt_internal.h"

namespace bt {

template <typename F>
static float time_ms(cudaStream_t s, F&& f, int reps = 3) {
  cudaEvent_t a, b;
  cudaEventCreate(&a);
  cudaEventCreate(&b);
  f();  // warm-up
  cudaEventRecord(a, s);
  for (int i = 0; i < reps; i++) f();
  cudaEventRecord(b, s);
  cudaEventSynchronize(b);
  float ms = 0;
  cudaEventElapsedTime(&ms, a, b);
  cudaEventDestroy(a);
  cudaEventDestroy(b);
  return ms / reps;
}

int autotune(Handle* h, const uint64_t* keys, size_t n, cudaStream_t s, double* rep) {
  Work& w = h->w;
  if (n == 0 || n > w.cap) return -6;
  double out[16] = {};
  // unsorted plain search
  const int gs[4] = {4, 8, 16, 32};
  float best = 1e30f;
  int best_g = h->search_group;
  for (int i = 0; i < 4; i++) {
    h->search_group = gs[i];
    const float ms = time_ms(s, [&] { launch_search(h, keys, nullptr, nullptr, n, w.uans, w.uans_st, s); });
    out[4 + i] = ms;
    if (ms < best) {
      best = ms;
      best_g = gs[i];
    }
  }
  h->search_group = best_g;
  out[0] = best_g;
  // unsorted learned search
  if (h->L.valid) {
    const int lg[3] = {8, 16, 32};
    float bl = 1e30f;
    int best_l = h->learned_group;
    for (int i = 0; i < 3; i++) {
      h->learned_group = lg[i];
      const float ms =
          time_ms(s, [&] { launch_learned_search(h, keys, nullptr, nullptr, n, w.uans, w.uans_st, s, false); });
      out[8 + i] = ms;
      if (ms < bl) {
        bl = ms;
        best_l = lg[i];
      }
    }
    h->learned_group = best_l;
    out[1] = best_l;
  }
  // sorted sample for the batch GET phase
  uint64_t* sk = nullptr;
  uint32_t* sv = nullptr;
  if (radix_sort_pairs(keys, nullptr, nullptr, w.k_a, w.v_a, w.k_b, w.v_b, n, 0, 64, w.sort_scratch, s, &sk, &sv,
                       &h->tree.ctrl->error) != cudaSuccess)
    return -2;
  float bs = 1e30f;
  int best_lv = 0;
  for (int lv = 0; lv < 2; lv++) {
    h->sorted_leaf_vals = lv;
    const float ms = time_ms(s, [&] { launch_search_sorted(h, sk, nullptr, nullptr, n, w.uans, w.uans_st, s); });
    out[12 + lv] = ms;
    if (ms < bs) {
      bs = ms;
      best_lv = lv;
    }
  }
  h->sorted_leaf_vals = best_lv;
  out[2] = best_lv;
  int desc = 0;
  if (h->L.valid) {
    const float ms =
        time_ms(s, [&] { launch_learned_search(h, sk, nullptr, nullptr, n, w.uans, w.uans_st, s, true); });
    out[14] = ms;
    if (ms < bs) desc = 1;
  }
  h->batch_descent = desc;
  out[3] = desc;
  if (cudaStreamSynchronize(s) != cudaSuccess) return -2;
  if (rep)
    for (int i = 0; i < 16; i++) rep[i] = out[i];
  return 0;
}

}  // namespace bt
