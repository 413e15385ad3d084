// Autotuner: times the candidate configurations on the live tree with a
// caller-supplied sample of keys and keeps the fastest.  Tuned: lanes per
// request of the unsorted plain search, lanes per request and the form of
// the unsorted learned lookup, the sorted search's leaf-value load, which
// descent serves the batch GET phase, and the radix sort's tile for whole
// batches and for the hash front end's touched requests.  Lookups and sorts
// only: the tree is not modified.  The node fill (fanout) is tuned on a
// sample tree by bt_autotune_fill (bt_api.cu).
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
  double out[kTuneReport] = {};
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
  // unsorted learned lookup: lanes per request x requests per group
  float best_learned = 1e30f;
  if (h->L.valid) {
    // (lanes, mode): pipelined 4 and 2 lanes, one request per 4 and per 2 lanes
    const int lg[4][2] = {{4, 3}, {2, 3}, {4, 1}, {2, 1}};
    int best_i = 0;
    for (int i = 0; i < 4; i++) {
      h->learned_group = lg[i][0];
      h->learned_mode = lg[i][1];
      const float ms = time_ms(s, [&] { launch_learned_lookup(h, keys, nullptr, nullptr, n, w.uans, w.uans_st, s); });
      out[8 + i] = ms;
      if (ms < best_learned) {
        best_learned = ms;
        best_i = i;
      }
    }
    h->learned_group = lg[best_i][0];
    h->learned_mode = lg[best_i][1];
    out[1] = lg[best_i][0];
    out[15] = lg[best_i][1];
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
    // the hash front end's lookups are unsorted; the full-sort front end's are sorted
    if (h->front_end == 1 ? best_learned < best : ms < bs) desc = 1;
  }
  h->batch_descent = desc;
  out[3] = desc;
  // radix sort tile (threads x 8 items): on the whole sample (the full-sort
  // front end sorts whole batches) and on a sixteenth of it (about the
  // touched requests of a read-mostly batch under the hash front end)
  const int tt[3] = {256, 512, 1024};
  for (int pass = 0; pass < 2; pass++) {
    const size_t m = pass == 0 ? n : (n / 16 ? n / 16 : 1);
    float bt = 1e30f;
    int best_t = 512;
    for (int i = 0; i < 3; i++) {
      const float ms = time_ms(s, [&] {
        radix_sort_pairs(keys, nullptr, nullptr, w.k_a, w.v_a, w.k_b, w.v_b, m, 0, 64, w.sort_scratch, s, &sk, &sv,
                         &h->tree.ctrl->error, nullptr, tt[i]);
      });
      out[18 + 3 * pass + i] = ms;
      if (ms < bt) {
        bt = ms;
        best_t = tt[i];
      }
    }
    if (pass == 0) h->sort_threads = best_t;
    else h->sort_threads_touch = best_t;
    out[16 + pass] = best_t;
  }
  if (cudaStreamSynchronize(s) != cudaSuccess) return -2;
  if (rep)
    for (int i = 0; i < kTuneReport; i++) rep[i] = out[i];
  return 0;
}

}  // namespace bt
