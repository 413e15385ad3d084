// Learned leaf predictor (filled in below; placeholder entry points).
#include <cuda_runtime.h>

#include "bt_common.cuh"
#include "bt_internal.h"

namespace bt {

int learned_retrain(Handle* h, cudaStream_t s) {
  (void)h;
  (void)s;
  return -7;
}

void learned_free(Learned* L) { (void)L; }

cudaError_t launch_learned_search(Handle* h, const uint64_t* qkeys, const uint32_t* list, const uint32_t* n_dev,
                                  size_t n, uint64_t* out_vals, uint8_t* out_st, cudaStream_t s) {
  return launch_search(h, qkeys, list, n_dev, n, out_vals, out_st, s);
}

}  // namespace bt
