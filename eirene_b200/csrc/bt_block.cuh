// Block-wide scan primitives shared by the batch kernels.
#pragma once
#include <cstdint>

namespace bt {

// exclusive sum over the block (any multiple of 32 threads up to 1024);
// `ws` is 32 words of shared memory; optional block total.
__device__ __forceinline__ uint32_t blk_exclusive_sum(uint32_t v, uint32_t* ws, uint32_t* total) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
  uint32_t x = v;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    uint32_t y = __shfl_up_sync(0xffffffffu, x, o);
    if (lane >= o) x += y;
  }
  if (lane == 31) ws[warp] = x;
  __syncthreads();
  if (warp == 0) {
    uint32_t s = lane < nw ? ws[lane] : 0;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      uint32_t y = __shfl_up_sync(0xffffffffu, s, o);
      if (lane >= o) s += y;
    }
    if (lane < nw) ws[lane] = s;
  }
  __syncthreads();
  const uint32_t base = warp ? ws[warp - 1] : 0;
  if (total) *total = ws[nw - 1];
  __syncthreads();
  return base + x - v;
}

// "latest write in the current run" segment state: flags bit0 = a run head
// occurred, bit1 = a write (INSERT or DELETE) occurred after the last head,
// bit2 = that latest write was a DELETE; v = the latest INSERT's value.
struct Seg {
  uint32_t f;
  uint64_t v;
};
__device__ __forceinline__ Seg seg_combine(Seg a, Seg b) {
  Seg r;
  r.f = (a.f | b.f) & 1u;
  if (b.f & 2u) {
    r.f |= b.f & 6u;
    r.v = b.v;
  } else if (b.f & 1u) {
    r.v = 0;
  } else {
    r.f |= a.f & 6u;
    r.v = a.v;
  }
  return r;
}

// exclusive segmented scan over the block; `wsf`/`wsv` are 32-entry shared arrays.
// `prefix` is combined in front of the block; the block aggregate (without prefix)
// is returned through `agg`.
__device__ __forceinline__ Seg blk_exclusive_seg(Seg x, Seg prefix, uint32_t* wsf, uint64_t* wsv, Seg* agg) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
  Seg inc = x;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    Seg y;
    y.f = __shfl_up_sync(0xffffffffu, inc.f, o);
    y.v = __shfl_up_sync(0xffffffffu, inc.v, o);
    if (lane >= o) inc = seg_combine(y, inc);
  }
  Seg ex;
  ex.f = __shfl_up_sync(0xffffffffu, inc.f, 1);
  ex.v = __shfl_up_sync(0xffffffffu, inc.v, 1);
  if (lane == 0) {
    ex.f = 0;
    ex.v = 0;
  }
  if (lane == 31) {
    wsf[warp] = inc.f;
    wsv[warp] = inc.v;
  }
  __syncthreads();
  if (warp == 0) {
    Seg s;
    s.f = lane < nw ? wsf[lane] : 0u;
    s.v = lane < nw ? wsv[lane] : 0ull;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      Seg y;
      y.f = __shfl_up_sync(0xffffffffu, s.f, o);
      y.v = __shfl_up_sync(0xffffffffu, s.v, o);
      if (lane >= o) s = seg_combine(y, s);
    }
    if (lane < nw) {
      wsf[lane] = s.f;
      wsv[lane] = s.v;
    }
  }
  __syncthreads();
  Seg wp;
  if (warp) {
    wp.f = wsf[warp - 1];
    wp.v = wsv[warp - 1];
  } else {
    wp.f = 0;
    wp.v = 0;
  }
  if (agg) {
    agg->f = wsf[nw - 1];
    agg->v = wsv[nw - 1];
  }
  __syncthreads();
  return seg_combine(prefix, seg_combine(wp, ex));
}

}  // namespace bt
