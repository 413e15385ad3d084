// Grouped lock-free descent shared by the plain search kernel and the learned
// search's fallback.  A group of G lanes serves one request; each lane owns
// S = 32/G consecutive slots of a node row and loads them with 16-byte loads
// through the read-only path (valid only while no writer runs: the batch
// executor never overlaps this with the STM insert phase).
#pragma once
#include "bt_common.cuh"

namespace bt {

template <int G>
__device__ __forceinline__ uint32_t group_mask(uint32_t lane) {
  if constexpr (G == 32) return 0xffffffffu;
  else return ((1u << G) - 1u) << (lane - lane % G);
}

template <int S>
__device__ __forceinline__ void load_slots(const uint64_t* p, uint64_t (&x)[S]) {
  if constexpr (S == 1) {
    x[0] = __ldg(p);
  } else {
#pragma unroll
    for (int i = 0; i < S; i += 2) {
      ulonglong2 w = __ldg(reinterpret_cast<const ulonglong2*>(p + i));
      x[i] = w.x;
      x[i + 1] = w.y;
    }
  }
}

// L2 eviction priorities for the descent (createpolicy + ld.global.nc with
// an L2 cache hint, PTX ISA 7.4+): inner rows are read by every lookup and
// should stay in L2 (evict_last); a leaf row or value is read once per
// lookup and should not push them out (evict_first).
__device__ __forceinline__ uint64_t l2_keep() {
  uint64_t p;
  asm("createpolicy.fractional.L2::evict_last.b64 %0, 1.0;" : "=l"(p));
  return p;
}

__device__ __forceinline__ uint64_t l2_stream() {
  uint64_t p;
  asm("createpolicy.fractional.L2::evict_first.b64 %0, 1.0;" : "=l"(p));
  return p;
}

__device__ __forceinline__ uint64_t ldg_hint(const uint64_t* p, uint64_t pol) {
  uint64_t r;
  asm("ld.global.nc.L2::cache_hint.u64 %0, [%1], %2;" : "=l"(r) : "l"(p), "l"(pol));
  return r;
}

__device__ __forceinline__ ulonglong2 ldg2_hint(const void* p, uint64_t pol) {
  ulonglong2 r;
  asm("ld.global.nc.L2::cache_hint.v2.u64 {%0, %1}, [%2], %3;" : "=l"(r.x), "=l"(r.y) : "l"(p), "l"(pol));
  return r;
}

template <int S>
__device__ __forceinline__ void load_slots_hint(const uint64_t* p, uint64_t (&x)[S], uint64_t pol) {
  if constexpr (S == 1) {
    x[0] = ldg_hint(p, pol);
  } else {
#pragma unroll
    for (int i = 0; i < S; i += 2)
      asm("ld.global.nc.L2::cache_hint.v2.u64 {%0, %1}, [%2], %3;"
          : "=l"(x[i]), "=l"(x[i + 1])
          : "l"(p + i), "l"(pol));
  }
}

// A row of 32 slots read by a group of G lanes in 16-byte chunks interleaved
// across the lanes: load i of lane g reads chunk i * G + g (slots 2(iG + g)
// and 2(iG + g) + 1), so one warp-wide load instruction covers one contiguous
// 16G-byte piece of each group's row instead of G pieces 64 bytes apart:
// half the 128-byte lines per instruction at G = 4, the unit the L1 data
// pipe works in.  Slot s lives in lane (s / 2) % G, element 2 * (s / 2 / G) +
// s % 2; slot 31 (the header) in lane G - 1, element S - 1.
template <int G>
__device__ __forceinline__ void load_row_il(const uint64_t* row, uint32_t g, uint64_t (&x)[32 / G], uint64_t pol) {
  constexpr int S = 32 / G;
  if constexpr (S == 1) {
    x[0] = ldg_hint(row + g, pol);
  } else {
#pragma unroll
    for (int i = 0; i < S / 2; i++)
      asm("ld.global.nc.L2::cache_hint.v2.u64 {%0, %1}, [%2], %3;"
          : "=l"(x[2 * i]), "=l"(x[2 * i + 1])
          : "l"(row + 2 * (i * G + g)), "l"(pol));
  }
}

// owner lane and element of slot s in an interleaved row
template <int G>
__device__ __forceinline__ uint32_t il_lane(uint32_t s) {
  return G == 32 ? s : (s >> 1) % G;
}
template <int G>
__device__ __forceinline__ uint32_t il_elem(uint32_t s) {
  return G == 32 ? 0 : 2 * ((s >> 1) / G) + (s & 1);
}

// S 32-bit separator prefixes of a row (S = 2, 4 or 8)
template <int S>
__device__ __forceinline__ void load_pfx(const uint32_t* p, uint32_t (&x)[S], uint64_t pol) {
  if constexpr (S == 2) {
    asm("ld.global.nc.L2::cache_hint.v2.u32 {%0, %1}, [%2], %3;" : "=r"(x[0]), "=r"(x[1]) : "l"(p), "l"(pol));
  } else {
#pragma unroll
    for (int i = 0; i < S; i += 4)
      asm("ld.global.nc.L2::cache_hint.v4.u32 {%0, %1, %2, %3}, [%4], %5;"
          : "=r"(x[i]), "=r"(x[i + 1]), "=r"(x[i + 2]), "=r"(x[i + 3])
          : "l"(p + i), "l"(pol));
  }
}

template <int S>
__device__ __forceinline__ uint64_t pick(const uint64_t (&x)[S], uint32_t e) {
  uint64_t r = x[0];
#pragma unroll
  for (int i = 1; i < S; i++)
    if (e == (uint32_t)i) r = x[i];
  return r;
}

template <int G>
__device__ __forceinline__ uint32_t group_sum(uint32_t c, uint32_t gmask) {
#pragma unroll
  for (int o = G / 2; o >= 1; o >>= 1) c += __shfl_xor_sync(gmask, c, o, G);
  return c;
}

// Rank of `key` in an inner row from the prefixes: slots whose prefix is
// below the key's count, slots with an equal prefix are counted in bits
// 16.. (the caller then ranks with the full keys); slot 31 is the header.
template <int G, int S>
__device__ __forceinline__ uint32_t pfx_rank(const uint32_t (&p)[S], uint64_t key, uint32_t g, uint32_t gmask) {
  const uint32_t kp = (uint32_t)(key >> 32);
  uint32_t x = 0;
#pragma unroll
  for (int i = 0; i < S; i++)
    if (!(g == (uint32_t)(G - 1) && i == S - 1)) x += p[i] < kp ? 1u : (p[i] == kp ? 0x10000u : 0u);
  return group_sum<G>(x, gmask);
}

// Look `key` up in leaf `node` (slots loaded by the group); returns the status
// and the value (deferred 32 B load of the one matching slot).
template <int G, bool kLeafVals>
__device__ __forceinline__ uint8_t group_leaf_lookup(const DevTree& t, uint32_t node, uint64_t key, uint32_t g,
                                                     uint32_t gmask, const uint64_t (&k)[32 / G],
                                                     const uint64_t (&v)[32 / G], uint32_t cnt, uint64_t& ans) {
  constexpr int S = 32 / G;
  ans = 0;
  if (cnt == 0) return kAbsent;
  const uint32_t slot = cnt - 1;
  const uint32_t owner = slot / S, e = slot % S;
  const uint64_t kk = __shfl_sync(gmask, pick<S>(k, e), owner, G);
  if (kk != key) return kAbsent;
  if (kLeafVals) ans = __shfl_sync(gmask, pick<S>(v, e), owner, G);
  else ans = (g == 0) ? __ldg(t.vals + (size_t)node * 32 + slot) : 0;
  return kFound;
}

// The same for a leaf row loaded without its values, with the value load
// given L2 eviction policy `pol`.
template <int G>
__device__ __forceinline__ uint8_t group_leaf_lookup_hint(const DevTree& t, uint32_t node, uint64_t key, uint32_t g,
                                                          uint32_t gmask, const uint64_t (&k)[32 / G], uint32_t cnt,
                                                          uint64_t pol, uint64_t& ans) {
  constexpr int S = 32 / G;
  ans = 0;
  if (cnt == 0) return kAbsent;
  const uint32_t slot = cnt - 1;
  const uint64_t kk = __shfl_sync(gmask, pick<S>(k, slot % S), slot / S, G);
  if (kk != key) return kAbsent;
  ans = (g == 0) ? ldg_hint(t.vals + (size_t)node * 32 + slot, pol) : 0;
  return kFound;
}

// Root-to-leaf descent: child slot = number of keys <= target (child i covers
// [key[i-1], key[i]), src/tree.h:7-19).
template <int G, bool kLeafVals>
__device__ __forceinline__ uint8_t group_descend(const DevTree& t, uint32_t node, uint32_t level, uint64_t key,
                                                 uint32_t g, uint32_t gmask, uint64_t& ans) {
  constexpr int S = 32 / G;
  uint64_t k[S];
  uint64_t v[S];
  uint32_t cnt;
  for (;;) {
    const size_t row = (size_t)node * 32 + g * S;
    load_slots<S>(t.keys + row, k);
    if (level > 0 || kLeafVals) load_slots<S>(t.vals + row, v);
    if (g == G - 1) k[S - 1] = kKeyMax;  // slot 31 holds the header
    uint32_t c = 0;
#pragma unroll
    for (int i = 0; i < S; i++) c += (k[i] <= key) ? 1u : 0u;
    cnt = group_sum<G>(c, gmask);
    if (level == 0) break;
    const uint64_t mine = pick<S>(v, cnt % S);
    node = (uint32_t)__shfl_sync(gmask, mine, cnt / S, G);
    level--;
  }
  return group_leaf_lookup<G, kLeafVals>(t, node, key, g, gmask, k, v, cnt, ans);
}

// Two descents in lock step (same tree, same height): every level issues the
// row loads of both requests before using either, doubling the loads a group
// keeps in flight.  Results as group_descend for each key.
// kChild: at inner levels load only the chosen child id (one 32 B sector)
// after the key comparison instead of the whole 256 B child row with the keys:
// fewer bytes per level, one more dependent load.
// use_pfx (kChild only): inner levels compare the 32-bit separator prefixes
// (half the bytes of the key row) and read the full keys only when a prefix
// equals the key's.
template <int G, bool kLeafVals, bool kChild = false>
__device__ __forceinline__ void group_descend2(const DevTree& t, uint32_t node, uint32_t level, uint64_t key_a,
                                               uint64_t key_b, uint32_t g, uint32_t gmask, uint64_t& ans_a,
                                               uint8_t& st_a, uint64_t& ans_b, uint8_t& st_b,
                                               bool use_pfx = false) {
  constexpr int S = 32 / G;
  uint64_t ka[S], va[S], kb[S], vb[S];
  uint32_t na = node, nb = node;
  uint32_t ca, cb;
  const uint64_t keep = l2_keep(), stream = l2_stream();
  for (;;) {
    const size_t ra = (size_t)na * 32 + g * S, rb = (size_t)nb * 32 + g * S;
    if (kChild && use_pfx && level > 0) {
      uint32_t pa[S], pb[S];
      load_pfx<S>(t.pfx + ra, pa, keep);
      load_pfx<S>(t.pfx + rb, pb, keep);
      const uint32_t xa = pfx_rank<G, S>(pa, key_a, g, gmask), xb = pfx_rank<G, S>(pb, key_b, g, gmask);
      ca = xa & 0xffffu;
      cb = xb & 0xffffu;
      if (xa >> 16) {  // a separator shares the key's prefix: rank with the full keys
        load_slots_hint<S>(t.keys + ra, ka, keep);
        if (g == G - 1) ka[S - 1] = kKeyMax;
        uint32_t c = 0;
#pragma unroll
        for (int i = 0; i < S; i++) c += (ka[i] <= key_a) ? 1u : 0u;
        ca = group_sum<G>(c, gmask);
      }
      if (xb >> 16) {
        load_slots_hint<S>(t.keys + rb, kb, keep);
        if (g == G - 1) kb[S - 1] = kKeyMax;
        uint32_t c = 0;
#pragma unroll
        for (int i = 0; i < S; i++) c += (kb[i] <= key_b) ? 1u : 0u;
        cb = group_sum<G>(c, gmask);
      }
      na = (uint32_t)ldg_hint(t.vals + (size_t)na * 32 + ca, keep);
      nb = (uint32_t)ldg_hint(t.vals + (size_t)nb * 32 + cb, keep);
      level--;
      continue;
    }
    if (kChild) {
      // interleaved 16-byte chunks (load_row_il): the lane counts below do
      // not depend on which slots a lane holds, only the leaf's key pick does
      const uint64_t pol = level > 0 ? keep : stream;
      load_row_il<G>(t.keys + (size_t)na * 32, g, ka, pol);
      load_row_il<G>(t.keys + (size_t)nb * 32, g, kb, pol);
    } else {
      load_slots<S>(t.keys + ra, ka);
      load_slots<S>(t.keys + rb, kb);
    }
    if ((level > 0 && !kChild) || (level == 0 && kLeafVals)) {
      load_slots<S>(t.vals + ra, va);
      load_slots<S>(t.vals + rb, vb);
    }
    if (g == G - 1) {
      ka[S - 1] = kKeyMax;  // slot 31 holds the header
      kb[S - 1] = kKeyMax;
    }
    uint32_t xa = 0, xb = 0;
#pragma unroll
    for (int i = 0; i < S; i++) {
      xa += (ka[i] <= key_a) ? 1u : 0u;
      xb += (kb[i] <= key_b) ? 1u : 0u;
    }
    ca = group_sum<G>(xa, gmask);
    cb = group_sum<G>(xb, gmask);
    if (level == 0) break;
    if (kChild) {
      na = (uint32_t)ldg_hint(t.vals + (size_t)na * 32 + ca, keep);
      nb = (uint32_t)ldg_hint(t.vals + (size_t)nb * 32 + cb, keep);
    } else {
      const uint64_t ma = pick<S>(va, ca % S), mb = pick<S>(vb, cb % S);
      na = (uint32_t)__shfl_sync(gmask, ma, ca / S, G);
      nb = (uint32_t)__shfl_sync(gmask, mb, cb / S, G);
    }
    level--;
  }
  // leaf: find both slots, then issue both value loads together
  const uint32_t sa = ca > 0 ? ca - 1 : 0, sb = cb > 0 ? cb - 1 : 0;
  const uint64_t kka = kChild ? __shfl_sync(gmask, pick<S>(ka, il_elem<G>(sa)), il_lane<G>(sa), G)
                              : __shfl_sync(gmask, pick<S>(ka, sa % S), sa / S, G);
  const uint64_t kkb = kChild ? __shfl_sync(gmask, pick<S>(kb, il_elem<G>(sb)), il_lane<G>(sb), G)
                              : __shfl_sync(gmask, pick<S>(kb, sb % S), sb / S, G);
  const bool fa = ca > 0 && kka == key_a, fb = cb > 0 && kkb == key_b;
  ans_a = 0;
  ans_b = 0;
  if (kLeafVals) {
    const uint64_t xa = __shfl_sync(gmask, pick<S>(va, sa % S), sa / S, G);
    const uint64_t xb = __shfl_sync(gmask, pick<S>(vb, sb % S), sb / S, G);
    ans_a = fa ? xa : 0;
    ans_b = fb ? xb : 0;
  } else if (g == 0) {
    if (fa) ans_a = kChild ? ldg_hint(t.vals + (size_t)na * 32 + sa, stream) : __ldg(t.vals + (size_t)na * 32 + sa);
    if (fb) ans_b = kChild ? ldg_hint(t.vals + (size_t)nb * 32 + sb, stream) : __ldg(t.vals + (size_t)nb * 32 + sb);
  }
  st_a = fa ? kFound : kAbsent;
  st_b = fb ? kFound : kAbsent;
}

}  // namespace bt
