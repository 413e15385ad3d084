// C ABI of libeirene_b200 (declared in include/eirene_b200.h).
#include <cstdlib>
#include <cstring>
#include <new>
#include <vector>

#include <cuda_runtime.h>

#include "../../include/eirene_b200.h"
#include "bt_common.cuh"
#include "bt_internal.h"


namespace {

// Make h's device current for the duration of a call; restore on exit.
struct DeviceGuard {
  int prev = -1;
  bool ok = true;
  explicit DeviceGuard(int dev) {
    if (cudaGetDevice(&prev) != cudaSuccess) prev = -1;
    if (prev != dev) ok = cudaSetDevice(dev) == cudaSuccess;
  }
  ~DeviceGuard() {
    int cur = -1;
    if (prev >= 0 && cudaGetDevice(&cur) == cudaSuccess && cur != prev) cudaSetDevice(prev);
  }
};

// DeviceGuard for an entry point that may use the handle's buffers: it also
// closes the chain of host batches (the next host batch's front part then
// waits for everything queued before it)
struct EntryGuard : DeviceGuard {
  explicit EntryGuard(bt_handle* H) : DeviceGuard(H->h.device) { H->h.chain_open = false; }
};

inline cudaStream_t S(void* s) { return reinterpret_cast<cudaStream_t>(s); }

int map_internal(int rc) {
  switch (rc) {
    case 0: return BT_OK;
    case -1: return BT_ERR_INVALID_ARG;
    case -2: return BT_ERR_CUDA;
    case -3: return BT_ERR_NO_MEMORY;
    case -4: return BT_ERR_CAPACITY;
    case -5: return BT_ERR_RESERVED_KEY;
    case -6: return BT_ERR_BATCH_TOO_LARGE;
    case -7: return BT_ERR_NOT_TRAINED;
    default: return BT_ERR_CUDA;
  }
}

// node pool size for max_keys: every node holds at least 15 keys except the
// few rightmost/root nodes, so 2*max_keys/15 + slack bounds the count for
// any insert order; the bulk layout needs far fewer.
uint64_t pool_nodes(uint64_t max_keys) { return max_keys / 7 + 4096; }

}  // namespace

namespace bt {
cudaError_t sort_prepare();
std::atomic<unsigned long long> g_launches{0};

void prof_mark(Handle* h, int which, cudaStream_t s) {
  if (!h->prof) return;
  const size_t base = h->prof_batches * kProfEvents;
  if (which == 0) {
    // grow the event pool by one batch
    while (h->prof_ev.size() < base + kProfEvents) {
      cudaEvent_t e;
      if (cudaEventCreate(&e) != cudaSuccess) return;
      h->prof_ev.push_back(e);
    }
    if (h->prof_layout.size() <= h->prof_batches) h->prof_layout.resize(h->prof_batches + 1);
    h->prof_layout[h->prof_batches] = 0;
  }
  if (base + which < h->prof_ev.size()) cudaEventRecord(h->prof_ev[base + which], s);
  if (which == kNumPhases) h->prof_batches++;
}

void prof_set_layout(Handle* h, int layout) {
  if (h->prof && h->prof_batches < h->prof_layout.size()) h->prof_layout[h->prof_batches] = (char)layout;
}

cudaError_t tree_join(Handle* h, cudaStream_t s) {
  return h->tree_pending ? cudaStreamWaitEvent(s, h->tree_ev, 0) : cudaSuccess;
}

cudaError_t tree_sync(Handle* h) {
  if (!h->tree_pending) return cudaSuccess;
  const cudaError_t e = cudaEventSynchronize(h->tree_ev);
  if (e == cudaSuccess) h->tree_pending = false;
  return e;
}
}  // namespace bt

namespace {
// fold recorded batches into phase_ms (synchronises on the events)
int prof_resolve(bt::Handle& h) {
  for (size_t b = 0; b < h.prof_batches; b++) {
    cudaEvent_t* e = &h.prof_ev[b * bt::kProfEvents];
    if (cudaEventSynchronize(e[bt::kNumPhases]) != cudaSuccess) return BT_ERR_CUDA;
    auto t = [&](int a, int z, float* ms) { return cudaEventElapsedTime(ms, e[a], e[z]) == cudaSuccess; };
    float ms[bt::kNumPhases] = {};
    bool ok = true;
    const int layout = b < h.prof_layout.size() ? h.prof_layout[b] : 0;
    if (layout & bt::kLayoutOverlap) {
      // front + touched sort | merge passes, then the locates (side stream) |
      // lookups (main stream, beside the locates)
      ok = t(0, bt::kEvSortEnd, &ms[bt::kPhSort]) && t(bt::kEvSortEnd, 2, &ms[bt::kPhMerge]) &&
           t(1, bt::kEvLookupEnd, &ms[bt::kPhSearch]);
    } else {
      for (int p = 0; ok && p < bt::kPhInsert; p++) ok = t(p, p + 1, &ms[p]);
    }
    if (layout & bt::kLayoutEarly) {
      // insert = DELETE apply + leaf reservation, then the leaf/inner merge
      // (on the tree stream when deferred); writeback between the two
      float a = 0, z = 0;
      ok = ok && t(3, bt::kEvWbStart, &a) && t(4, 5, &z) && t(bt::kEvWbStart, 4, &ms[bt::kPhWriteback]);
      ms[bt::kPhInsert] = a + z;
    } else {
      ok = ok && t(3, 4, &ms[bt::kPhInsert]) && t(4, 5, &ms[bt::kPhWriteback]);
    }
    if (!ok) return BT_ERR_CUDA;
    for (int p = 0; p < bt::kNumPhases; p++) h.phase_ms[p] += ms[p];
    h.phase_batches++;
  }
  h.prof_batches = 0;
  return BT_OK;
}
}  // namespace

extern "C" {

int bt_config_init(bt_config* c) {
  if (!c) return BT_ERR_INVALID_ARG;
  std::memset(c, 0, sizeof(*c));
  c->max_keys = 1ull << 20;
  c->max_batch = 1ull << 22;
  c->leaf_fill = 24;
  c->inner_fill = 24;
  c->retry_limit = 1u << 16;
  c->device = 0;
  c->search_group = 4;
  c->n_segments = 0;
  c->window = 64;
  return BT_OK;
}

static void hostpipe_free(bt::HostPipe& p);

int bt_create(const bt_config* cfg_in, bt_handle** out) {
  if (!out) return BT_ERR_INVALID_ARG;
  *out = nullptr;
  bt_config cfg;
  if (cfg_in) cfg = *cfg_in;
  else bt_config_init(&cfg);
  if (cfg.leaf_fill < 2 || cfg.leaf_fill > 31 || cfg.inner_fill < 1 || cfg.inner_fill > 31) return BT_ERR_INVALID_ARG;
  if (cfg.search_group != 4 && cfg.search_group != 8 && cfg.search_group != 16 && cfg.search_group != 32)
    return BT_ERR_INVALID_ARG;
  if (cfg.max_batch == 0 || cfg.max_batch > (1ull << 30)) return BT_ERR_INVALID_ARG;
  const uint64_t nodes = pool_nodes(cfg.max_keys);
  if (nodes >= 0xFFFFFFF0ull) return BT_ERR_INVALID_ARG;
  int n_dev = 0;
  if (cudaGetDeviceCount(&n_dev) != cudaSuccess || cfg.device < 0 || cfg.device >= n_dev) return BT_ERR_CUDA;
  DeviceGuard g(cfg.device);
  if (!g.ok) return BT_ERR_CUDA;
  bt_handle* H = new (std::nothrow) bt_handle();
  if (!H) return BT_ERR_NO_MEMORY;
  bt::Handle& h = H->h;
  h.device = cfg.device;
  h.leaf_fill = cfg.leaf_fill;
  h.inner_fill = cfg.inner_fill;
  h.retry_limit = cfg.retry_limit ? cfg.retry_limit : (1u << 16);
  h.search_group = (int)cfg.search_group;
  h.L.seg_config = cfg.n_segments;
  h.L.n_segments = cfg.n_segments ? cfg.n_segments : 4096;
  h.L.window = cfg.window ? cfg.window : 64;
  cudaDeviceGetAttribute(&h.sm_count, cudaDevAttrMultiProcessorCount, cfg.device);
  bool ok = bt::sort_prepare() == cudaSuccess;
  h.tree.cap = (uint32_t)nodes;
  ok = ok && cudaMalloc(&h.tree.keys, nodes * 256) == cudaSuccess;
  ok = ok && cudaMalloc(&h.tree.vals, nodes * 256) == cudaSuccess;
  ok = ok && cudaMalloc(&h.tree.low, nodes * 8) == cudaSuccess;
  ok = ok && cudaMalloc(&h.tree.pfx, nodes * 128) == cudaSuccess;
  ok = ok && cudaMalloc(&h.tree.ctrl, sizeof(bt::Ctrl)) == cudaSuccess;
  // zeroed rows read as epoch 0, which no tree uses (see hdr_epoch)
  ok = ok && cudaMemset(h.tree.keys, 0, nodes * 256) == cudaSuccess;
  ok = ok && cudaMemset(h.tree.vals, 0, nodes * 256) == cudaSuccess;
  ok = ok && cudaMemset(h.tree.low, 0, nodes * 8) == cudaSuccess;
  ok = ok && cudaMemset(h.tree.pfx, 0xff, nodes * 128) == cudaSuccess;
  ok = ok && bt::work_alloc(&h.w, cfg.max_batch) == 0;
  ok = ok && cudaStreamCreateWithFlags(&h.internal_stream, cudaStreamNonBlocking) == cudaSuccess;
  {
    int lo_prio = 0, hi_prio = 0;
    cudaDeviceGetStreamPriorityRange(&lo_prio, &hi_prio);
    ok = ok && cudaStreamCreateWithPriority(&h.hi_stream, cudaStreamNonBlocking, hi_prio) == cudaSuccess &&
         cudaEventCreateWithFlags(&h.fork_ev, cudaEventDisableTiming) == cudaSuccess &&
         cudaEventCreateWithFlags(&h.join_ev, cudaEventDisableTiming) == cudaSuccess;
    ok = ok && cudaStreamCreateWithFlags(&h.tree_stream, cudaStreamNonBlocking) == cudaSuccess &&
         cudaEventCreateWithFlags(&h.tree_ev, cudaEventDisableTiming) == cudaSuccess &&
         cudaEventCreateWithFlags(&h.ans_ev, cudaEventDisableTiming) == cudaSuccess;
  }
  // the touched-request count of the batches, written by the front end into
  // page-locked mapped memory: the next batches' sort choice (BT_OPT_TOUCH_SORT 2)
  ok = ok && cudaHostAlloc((void**)&h.touch_hint, sizeof(uint32_t), cudaHostAllocMapped) == cudaSuccess &&
       cudaHostGetDevicePointer((void**)&h.touch_hint_dev, h.touch_hint, 0) == cudaSuccess;
  if (h.touch_hint) *h.touch_hint = UINT32_MAX;  // none seen yet
  ok = ok && bt::tree_reset(&h, h.internal_stream) == cudaSuccess;
  ok = ok && cudaStreamSynchronize(h.internal_stream) == cudaSuccess;
  if (!ok) {
    bt_destroy(H);
    return BT_ERR_NO_MEMORY;
  }
  *out = H;
  return BT_OK;
}

int bt_destroy(bt_handle* H) {
  if (!H) return BT_ERR_INVALID_ARG;
  EntryGuard g(H);
  bt::Handle& h = H->h;
  cudaDeviceSynchronize();
  cudaFree(h.tree.keys);
  cudaFree(h.tree.vals);
  cudaFree(h.tree.low);
  cudaFree(h.tree.pfx);
  cudaFree(h.tree.ctrl);
  bt::work_free(&h.w);
  bt::learned_free(&h.L);
  bt::learned_policy_free(&h.L);
  if (h.front_stream) cudaStreamDestroy(h.front_stream);
  if (h.touch_hint) cudaFreeHost(h.touch_hint);
  for (cudaEvent_t e : {h.front_done[0], h.front_done[1], h.tree_done[0], h.tree_done[1], h.pipe_ev,
                        h.chain_gate})
    if (e) cudaEventDestroy(e);
  cudaFree(h.enum_a);
  cudaFree(h.enum_b);
  cudaFree(h.enum_cnt);
  cudaFree(h.enum_scan_scratch);
  cudaFree(h.top);
  if (h.internal_stream) cudaStreamDestroy(h.internal_stream);
  if (h.hi_stream) cudaStreamDestroy(h.hi_stream);
  if (h.fork_ev) cudaEventDestroy(h.fork_ev);
  if (h.join_ev) cudaEventDestroy(h.join_ev);
  hostpipe_free(h.hp);
  if (h.tree_stream) cudaStreamDestroy(h.tree_stream);
  if (h.tree_ev) cudaEventDestroy(h.tree_ev);
  if (h.ans_ev) cudaEventDestroy(h.ans_ev);
  for (cudaEvent_t e : h.prof_ev) cudaEventDestroy(e);
  delete H;
  return BT_OK;
}

int bt_bulk_build(bt_handle* H, const uint64_t* keys, const uint64_t* vals, size_t n, void* stream) {
  if (!H || (n && (!keys || !vals))) return BT_ERR_INVALID_ARG;
  EntryGuard g(H);
  H->h.L.valid = false;
  if (bt::tree_join(&H->h, S(stream)) != cudaSuccess) return BT_ERR_CUDA;
  return map_internal(bt::tree_bulk_build(&H->h, keys, vals, n, S(stream)));
}

int bt_execute_batch(bt_handle* H, const uint64_t* keys, const uint64_t* vals, const uint8_t* ops,
                     uint64_t* out_vals, uint8_t* out_status, size_t n, int mode, void* stream) {
  if (!H) return BT_ERR_INVALID_ARG;
  if (n == 0) return BT_OK;
  if (!keys || !ops || !out_vals || !out_status || !vals) return BT_ERR_INVALID_ARG;
  bt::Handle& h = H->h;
  if (n > h.w.cap) return BT_ERR_BATCH_TOO_LARGE;
  EntryGuard g(H);
  const int base = mode & 0xF;
  if (base == BT_MODE_STM) {
    if (bt::tree_join(&h, S(stream)) != cudaSuccess) return BT_ERR_CUDA;
    return map_internal(bt::batch_stm(&h, keys, vals, ops, out_vals, out_status, n, S(stream)));
  }
  if (base != BT_MODE_SORTED) return BT_ERR_INVALID_ARG;
  const int engine = (mode & BT_MODE_MERGE_ENGINE) ? 1 : 0;
  return map_internal(bt::batch_sorted(&h, keys, vals, ops, out_vals, out_status, n, engine, S(stream)));
}

int bt_execute_batches(bt_handle* H, size_t count, const uint64_t* const* keys, const uint64_t* const* vals,
                       const uint8_t* const* ops, uint64_t* const* out_vals, uint8_t* const* out_status,
                       const size_t* n, int mode, void* stream) {
  if (!H) return BT_ERR_INVALID_ARG;
  if (count == 0) return BT_OK;
  if (!keys || !vals || !ops || !out_vals || !out_status || !n) return BT_ERR_INVALID_ARG;
  bt::Handle& h = H->h;
  for (size_t j = 0; j < count; j++) {
    if (n[j] == 0) continue;
    if (!keys[j] || !vals[j] || !ops[j] || !out_vals[j] || !out_status[j]) return BT_ERR_INVALID_ARG;
    if (n[j] > h.w.cap) return BT_ERR_BATCH_TOO_LARGE;
  }
  const int base = mode & 0xF;
  if (base != BT_MODE_SORTED && base != BT_MODE_STM) return BT_ERR_INVALID_ARG;
  EntryGuard g(H);
  if (base != BT_MODE_SORTED || h.front_end != 1) {
    // only sorted batches with the hash front end have a front part to run ahead
    for (size_t j = 0; j < count; j++) {
      const int rc = bt_execute_batch(H, keys[j], vals[j], ops[j], out_vals[j], out_status[j], n[j], mode, stream);
      if (rc != BT_OK) return rc;
    }
    return BT_OK;
  }
  // empty batches do nothing: drop them
  std::vector<const uint64_t*> k, v;
  std::vector<const uint8_t*> o;
  std::vector<uint64_t*> ov;
  std::vector<uint8_t*> os;
  std::vector<size_t> m;
  for (size_t j = 0; j < count; j++)
    if (n[j]) {
      k.push_back(keys[j]);
      v.push_back(vals[j]);
      o.push_back(ops[j]);
      ov.push_back(out_vals[j]);
      os.push_back(out_status[j]);
      m.push_back(n[j]);
    }
  const int engine = (mode & BT_MODE_MERGE_ENGINE) ? 1 : 0;
  return map_internal(bt::batches_pipelined(&h, m.size(), k.data(), v.data(), o.data(), ov.data(), os.data(), m.data(),
                                            engine, S(stream)));
}

// ---- host-buffer entry points ----
// A batch from host buffers runs as: op codes and keys copied in on the copy-in
// stream; the values copied in after them (the front end and the sort need
// none; the merge passes wait for them) or, when the caller's value array is
// page-locked, not copied at all: the merge passes read the values of the
// batch's writes over the bus; the batch's kernels on the caller's stream;
// the answers copied out on the copy-out stream as soon as they are final,
// while the leaf merge still runs.  Three staging sets let the next batch's
// copy-in and the previous batch's copy-out run beside this batch's kernels.

static void hostpipe_free(bt::HostPipe& p) {
  for (bt::Staging& st : p.set) {
    cudaFree(st.keys);
    cudaFree(st.vals);
    cudaFree(st.ops);
    cudaFree(st.out_vals);
    cudaFree(st.out_st);
    cudaFree(st.packed);
    cudaFree(st.pack_scratch);
    if (st.pack_err) cudaFreeHost(st.pack_err);
    for (cudaEvent_t e : {st.in_ev, st.vals_ev, st.ans_ev, st.done_ev})
      if (e) cudaEventDestroy(e);
    st = bt::Staging{};
  }
  if (p.in_stream) cudaStreamDestroy(p.in_stream);
  if (p.out_stream) cudaStreamDestroy(p.out_stream);
  p = bt::HostPipe{};
}

static int hostpipe_init(bt::Handle& h) {
  bt::HostPipe& p = h.hp;
  if (p.cap) return BT_OK;
  const size_t cap = h.w.cap;
  // the copy-in stream at the highest priority: its small kernels (the
  // packed values' count and placement) go ahead of the running batch's
  // blocks.  They still wait for SM room behind the running batch's lookup
  // grid, which holds the next batch's key copy back until the lookups end;
  // measured, that is 6 % faster per batch than running them on the batch's
  // own stream: copies beside the latency-bound lookups slow them (a 2^22
  // batch takes 0.91 ms alone, 1.05-1.25 ms with a PCIe copy beside it, in
  // either direction, whatever the copy's footprint in L2)
  int lo_prio = 0, hi_prio = 0;
  cudaDeviceGetStreamPriorityRange(&lo_prio, &hi_prio);
  bool ok = cudaStreamCreateWithPriority(&p.in_stream, cudaStreamNonBlocking, hi_prio) == cudaSuccess &&
            cudaStreamCreateWithFlags(&p.out_stream, cudaStreamNonBlocking) == cudaSuccess;
  for (bt::Staging& st : p.set) {
    ok = ok && cudaMalloc(&st.keys, cap * 8) == cudaSuccess && cudaMalloc(&st.vals, cap * 8) == cudaSuccess &&
         cudaMalloc(&st.ops, cap) == cudaSuccess && cudaMalloc(&st.out_vals, cap * 8) == cudaSuccess &&
         cudaMalloc(&st.out_st, cap) == cudaSuccess;
    for (cudaEvent_t* e : {&st.in_ev, &st.vals_ev, &st.ans_ev, &st.done_ev})
      ok = ok && cudaEventCreateWithFlags(e, cudaEventDisableTiming) == cudaSuccess;
  }
  if (!ok) {
    hostpipe_free(p);
    return BT_ERR_NO_MEMORY;
  }
  p.cap = cap;
  return BT_OK;
}

// the device-side alias of a page-locked host array, or nullptr for
// pageable memory (which the kernels cannot read)
static const uint64_t* mapped_alias(const uint64_t* p) {
  cudaPointerAttributes a{};
  if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
    cudaGetLastError();
    return nullptr;
  }
  return a.type == cudaMemoryTypeHost && a.devicePointer ? static_cast<const uint64_t*>(a.devicePointer) : nullptr;
}

// packed: `vals` holds the values of the batch's INSERTs only, n_packed of
// them in request order; otherwise one value per request.  The count is
// checked on the device, between the op codes' copy and the front end: a
// mismatch turns the batch into one whose every request is rejected, and
// bt_host_wait reports it (a count on the host cost 0.35 ms of the host
// thread per 2^22 requests, more than the copy it saved)
static int host_submit(bt_handle* H, const uint64_t* keys, const uint64_t* vals, size_t n_packed, bool packed,
                       const uint8_t* ops, uint64_t* out_vals, uint8_t* out_status, size_t n, int mode,
                       cudaStream_t s, uint64_t* ticket) {
  bt::Handle& h = H->h;
  const int base = mode & 0xF;
  if (base != BT_MODE_SORTED && base != BT_MODE_STM) return BT_ERR_INVALID_ARG;
  int rc = hostpipe_init(h);
  if (rc != BT_OK) return rc;
  bt::HostPipe& p = h.hp;
  bt::Staging& st = p.set[p.issued % bt::kStagingSets];
  // the set was used kStagingSets batches ago: its answers must be out before
  // its buffers are written again
  if (st.ticket && cudaEventSynchronize(st.done_ev) != cudaSuccess) return BT_ERR_CUDA;
  if (st.ticket && st.packed_batch && *st.pack_err) {
    if (p.refused.size() >= 1024) p.refused.erase(p.refused.begin());  // the oldest are forgotten
    p.refused.push_back(st.ticket);
  }
  st.packed_batch = false;
  if (packed && !st.packed) {
    if (cudaMalloc(&st.packed, p.cap * 8) != cudaSuccess ||
        cudaMalloc(&st.pack_scratch, bt::pack_scratch_words(p.cap) * 4) != cudaSuccess ||
        cudaMallocHost(&st.pack_err, 4) != cudaSuccess) {
      cudaFree(st.packed);
      cudaFree(st.pack_scratch);
      st.packed = nullptr;
      st.pack_scratch = nullptr;
      st.pack_err = nullptr;
      return BT_ERR_NO_MEMORY;
    }
  }
  const auto H2D = cudaMemcpyHostToDevice;
  const auto D2H = cudaMemcpyDeviceToHost;
  // values read in place only when asked for: the merge passes' scattered
  // 8-byte reads over the bus cost more than copying the whole array, which
  // the copy-in stream overlaps with the previous batch's kernels
  const uint64_t* remote =
      (!packed && base == BT_MODE_SORTED && h.host_vals_in_place) ? mapped_alias(vals) : nullptr;
  cudaStream_t in = p.in_stream;
  if (cudaMemcpyAsync(st.ops, ops, n, H2D, in) != cudaSuccess ||
      (packed && bt::pack_check(st.ops, n, n_packed, st.pack_scratch, p.cap, h.sm_count, in) != cudaSuccess) ||
      cudaMemcpyAsync(st.keys, keys, n * 8, H2D, in) != cudaSuccess || cudaEventRecord(st.in_ev, in) != cudaSuccess)
    return BT_ERR_CUDA;
  if (packed) {
    // the INSERTs' values in, then each to its request's slot of st.vals
    if ((n_packed && cudaMemcpyAsync(st.packed, vals, n_packed * 8, H2D, in) != cudaSuccess) ||
        bt::pack_expand(st.ops, n, st.packed, n_packed, st.vals, st.pack_scratch, p.cap, in) != cudaSuccess ||
        cudaEventRecord(st.vals_ev, in) != cudaSuccess)
      return BT_ERR_CUDA;
  } else if (!remote && (cudaMemcpyAsync(st.vals, vals, n * 8, H2D, in) != cudaSuccess ||
                         cudaEventRecord(st.vals_ev, in) != cudaSuccess)) {
    return BT_ERR_CUDA;
  }
  const int engine = (mode & BT_MODE_MERGE_ENGINE) ? 1 : 0;
  // the front part on its own stream once the op codes and keys are in,
  // beside the previous host batch's tree part; the merge passes once the
  // values are in (a full value array: beside the lookups instead)
  const bool chained = base == BT_MODE_SORTED && h.front_end == 1 && h.host_front_overlap && !remote && !h.prof;
  if (chained) {
    h.ans_ready = st.ans_ev;
    rc = map_internal(bt::batch_chained(&h, st.keys, st.vals, st.ops, st.out_vals, st.out_st, n, engine, s,
                                        st.in_ev, st.vals_ev, !packed));
    h.ans_ready = nullptr;
  } else if (cudaStreamWaitEvent(s, st.in_ev, 0) != cudaSuccess) {
    return BT_ERR_CUDA;
  } else if (base == BT_MODE_SORTED) {
    h.chain_open = false;
    h.vals_wait = remote ? nullptr : st.vals_ev;
    h.vals_remote = remote != nullptr;
    h.ans_ready = st.ans_ev;
    rc = map_internal(bt::batch_sorted(&h, st.keys, remote ? remote : st.vals, st.ops, st.out_vals, st.out_st, n,
                                       engine, s));
    h.vals_wait = nullptr;
    h.vals_remote = false;
    h.ans_ready = nullptr;
  } else {
    h.chain_open = false;
    rc = cudaStreamWaitEvent(s, st.vals_ev, 0) == cudaSuccess
             ? bt_execute_batch(H, st.keys, st.vals, st.ops, st.out_vals, st.out_st, n, mode, s)
             : BT_ERR_CUDA;
    if (rc == BT_OK && cudaEventRecord(st.ans_ev, s) != cudaSuccess) rc = BT_ERR_CUDA;
  }
  if (rc != BT_OK) {
    cudaStreamSynchronize(in);
    return rc;
  }
  cudaStream_t out = p.out_stream;
  if (cudaStreamWaitEvent(out, st.ans_ev, 0) != cudaSuccess ||
      cudaMemcpyAsync(out_vals, st.out_vals, n * 8, D2H, out) != cudaSuccess ||
      cudaMemcpyAsync(out_status, st.out_st, n, D2H, out) != cudaSuccess ||
      (packed && cudaMemcpyAsync(st.pack_err, bt::pack_error_word(st.pack_scratch, p.cap), 4, D2H, out) !=
                     cudaSuccess) ||
      cudaEventRecord(st.done_ev, out) != cudaSuccess)
    return BT_ERR_CUDA;
  st.packed_batch = packed;
  st.ticket = ++p.issued;
  if (ticket) *ticket = st.ticket;
  return BT_OK;
}

// BT_ERR_INVALID_ARG for a packed batch whose value count did not match its
// INSERTs (every request answered kRejected, nothing applied)
static int host_wait(bt::Handle& h, uint64_t ticket) {
  bt::HostPipe& p = h.hp;
  if (ticket == 0 || ticket > p.issued) return BT_ERR_INVALID_ARG;
  for (bt::Staging& st : p.set)
    if (st.ticket == ticket) {
      if (cudaEventSynchronize(st.done_ev) != cudaSuccess) return BT_ERR_CUDA;
      return st.packed_batch && *st.pack_err ? BT_ERR_INVALID_ARG : BT_OK;
    }
  // an older batch: its set has been reused, so it has finished
  for (uint64_t t : p.refused)
    if (t == ticket) return BT_ERR_INVALID_ARG;
  return BT_OK;
}

int bt_execute_batch_host_async(bt_handle* H, const uint64_t* keys, const uint64_t* vals, const uint8_t* ops,
                                uint64_t* out_vals, uint8_t* out_status, size_t n, int mode, void* stream,
                                uint64_t* ticket) {
  if (!H || !ticket) return BT_ERR_INVALID_ARG;
  *ticket = 0;
  if (n == 0) return BT_OK;
  if (!keys || !ops || !out_vals || !out_status || !vals) return BT_ERR_INVALID_ARG;
  if (n > H->h.w.cap) return BT_ERR_BATCH_TOO_LARGE;
  DeviceGuard g(H->h.device);
  return host_submit(H, keys, vals, 0, false, ops, out_vals, out_status, n, mode, S(stream), ticket);
}

int bt_execute_batch_host_packed_async(bt_handle* H, const uint64_t* keys, const uint8_t* ops,
                                       const uint64_t* insert_vals, size_t n_inserts, uint64_t* out_vals,
                                       uint8_t* out_status, size_t n, int mode, void* stream, uint64_t* ticket) {
  if (!H || !ticket) return BT_ERR_INVALID_ARG;
  *ticket = 0;
  if (n == 0) return n_inserts == 0 ? BT_OK : BT_ERR_INVALID_ARG;
  if (!keys || !ops || !out_vals || !out_status || (n_inserts && !insert_vals)) return BT_ERR_INVALID_ARG;
  if (n > H->h.w.cap) return BT_ERR_BATCH_TOO_LARGE;
  DeviceGuard g(H->h.device);
  return host_submit(H, keys, insert_vals, n_inserts, true, ops, out_vals, out_status, n, mode, S(stream), ticket);
}

int bt_host_wait(bt_handle* H, uint64_t ticket) {
  if (!H) return BT_ERR_INVALID_ARG;
  if (ticket == 0) return BT_OK;  // an empty batch
  DeviceGuard g(H->h.device);
  return host_wait(H->h, ticket);
}

int bt_execute_batch_host(bt_handle* H, const uint64_t* keys, const uint64_t* vals, const uint8_t* ops,
                          uint64_t* out_vals, uint8_t* out_status, size_t n, int mode, void* stream) {
  if (!H) return BT_ERR_INVALID_ARG;
  if (n == 0) return BT_OK;
  if (!keys || !ops || !out_vals || !out_status || !vals) return BT_ERR_INVALID_ARG;
  if (n > H->h.w.cap) return BT_ERR_BATCH_TOO_LARGE;
  EntryGuard g(H);
  uint64_t t = 0;
  int rc = host_submit(H, keys, vals, 0, false, ops, out_vals, out_status, n, mode, S(stream), &t);
  if (rc != BT_OK) return rc;
  rc = host_wait(H->h, t);
  if (rc != BT_OK) return rc;
  return cudaStreamSynchronize(S(stream)) == cudaSuccess ? BT_OK : BT_ERR_CUDA;
}

int bt_search_batch(bt_handle* H, const uint64_t* keys, uint64_t* out_vals, uint8_t* out_status, size_t n,
                    void* stream) {
  if (!H) return BT_ERR_INVALID_ARG;
  if (n == 0) return BT_OK;
  if (!keys || !out_vals || !out_status) return BT_ERR_INVALID_ARG;
  bt::Handle& h = H->h;
  EntryGuard g(H);
  // searches alone never conflict: run the search kernel directly on the batch
  cudaError_t e = bt::tree_join(&h, S(stream));
  if (e != cudaSuccess) return BT_ERR_CUDA;
  if (h.descent == BT_DESCENT_LEARNED && h.L.valid)
    e = bt::launch_learned_lookup(&h, keys, nullptr, nullptr, n, out_vals, out_status, S(stream));
  else
    e = bt::launch_search(&h, keys, nullptr, nullptr, n, out_vals, out_status, S(stream));
  return e == cudaSuccess ? BT_OK : BT_ERR_CUDA;
}

int bt_range_batch(bt_handle* H, const uint64_t* lo, const uint64_t* hi, size_t n, uint32_t max_per,
                   uint64_t* out_keys, uint64_t* out_vals, uint32_t* out_counts, void* stream) {
  if (!H) return BT_ERR_INVALID_ARG;
  if (n == 0) return BT_OK;
  if (!lo || !hi || !out_counts || (max_per && (!out_keys || !out_vals))) return BT_ERR_INVALID_ARG;
  EntryGuard g(H);
  if (bt::tree_join(&H->h, S(stream)) != cudaSuccess) return BT_ERR_CUDA;
  return bt::launch_range(&H->h, lo, hi, n, max_per, out_keys, out_vals, out_counts, S(stream)) == cudaSuccess
             ? BT_OK
             : BT_ERR_CUDA;
}

int bt_insert_batch(bt_handle* H, const uint64_t* keys, const uint64_t* vals, uint64_t* out_vals,
                    uint8_t* out_status, size_t n, void* stream) {
  if (!H) return BT_ERR_INVALID_ARG;
  if (n == 0) return BT_OK;
  if (!keys || !vals || !out_vals || !out_status) return BT_ERR_INVALID_ARG;
  bt::Handle& h = H->h;
  if (n > h.w.cap) return BT_ERR_BATCH_TOO_LARGE;
  EntryGuard g(H);
  // an all-insert op array
  if (cudaMemsetAsync(h.w.ins_ops, BT_OP_INSERT, n, S(stream)) != cudaSuccess) return BT_ERR_CUDA;
  return map_internal(bt::batch_sorted(&h, keys, vals, h.w.ins_ops, out_vals, out_status, n, 0, S(stream)));
}

int bt_size(bt_handle* H, uint64_t* n_keys) {
  if (!H || !n_keys) return BT_ERR_INVALID_ARG;
  EntryGuard g(H);
  bt::Ctrl c;
  if (bt::tree_sync(&H->h) != cudaSuccess) return BT_ERR_CUDA;
  if (cudaMemcpy(&c, H->h.tree.ctrl, sizeof(c), cudaMemcpyDeviceToHost) != cudaSuccess) return BT_ERR_CUDA;
  *n_keys = c.n_keys;
  return BT_OK;
}

int bt_dump_sorted(bt_handle* H, uint64_t* keys, uint64_t* vals, size_t cap, size_t* n_out, void* stream) {
  if (!H || !n_out) return BT_ERR_INVALID_ARG;
  EntryGuard g(H);
  cudaStream_t s = stream ? S(stream) : H->h.internal_stream;
  if (stream == nullptr) cudaDeviceSynchronize();
  if (bt::tree_join(&H->h, s) != cudaSuccess) return BT_ERR_CUDA;
  return map_internal(bt::tree_dump(&H->h, keys, vals, cap, n_out, s));
}

int bt_leaf_sizes(bt_handle* H, uint32_t* sizes_host, size_t cap, size_t* n_leaves) {
  if (!H || !n_leaves) return BT_ERR_INVALID_ARG;
  EntryGuard g(H);
  cudaDeviceSynchronize();
  bt::Handle& h = H->h;
  uint32_t* leaves = nullptr;
  size_t nl = 0;
  int rc = bt::enumerate_leaves(&h, h.internal_stream, &leaves, &nl);
  if (rc) return map_internal(rc);
  *n_leaves = nl;
  if (!sizes_host || nl == 0) return BT_OK;
  uint32_t* sizes = (leaves == h.enum_a) ? h.enum_b : h.enum_a;
  if (bt::leaf_sizes_device(&h, leaves, nl, sizes, h.internal_stream) != cudaSuccess) return BT_ERR_CUDA;
  const size_t m = nl < cap ? nl : cap;
  if (cudaMemcpyAsync(sizes_host, sizes, m * 4, cudaMemcpyDeviceToHost, h.internal_stream) != cudaSuccess)
    return BT_ERR_CUDA;
  return cudaStreamSynchronize(h.internal_stream) == cudaSuccess ? BT_OK : BT_ERR_CUDA;
}

int bt_level_counts(bt_handle* H, uint64_t* counts_host, uint32_t cap, uint32_t* height) {
  if (!H || !height) return BT_ERR_INVALID_ARG;
  EntryGuard g(H);
  cudaDeviceSynchronize();
  uint32_t* leaves = nullptr;
  size_t nl = 0;
  int rc = bt::enumerate_leaves(&H->h, H->h.internal_stream, &leaves, &nl);
  if (rc) return map_internal(rc);
  *height = H->h.n_levels;
  if (counts_host)
    for (uint32_t i = 0; i < cap; i++) counts_host[i] = (i < H->h.n_levels && i < 48) ? H->h.level_counts[i] : 0;
  return BT_OK;
}

int bt_stats_get(bt_handle* H, bt_stats* st, int with_leaves) {
  if (!H || !st) return BT_ERR_INVALID_ARG;
  EntryGuard g(H);
  cudaDeviceSynchronize();
  bt::Ctrl c;
  if (cudaMemcpy(&c, H->h.tree.ctrl, sizeof(c), cudaMemcpyDeviceToHost) != cudaSuccess) return BT_ERR_CUDA;
  std::memset(st, 0, sizeof(*st));
  st->n_keys = c.n_keys;
  st->n_nodes = c.n_nodes < H->h.tree.cap ? c.n_nodes : H->h.tree.cap;
  st->height = c.root == bt::kNil ? 0 : c.root_level + 1;
  st->error = c.error;
  st->commits = c.commits;
  st->aborts = c.aborts;
  st->leaf_splits = c.leaf_splits;
  st->inner_splits = c.inner_splits;
  st->new_roots = c.new_roots;
  st->retry_exhausted = c.retry_exhausted;
  st->learned_hits = c.learned_hits;
  st->learned_fallbacks = c.learned_fallbacks;
  st->learned_probe_sum = c.learned_probe_sum;
  st->capacity_nodes = H->h.tree.cap;
  if (with_leaves) {
    uint32_t* leaves = nullptr;
    size_t nl = 0;
    int rc = bt::enumerate_leaves(&H->h, H->h.internal_stream, &leaves, &nl);
    if (rc) return map_internal(rc);
    st->n_leaves = nl;
  }
  return BT_OK;
}

int bt_stats_reset(bt_handle* H) {
  if (!H) return BT_ERR_INVALID_ARG;
  EntryGuard g(H);
  cudaDeviceSynchronize();
  bt::Ctrl c;
  if (cudaMemcpy(&c, H->h.tree.ctrl, sizeof(c), cudaMemcpyDeviceToHost) != cudaSuccess) return BT_ERR_CUDA;
  c.commits = c.aborts = c.leaf_splits = c.inner_splits = c.new_roots = c.retry_exhausted = 0;
  c.learned_hits = c.learned_fallbacks = c.learned_probe_sum = 0;
  c.error = 0;
  return cudaMemcpy(H->h.tree.ctrl, &c, sizeof(c), cudaMemcpyHostToDevice) == cudaSuccess ? BT_OK : BT_ERR_CUDA;
}

int bt_retrain(bt_handle* H, void* stream) {
  if (!H) return BT_ERR_INVALID_ARG;
  EntryGuard g(H);
  cudaStream_t s = stream ? S(stream) : H->h.internal_stream;
  if (stream == nullptr) cudaDeviceSynchronize();
  if (bt::tree_join(&H->h, s) != cudaSuccess) return BT_ERR_CUDA;
  return map_internal(bt::learned_retrain(&H->h, s));
}

int bt_refit(bt_handle* H, void* stream) {
  if (!H) return BT_ERR_INVALID_ARG;
  if (!H->h.L.trained) return BT_ERR_NOT_TRAINED;
  EntryGuard g(H);
  cudaStream_t s = stream ? S(stream) : H->h.internal_stream;
  if (stream == nullptr) cudaDeviceSynchronize();
  if (bt::tree_join(&H->h, s) != cudaSuccess) return BT_ERR_CUDA;
  const int rc = map_internal(bt::learned_retrain(&H->h, s, true));
  if (rc == BT_OK && stream == nullptr && cudaStreamSynchronize(s) != cudaSuccess) return BT_ERR_CUDA;
  return rc;
}

int bt_set_descent(bt_handle* H, int descent) {
  if (!H || (descent != BT_DESCENT_PLAIN && descent != BT_DESCENT_LEARNED)) return BT_ERR_INVALID_ARG;
  if (descent == BT_DESCENT_LEARNED && !H->h.L.valid) return BT_ERR_NOT_TRAINED;
  H->h.descent = descent;
  return BT_OK;
}

int bt_set_root_model(bt_handle* H, int mlp) {
  if (!H) return BT_ERR_INVALID_ARG;
  H->h.L.stage1 = mlp ? 1 : 0;
  return BT_OK;
}

int bt_set_search_group(bt_handle* H, uint32_t lanes) {
  if (!H) return BT_ERR_INVALID_ARG;
  if (lanes != 4 && lanes != 8 && lanes != 16 && lanes != 32) return BT_ERR_INVALID_ARG;
  H->h.search_group = (int)lanes;
  return BT_OK;
}

int bt_profile(bt_handle* H, int enable) {
  if (!H) return BT_ERR_INVALID_ARG;
  EntryGuard g(H);
  int rc = prof_resolve(H->h);
  H->h.prof = enable != 0;
  return rc;
}

int bt_profile_read(bt_handle* H, double* phase_ms, uint64_t* batches, int reset) {
  if (!H) return BT_ERR_INVALID_ARG;
  EntryGuard g(H);
  int rc = prof_resolve(H->h);
  if (rc != BT_OK) return rc;
  if (phase_ms)
    for (int p = 0; p < bt::kNumPhases; p++) phase_ms[p] = H->h.phase_ms[p];
  if (batches) *batches = H->h.phase_batches;
  if (reset) {
    for (int p = 0; p < bt::kNumPhases; p++) H->h.phase_ms[p] = 0;
    H->h.phase_batches = 0;
  }
  return BT_OK;
}

int bt_sync(bt_handle* H, void* stream) {
  if (!H) return BT_ERR_INVALID_ARG;
  EntryGuard g(H);
  const cudaError_t e = stream ? bt::tree_join(&H->h, S(stream)) : bt::tree_sync(&H->h);
  return e == cudaSuccess ? BT_OK : BT_ERR_CUDA;
}

uint64_t bt_launch_count(void) { return bt::g_launches.load(); }

int bt_set_option(bt_handle* H, int option, int64_t value) {
  if (!H) return BT_ERR_INVALID_ARG;
  switch (option) {
    case BT_OPT_SORTED_SEARCH: H->h.sorted_search = value ? 1 : 0; return BT_OK;
    case BT_OPT_SORTED_LEAF_VALS: H->h.sorted_leaf_vals = value ? 1 : 0; return BT_OK;
    case BT_OPT_FRONT_END: H->h.front_end = value ? 1 : 0; return BT_OK;
    case BT_OPT_ASYNC_WRITE: H->h.async_write = value ? 1 : 0; return BT_OK;
    case BT_OPT_TOP_CACHE: H->h.top_cache = value ? 1 : 0; return BT_OK;
    case BT_OPT_OVERLAP:
      // 0 off; 1 on (default reserve); > 1 on, leaving value - 1 lookup block slots for the side stream
      if (value < 0) return BT_ERR_INVALID_ARG;
      H->h.overlap = value ? 1 : 0;
      if (value > 1) H->h.overlap_reserve = (int)(value - 1);
      return BT_OK;
    case BT_OPT_SEARCH_PAIRS:
      if (value < 0 || value > 2) return BT_ERR_INVALID_ARG;
      H->h.search_pairs = (int)value;
      return BT_OK;
    case BT_OPT_BATCH_DESCENT:
      if (value < -1 || value > 1) return BT_ERR_INVALID_ARG;
      H->h.batch_descent = (int)value;
      return BT_OK;
    case BT_OPT_RETRY_LIMIT:
      if (value < 1 || value > 0x7fffffff) return BT_ERR_INVALID_ARG;
      H->h.retry_limit = (uint32_t)value;
      return BT_OK;
    case BT_OPT_TRAIN_STEPS:
      if (value < 0 || value > 1000000) return BT_ERR_INVALID_ARG;
      H->h.L.train_steps = (uint32_t)value;
      return BT_OK;
    case BT_OPT_REFIT_STEPS:
      if (value < 0 || value > 1000000) return BT_ERR_INVALID_ARG;
      H->h.L.refit_steps = (uint32_t)value;
      return BT_OK;
    case BT_OPT_SORT_TILE:
      if (value != 256 && value != 512 && value != 1024) return BT_ERR_INVALID_ARG;
      H->h.sort_threads = H->h.sort_threads_touch = (int)value;
      return BT_OK;
    case BT_OPT_HOST_VALUES_IN_PLACE:
      H->h.host_vals_in_place = value ? 1 : 0;
      return BT_OK;
    case BT_OPT_STM_COMBINE:
      H->h.stm_combine = value ? 1 : 0;
      return BT_OK;
    case BT_OPT_HOST_FRONT_OVERLAP:
      H->h.host_front_overlap = value ? 1 : 0;
      return BT_OK;
    case BT_OPT_TOUCH_SORT:
      if (value < 0 || value > 2) return BT_ERR_INVALID_ARG;
      H->h.touch_sort = (int)value;
      return BT_OK;
    case BT_OPT_LEARNED_POLICY:
      if (value < 0 || value > 2) return BT_ERR_INVALID_ARG;
      H->h.L.policy = (int)value;
      H->h.L.stale = false;
      return BT_OK;
    case BT_OPT_LEARNED_MODE:
      if (value < 1 || value > 3) return BT_ERR_INVALID_ARG;
      H->h.learned_mode = (int)value;
      return BT_OK;
    default: return BT_ERR_INVALID_ARG;
  }
}

int bt_autotune(bt_handle* H, const uint64_t* sample_keys, size_t n, void* stream, double* report) {
  if (!H || !sample_keys || n == 0) return BT_ERR_INVALID_ARG;
  EntryGuard g(H);
  cudaStream_t s = stream ? S(stream) : H->h.internal_stream;
  if (stream == nullptr) cudaDeviceSynchronize();
  if (bt::tree_join(&H->h, s) != cudaSuccess) return BT_ERR_CUDA;
  return map_internal(bt::autotune(&H->h, sample_keys, n, s, report));
}

// Node fill: a temporary handle per candidate fill holds a sample tree built
// from the caller's keys; a sorted 95/5 batch of the same size (half of its
// searches for sample keys, inserts of fresh keys) is timed on it, and the
// handle keeps the fill of the fastest for its later bulk builds and splits.
int bt_autotune_fill(bt_handle* H, const uint64_t* sample_keys, size_t n, void* stream, double* report) {
  if (!H || !sample_keys || n < 64) return BT_ERR_INVALID_ARG;
  EntryGuard g(H);
  cudaStream_t s = S(stream);
  if (cudaStreamSynchronize(s) != cudaSuccess || bt::tree_sync(&H->h) != cudaSuccess) return BT_ERR_CUDA;
  const uint32_t fills[4] = {16, 20, 24, 28};
  double out[8] = {};
  uint64_t *rk = nullptr, *rv = nullptr, *ov = nullptr;
  uint8_t *ro = nullptr, *os = nullptr;
  const size_t nb = 2;  // timed batches
  bool ok = cudaMalloc(&rk, nb * n * 8) == cudaSuccess && cudaMalloc(&rv, nb * n * 8) == cudaSuccess &&
            cudaMalloc(&ro, nb * n) == cudaSuccess && cudaMalloc(&ov, n * 8) == cudaSuccess &&
            cudaMalloc(&os, n) == cudaSuccess;
  // 95/5 batches shaped like the sample (uniform fresh keys would all land
  // beyond the range of a skewed sample, in its two edge leaves)
  for (size_t b = 0; ok && b < nb; b++)
    ok = bt::gen_sample_requests(0xF111u + b, sample_keys, n, n, 95, rk + b * n, rv + b * n, ro + b * n, s) ==
         cudaSuccess;
  double best = 1e30;
  uint32_t best_fill = H->h.leaf_fill;
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  ok = ok && cudaEventCreate(&e0) == cudaSuccess && cudaEventCreate(&e1) == cudaSuccess;
  for (int i = 0; ok && i < 4; i++) {
    bt_config c;
    bt_config_init(&c);
    c.device = H->h.device;
    c.max_keys = 3 * n;
    c.max_batch = n;
    c.leaf_fill = c.inner_fill = fills[i];
    bt_handle* T = nullptr;
    if (bt_create(&c, &T) != BT_OK) {
      ok = false;
      break;
    }
    const int mode = BT_MODE_SORTED | BT_MODE_MERGE_ENGINE;
    bool run = bt_bulk_build(T, sample_keys, sample_keys, n, s) == BT_OK;
    // one untimed batch (first touch of the buffers), then the timed ones on a fresh build
    run = run && bt_execute_batch(T, rk, rv, ro, ov, os, n, mode, s) == BT_OK && bt_sync(T, s) == BT_OK;
    run = run && bt_bulk_build(T, sample_keys, sample_keys, n, s) == BT_OK;
    run = run && cudaEventRecord(e0, s) == cudaSuccess;
    for (size_t b = 0; run && b < nb; b++)
      run = bt_execute_batch(T, rk + b * n, rv + b * n, ro + b * n, ov, os, n, mode, s) == BT_OK;
    run = run && bt_sync(T, s) == BT_OK && cudaEventRecord(e1, s) == cudaSuccess && cudaEventSynchronize(e1) == cudaSuccess;
    float ms = 0;
    run = run && cudaEventElapsedTime(&ms, e0, e1) == cudaSuccess;
    bt_destroy(T);
    if (!run) {
      ok = false;
      break;
    }
    out[2 + i] = ms / nb;
    if (ms < best) {
      best = ms;
      best_fill = fills[i];
    }
  }
  if (e0) cudaEventDestroy(e0);
  if (e1) cudaEventDestroy(e1);
  cudaFree(rk);
  cudaFree(rv);
  cudaFree(ro);
  cudaFree(ov);
  cudaFree(os);
  if (!ok) return BT_ERR_CUDA;
  H->h.leaf_fill = H->h.inner_fill = best_fill;
  out[0] = out[1] = best_fill;
  if (report)
    for (int i = 0; i < 8; i++) report[i] = out[i];
  return BT_OK;
}

int bt_set_learned_group(bt_handle* H, uint32_t lanes) {
  if (!H) return BT_ERR_INVALID_ARG;
  if (lanes != 2 && lanes != 4 && lanes != 8 && lanes != 16 && lanes != 32) return BT_ERR_INVALID_ARG;
  H->h.learned_group = (int)lanes;
  return BT_OK;
}

int bt_learned_info(bt_handle* H, double* info) {
  if (!H || !info) return BT_ERR_INVALID_ARG;
  EntryGuard g(H);
  const bt::Learned& L = H->h.L;
  // the last (re)training's loss and segment count arrive in page-locked host words
  if (cudaDeviceSynchronize() != cudaSuccess) return BT_ERR_CUDA;
  float loss = 0.f;
  uint32_t bad = 0;
  if (L.host_words) {
    std::memcpy(&loss, &L.host_words[0], 4);
    bad = L.host_words[1];
  }
  info[0] = L.valid ? 1.0 : 0.0;
  info[1] = (double)L.n_leaves;
  info[2] = (double)L.n_segments;
  info[3] = (double)bad;
  info[4] = (double)L.window;
  info[5] = (double)loss;
  info[6] = (double)L.stage1;
  info[7] = (double)L.train_steps;
  return BT_OK;
}

int bt_mlp_grad(bt_handle* H, const float* params, const float* x, const float* y, size_t n, float* grad_out,
                float* loss_out, void* stream) {
  if (!H || !params || !x || !y || !grad_out || !loss_out || n == 0) return BT_ERR_INVALID_ARG;
  EntryGuard g(H);
  return map_internal(bt::learned_mlp_grad(&H->h, params, x, y, n, grad_out, loss_out, S(stream)));
}

int bt_host_alloc(void** p, size_t bytes) {
  if (!p) return BT_ERR_INVALID_ARG;
  return cudaMallocHost(p, bytes ? bytes : 1) == cudaSuccess ? BT_OK : BT_ERR_NO_MEMORY;
}

int bt_host_free(void* p) { return cudaFreeHost(p) == cudaSuccess ? BT_OK : BT_ERR_CUDA; }

int bt_route_batch(bt_handle* H, const uint64_t* splitters, int n_shards, const uint64_t* keys, const uint64_t* vals,
                   const uint8_t* ops, size_t n, uint64_t* out_keys, uint64_t* out_vals, uint8_t* out_ops,
                   uint32_t* out_perm, uint64_t* out_counts, void* stream) {
  if (!H || n_shards < 1 || n_shards > BT_MAX_SHARDS || !out_counts) return BT_ERR_INVALID_ARG;
  if (n_shards > 1 && !splitters) return BT_ERR_INVALID_ARG;
  if (n && (!keys || !out_keys || !out_perm || (vals && !out_vals) || (ops && !out_ops))) return BT_ERR_INVALID_ARG;
  if (n > 0xFFFFFFFFull) return BT_ERR_BATCH_TOO_LARGE;  // 32-bit permutation
  EntryGuard g(H);
  return bt::route_batch(&H->h, splitters, n_shards, keys, vals, ops, n, out_keys, out_vals, out_ops, out_perm,
                         out_counts, S(stream));
}

int bt_unroute_results(bt_handle* H, const uint32_t* perm, const uint64_t* in_vals, const uint8_t* in_status,
                       size_t n, uint64_t* out_vals, uint8_t* out_status, void* stream) {
  if (!H) return BT_ERR_INVALID_ARG;
  if (n == 0) return BT_OK;
  if (!perm || !in_vals || !in_status || !out_vals || !out_status) return BT_ERR_INVALID_ARG;
  EntryGuard g(H);
  return bt::unroute_results(&H->h, perm, in_vals, in_status, n, out_vals, out_status, S(stream));
}

const char* bt_status_string(int code) {
  switch (code) {
    case BT_OK: return "ok";
    case BT_ERR_INVALID_ARG: return "invalid argument";
    case BT_ERR_CUDA: return "CUDA error";
    case BT_ERR_NO_MEMORY: return "out of memory";
    case BT_ERR_CAPACITY: return "node pool exhausted";
    case BT_ERR_RESERVED_KEY: return "reserved key UINT64_MAX";
    case BT_ERR_BATCH_TOO_LARGE: return "batch larger than max_batch";
    case BT_ERR_NOT_TRAINED: return "learned predictor not trained";
    case BT_ERR_STATIC_LIMIT: return "more keys than BT_STATIC_BUILD_MAX_KEYS";
    case BT_ERR_BUSY: return "no free slot or arena space";
    case BT_ERR_TIMEOUT: return "timed out";
    case BT_ERR_IO: return "snapshot file error";
    default: return "unknown status";
  }
}

}  // extern "C"
