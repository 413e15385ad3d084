// Serving loop: continuous batching of request batches against one tree.
// No counterpart in the reference (one host thread runs batches one after the
// other, src/gpu-stm-tree-v39/bpt-gpustm.cpp:78-105).
//
//   bt_submit   admits a batch when a ring slot and enough arena bytes are
//               free (otherwise BT_ERR_BUSY), copies its requests into the
//               device arena on a copy stream, resets the slot's counters,
//               publishes its descriptor and bumps the device tail;
//   device      serve_kernel (bt_stm.cu): a persistent, graph-launched kernel
//               whose warps claim chunks of the oldest batch with work, so a
//               batch that arrives while others run overlaps with them;
//   completion  the warp finishing a batch writes its sequence number to
//               mapped host memory; the host then copies the answers out on a
//               second stream and retires slots and arena space in order.
// The kernel exits after idle_us without work; any host call that finds work
// in flight and the kernel gone relaunches the graph.  Everything on the copy
// stream is a copy (the slot counters are reset from a pinned zero word, not
// by a memset kernel): the persistent kernel holds the SMs, so a kernel queued
// on the copy stream would not start until blocks of it idle out, and a batch
// would not be published before that.
#include <algorithm>
#include <chrono>
#include <cstring>
#include <mutex>
#include <thread>
#include <vector>

#include <cuda_runtime.h>

#include "../../include/eirene_b200.h"
#include "bt_common.cuh"
#include "bt_internal.h"

namespace {

double now_ms() {
  return std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now().time_since_epoch()).count();
}
size_t up256(size_t x) { return (x + 255) & ~size_t(255); }

struct Slot {
  int state = 0;  // 0 free, 1 on the device, 2 copying answers out, 3 done (awaiting in-order retirement)
  uint32_t seq = 0;
  size_t n = 0;
  uint64_t* out_vals = nullptr;
  uint8_t* out_st = nullptr;
  size_t a_off = 0, a_len = 0;
  cudaEvent_t out_ev = nullptr;
  double t_submit = 0;
};

}  // namespace

struct bt_server {
  bt_handle* H = nullptr;
  int device = 0;
  cudaStream_t s_in = nullptr, s_out = nullptr, s_k = nullptr;
  char* arena = nullptr;
  size_t arena_bytes = 0;
  bt::ServeDesc* d_desc = nullptr;
  uint32_t* d_tail = nullptr;
  uint32_t* d_cursor = nullptr;
  unsigned long long* d_claimed = nullptr;
  uint32_t* d_done = nullptr;
  uint32_t* d_stop = nullptr;
  uint32_t* h_done = nullptr;  // mapped
  unsigned long long* h_tend = nullptr;
  unsigned long long* h_tclaim = nullptr;  // mapped: device clock of each batch's first claim
  uint32_t policy = 0;
  bt::ServeDesc* st_desc = nullptr;  // pinned staging (outlives the async copies)
  uint32_t* st_tail = nullptr;
  unsigned long long* st_claim = nullptr;
  uint32_t* st_stop = nullptr;
  uint32_t* st_zero = nullptr;  // pinned zero word: counters are reset by the copy engine
  uint32_t cap = 0;
  std::vector<Slot> slots;
  uint32_t next_seq = 0, retire_seq = 0;
  size_t a_head = 0, a_tail = 0;
  uint32_t live = 0;
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
  cudaEvent_t k_ev = nullptr;
  bool k_launched = false;
  unsigned long long launches = 0;
  std::vector<double> lat_ms;
  std::vector<double> svc_ms;
  unsigned long long dev_t0 = ~0ull, dev_t1 = 0;  // earliest first claim, latest completion (device clock)
  unsigned long long completed = 0, requests = 0;
  double t_first = -1, t_last = 0;
  std::mutex mu;
};

namespace {

// contiguous ring allocation in submission order; freed in the same order
bool ring_alloc(bt_server* S, size_t len, size_t* off) {
  if (S->live == 0) S->a_head = S->a_tail = 0;
  if (len > S->arena_bytes) return false;
  if (S->live == 0 || S->a_tail > S->a_head) {
    if (S->arena_bytes - S->a_tail >= len) {
      *off = S->a_tail;
      S->a_tail += len;
      return true;
    }
    if (S->a_head > len || (S->live == 0 && S->arena_bytes >= len)) {
      *off = 0;
      S->a_tail = len;
      return true;
    }
    return false;
  }
  if (S->a_tail < S->a_head && S->a_head - S->a_tail >= len) {
    *off = S->a_tail;
    S->a_tail += len;
    return true;
  }
  return false;
}

int ensure_kernel(bt_server* S) {
  bool running = S->k_launched && cudaEventQuery(S->k_ev) == cudaErrorNotReady;
  if (running) return BT_OK;
  if (cudaGraphLaunch(S->exec, S->s_k) != cudaSuccess) return BT_ERR_CUDA;
  bt::count_launch();
  if (cudaEventRecord(S->k_ev, S->s_k) != cudaSuccess) return BT_ERR_CUDA;
  S->k_launched = true;
  S->launches++;
  return BT_OK;
}

int pump(bt_server* S) {
  bool on_device = false;
  for (uint32_t q = S->retire_seq; q != S->next_seq; q++) {
    Slot& sl = S->slots[q % S->cap];
    if (sl.state == 1) {
      const uint32_t d = *reinterpret_cast<volatile uint32_t*>(S->h_done + (q % S->cap));
      if (d == q) {
        char* base = S->arena + sl.a_off;
        const size_t n = sl.n;
        char* outv = base + up256(n * 8) * 2;
        char* outs = outv + up256(n * 8) + up256(n);
        if (cudaMemcpyAsync(sl.out_vals, outv, n * 8, cudaMemcpyDeviceToHost, S->s_out) != cudaSuccess ||
            cudaMemcpyAsync(sl.out_st, outs, n, cudaMemcpyDeviceToHost, S->s_out) != cudaSuccess ||
            cudaEventRecord(sl.out_ev, S->s_out) != cudaSuccess)
          return BT_ERR_CUDA;
        sl.state = 2;
      } else {
        on_device = true;
      }
    }
    if (sl.state == 2 && cudaEventQuery(sl.out_ev) == cudaSuccess) {
      sl.state = 3;
      const double t = now_ms();
      S->lat_ms.push_back(t - sl.t_submit);
      const volatile unsigned long long* te = S->h_tend + (q % S->cap);
      const volatile unsigned long long* tc = S->h_tclaim + (q % S->cap);
      const unsigned long long tev = *te, tcv = *tc;
      if (tev >= tcv) {
        S->svc_ms.push_back((double)(tev - tcv) * 1e-6);
        S->dev_t0 = std::min(S->dev_t0, tcv);
        S->dev_t1 = std::max(S->dev_t1, tev);
      }
      S->completed++;
      S->requests += sl.n;
      S->t_last = t;
    }
  }
  while (S->retire_seq != S->next_seq && S->slots[S->retire_seq % S->cap].state == 3) {
    Slot& sl = S->slots[S->retire_seq % S->cap];
    sl.state = 0;
    S->live--;
    S->retire_seq++;
    if (S->live == 0) S->a_head = S->a_tail = 0;
    else S->a_head = S->slots[S->retire_seq % S->cap].a_off;
  }
  if (on_device) return ensure_kernel(S);
  return BT_OK;
}

}  // namespace

extern "C" {

int bt_serve_config_init(bt_serve_config* c) {
  if (!c) return BT_ERR_INVALID_ARG;
  std::memset(c, 0, sizeof(*c));
  c->arena_bytes = 1ull << 30;
  c->max_batches = 256;
  c->idle_us = 2000;
  c->policy = 0;
  return BT_OK;
}

int bt_serve_start(bt_handle* H, const bt_serve_config* cfg_in, bt_server** out) {
  if (!H || !out) return BT_ERR_INVALID_ARG;
  *out = nullptr;
  bt_serve_config cfg;
  if (cfg_in) cfg = *cfg_in;
  else bt_serve_config_init(&cfg);
  if (cfg.max_batches < 2 || cfg.max_batches > 65536 || cfg.arena_bytes < 4096 || cfg.policy > 1)
    return BT_ERR_INVALID_ARG;
  int prev = -1;
  cudaGetDevice(&prev);
  if (cudaSetDevice(H->h.device) != cudaSuccess) return BT_ERR_CUDA;
  H->h.chain_open = false;
  bt_server* S = new bt_server();
  S->H = H;
  S->device = H->h.device;
  S->cap = cfg.max_batches;
  S->arena_bytes = cfg.arena_bytes;
  S->slots.resize(S->cap);
  S->policy = cfg.policy;
  bool ok = cudaStreamCreateWithFlags(&S->s_in, cudaStreamNonBlocking) == cudaSuccess &&
            cudaStreamCreateWithFlags(&S->s_out, cudaStreamNonBlocking) == cudaSuccess &&
            cudaStreamCreateWithFlags(&S->s_k, cudaStreamNonBlocking) == cudaSuccess &&
            cudaMalloc(&S->arena, S->arena_bytes) == cudaSuccess &&
            cudaMalloc(&S->d_desc, S->cap * sizeof(bt::ServeDesc)) == cudaSuccess &&
            cudaMalloc(&S->d_tail, 256) == cudaSuccess &&
            cudaMalloc(&S->d_claimed, S->cap * sizeof(unsigned long long)) == cudaSuccess &&
            cudaMalloc(&S->d_done, S->cap * 4) == cudaSuccess &&
            cudaHostAlloc(&S->h_done, S->cap * 4, cudaHostAllocMapped) == cudaSuccess &&
            cudaHostAlloc(&S->h_tend, S->cap * 8, cudaHostAllocMapped) == cudaSuccess &&
            cudaHostAlloc(&S->h_tclaim, S->cap * 8, cudaHostAllocMapped) == cudaSuccess &&
            cudaMallocHost(&S->st_desc, S->cap * sizeof(bt::ServeDesc)) == cudaSuccess &&
            cudaMallocHost(&S->st_tail, S->cap * 4) == cudaSuccess &&
            cudaMallocHost(&S->st_claim, S->cap * 8) == cudaSuccess &&
            cudaMallocHost(&S->st_stop, 64) == cudaSuccess &&
            cudaMallocHost(&S->st_zero, 64) == cudaSuccess &&
            cudaEventCreateWithFlags(&S->k_ev, cudaEventDisableTiming) == cudaSuccess;
  for (uint32_t i = 0; ok && i < S->cap; i++)
    ok = cudaEventCreateWithFlags(&S->slots[i].out_ev, cudaEventDisableTiming) == cudaSuccess;
  if (ok) {
    S->d_cursor = S->d_tail + 16;
    S->d_stop = S->d_tail + 32;
    std::memset(S->h_done, 0xFF, S->cap * 4);
    std::memset(S->h_tclaim, 0, S->cap * 8);
    std::memset(S->h_tend, 0, S->cap * 8);
    std::memset(S->st_zero, 0, 64);
    ok = cudaMemset(S->d_tail, 0, 256) == cudaSuccess &&
         cudaMemset(S->d_claimed, 0xFF, S->cap * sizeof(unsigned long long)) == cudaSuccess &&
         cudaMemset(S->d_done, 0, S->cap * 4) == cudaSuccess;
  }
  uint32_t* h_done_dev = nullptr;
  unsigned long long* h_tend_dev = nullptr;
  unsigned long long* h_tclaim_dev = nullptr;
  ok = ok && cudaHostGetDevicePointer((void**)&h_done_dev, S->h_done, 0) == cudaSuccess &&
       cudaHostGetDevicePointer((void**)&h_tend_dev, S->h_tend, 0) == cudaSuccess &&
       cudaHostGetDevicePointer((void**)&h_tclaim_dev, S->h_tclaim, 0) == cudaSuccess;
  if (ok) {
    bt::ServeDev D;
    D.desc = S->d_desc;
    D.tail = S->d_tail;
    D.cursor = S->d_cursor;
    D.claimed = S->d_claimed;
    D.done = S->d_done;
    D.stop = S->d_stop;
    D.host_done = h_done_dev;
    D.host_tend = h_tend_dev;
    D.host_tclaim = h_tclaim_dev;
    D.policy = S->policy;
    D.cap = S->cap;
    D.idle_ns = (unsigned long long)(cfg.idle_us ? cfg.idle_us : 2000) * 1000ull;
    D.last_busy = reinterpret_cast<unsigned long long*>(S->d_tail + 48);
    D.exiting = S->d_tail + 56;
    // the persistent kernel, captured once and relaunched as a graph; the
    // graph first clears the exit flag the previous launch left set
    ok = cudaStreamBeginCapture(S->s_k, cudaStreamCaptureModeThreadLocal) == cudaSuccess;
    if (ok) {
      cudaMemsetAsync(D.exiting, 0, 4, S->s_k);
      bt::launch_serve(&H->h, D, S->s_k);
      ok = cudaStreamEndCapture(S->s_k, &S->graph) == cudaSuccess;
    }
    ok = ok && cudaGraphInstantiate(&S->exec, S->graph, 0) == cudaSuccess;
  }
  ok = ok && cudaDeviceSynchronize() == cudaSuccess;
  if (prev >= 0) cudaSetDevice(prev);
  if (!ok) {
    bt_serve_stop(S);
    return BT_ERR_NO_MEMORY;
  }
  *out = S;
  return BT_OK;
}

int bt_submit(bt_server* S, const uint64_t* keys, const uint64_t* vals, const uint8_t* ops, size_t n,
              uint64_t* out_vals, uint8_t* out_status, uint64_t* ticket) {
  if (!S || !keys || !vals || !ops || !out_vals || !out_status || !ticket || n == 0 || n > 0xFFFFFFFFull)
    return BT_ERR_INVALID_ARG;
  std::lock_guard<std::mutex> lk(S->mu);
  int prev = -1;
  cudaGetDevice(&prev);
  if (prev != S->device) cudaSetDevice(S->device);
  int rc = pump(S);
  const size_t len = up256(n * 8) * 3 + up256(n) * 2;
  const uint32_t seq = S->next_seq;
  Slot& sl = S->slots[seq % S->cap];
  size_t off = 0;
  if (rc == BT_OK && len > S->arena_bytes) rc = BT_ERR_BATCH_TOO_LARGE;
  else if (rc == BT_OK && (sl.state != 0 || !ring_alloc(S, len, &off))) rc = BT_ERR_BUSY;
  if (rc == BT_OK) {
    char* base = S->arena + off;
    uint64_t* dk = reinterpret_cast<uint64_t*>(base);
    uint64_t* dv = reinterpret_cast<uint64_t*>(base + up256(n * 8));
    uint64_t* dov = reinterpret_cast<uint64_t*>(base + up256(n * 8) * 2);
    uint8_t* dops = reinterpret_cast<uint8_t*>(base + up256(n * 8) * 3);
    uint8_t* dos = dops + up256(n);
    const uint32_t slot = seq % S->cap;
    S->st_claim[slot] = (unsigned long long)seq << 32;
    bt::ServeDesc& d = S->st_desc[slot];
    d.keys = dk;
    d.vals = dv;
    d.ops = dops;
    d.out_vals = dov;
    d.out_st = dos;
    d.n = (uint32_t)n;
    d.seq = seq;
    S->st_tail[slot] = seq + 1;
    bool ok = cudaMemcpyAsync(dk, keys, n * 8, cudaMemcpyHostToDevice, S->s_in) == cudaSuccess &&
              cudaMemcpyAsync(dv, vals, n * 8, cudaMemcpyHostToDevice, S->s_in) == cudaSuccess &&
              cudaMemcpyAsync(dops, ops, n, cudaMemcpyHostToDevice, S->s_in) == cudaSuccess &&
              cudaMemcpyAsync(S->d_claimed + slot, &S->st_claim[slot], 8, cudaMemcpyHostToDevice, S->s_in) ==
                  cudaSuccess &&
              cudaMemcpyAsync(S->d_done + slot, S->st_zero, 4, cudaMemcpyHostToDevice, S->s_in) == cudaSuccess &&
              cudaMemcpyAsync(S->d_desc + slot, &d, sizeof(d), cudaMemcpyHostToDevice, S->s_in) == cudaSuccess &&
              cudaMemcpyAsync(S->d_tail, &S->st_tail[slot], 4, cudaMemcpyHostToDevice, S->s_in) == cudaSuccess;
    if (!ok) {
      rc = BT_ERR_CUDA;
    } else {
      sl.state = 1;
      sl.seq = seq;
      sl.n = n;
      sl.out_vals = out_vals;
      sl.out_st = out_status;
      sl.a_off = off;
      sl.a_len = len;
      sl.t_submit = now_ms();
      if (S->t_first < 0) S->t_first = sl.t_submit;
      S->live++;
      S->next_seq++;
      *ticket = seq;
      rc = ensure_kernel(S);
    }
  }
  if (prev >= 0 && prev != S->device) cudaSetDevice(prev);
  return rc;
}

int bt_poll(bt_server* S, uint64_t ticket, int* done) {
  if (!S || !done) return BT_ERR_INVALID_ARG;
  std::lock_guard<std::mutex> lk(S->mu);
  int prev = -1;
  cudaGetDevice(&prev);
  if (prev != S->device) cudaSetDevice(S->device);
  const int rc = pump(S);
  // tickets are batch sequence numbers (at most 2^32 batches per server)
  if (ticket >= S->next_seq) *done = -1;
  else if (ticket < S->retire_seq) *done = 1;
  else *done = S->slots[(uint32_t)ticket % S->cap].state == 3 ? 1 : 0;
  if (prev >= 0 && prev != S->device) cudaSetDevice(prev);
  return rc;
}

int bt_wait(bt_server* S, uint64_t ticket, uint32_t timeout_ms) {
  const double t0 = now_ms();
  for (;;) {
    int done = 0;
    const int rc = bt_poll(S, ticket, &done);
    if (rc != BT_OK) return rc;
    if (done < 0) return BT_ERR_INVALID_ARG;
    if (done) return BT_OK;
    if (timeout_ms && now_ms() - t0 > timeout_ms) return BT_ERR_TIMEOUT;
    std::this_thread::sleep_for(std::chrono::microseconds(10));
  }
}

int bt_serve_batch_times(bt_server* S, uint64_t ticket, uint64_t* first_claim_ns, uint64_t* done_ns) {
  if (!S || !first_claim_ns || !done_ns) return BT_ERR_INVALID_ARG;
  std::lock_guard<std::mutex> lk(S->mu);
  // finished, and its slot not reused since
  if (ticket >= S->next_seq || ticket + S->cap < S->next_seq) return BT_ERR_INVALID_ARG;
  const uint32_t q = (uint32_t)ticket;
  if (q >= S->retire_seq && S->slots[q % S->cap].state != 3) return BT_ERR_INVALID_ARG;
  *first_claim_ns = *reinterpret_cast<volatile unsigned long long*>(S->h_tclaim + q % S->cap);
  *done_ns = *reinterpret_cast<volatile unsigned long long*>(S->h_tend + q % S->cap);
  return BT_OK;
}

int bt_serve_get_stats(bt_server* S, bt_serve_stats* st, int reset) {
  if (!S || !st) return BT_ERR_INVALID_ARG;
  std::lock_guard<std::mutex> lk(S->mu);
  std::memset(st, 0, sizeof(*st));
  st->batches = S->completed;
  st->requests = S->requests;
  st->kernel_launches = S->launches;
  st->in_flight = S->next_seq - S->retire_seq;
  if (!S->lat_ms.empty()) {
    std::vector<double> v = S->lat_ms;
    std::sort(v.begin(), v.end());
    auto pct = [&](double p) { return v[std::min(v.size() - 1, (size_t)(p * (v.size() - 1) + 0.5))]; };
    st->p50_ms = pct(0.50);
    st->p99_ms = pct(0.99);
    st->max_ms = v.back();
    double s = 0;
    for (double x : v) s += x;
    st->mean_ms = s / v.size();
  }
  if (!S->svc_ms.empty()) {
    std::vector<double> v = S->svc_ms;
    std::sort(v.begin(), v.end());
    st->p50_service_ms = v[std::min(v.size() - 1, (size_t)(0.50 * (v.size() - 1) + 0.5))];
    st->p99_service_ms = v[std::min(v.size() - 1, (size_t)(0.99 * (v.size() - 1) + 0.5))];
  }
  if (S->t_first >= 0 && S->t_last > S->t_first) st->mops = S->requests / ((S->t_last - S->t_first) * 1e3);
  if (S->dev_t1 > S->dev_t0) st->device_mops = (double)S->requests / ((double)(S->dev_t1 - S->dev_t0) * 1e-3);
  if (reset) {
    S->lat_ms.clear();
    S->svc_ms.clear();
    S->dev_t0 = ~0ull;
    S->dev_t1 = 0;
    S->completed = S->requests = 0;
    S->t_first = -1;
    S->t_last = 0;
    S->launches = 0;
  }
  return BT_OK;
}

int bt_serve_stop(bt_server* S) {
  if (!S) return BT_ERR_INVALID_ARG;
  int prev = -1;
  cudaGetDevice(&prev);
  cudaSetDevice(S->device);
  // drain what is in flight (bounded), then stop the kernel
  for (uint32_t q = S->retire_seq; q != S->next_seq; q++) bt_wait(S, q, 60000);
  if (S->st_stop && S->d_stop) {
    *S->st_stop = 1;
    cudaMemcpyAsync(S->d_stop, S->st_stop, 4, cudaMemcpyHostToDevice, S->s_in);
  }
  cudaDeviceSynchronize();
  for (auto& sl : S->slots)
    if (sl.out_ev) cudaEventDestroy(sl.out_ev);
  if (S->exec) cudaGraphExecDestroy(S->exec);
  if (S->graph) cudaGraphDestroy(S->graph);
  if (S->k_ev) cudaEventDestroy(S->k_ev);
  cudaFree(S->arena);
  cudaFree(S->d_desc);
  cudaFree(S->d_tail);
  cudaFree(S->d_claimed);
  cudaFree(S->d_done);
  if (S->h_done) cudaFreeHost(S->h_done);
  if (S->h_tend) cudaFreeHost(S->h_tend);
  if (S->h_tclaim) cudaFreeHost(S->h_tclaim);
  if (S->st_desc) cudaFreeHost(S->st_desc);
  if (S->st_tail) cudaFreeHost(S->st_tail);
  if (S->st_claim) cudaFreeHost(S->st_claim);
  if (S->st_stop) cudaFreeHost(S->st_stop);
  if (S->st_zero) cudaFreeHost(S->st_zero);
  if (S->s_in) cudaStreamDestroy(S->s_in);
  if (S->s_out) cudaStreamDestroy(S->s_out);
  if (S->s_k) cudaStreamDestroy(S->s_k);
  delete S;
  if (prev >= 0) cudaSetDevice(prev);
  return BT_OK;
}

}  // extern "C"
