// Host-side internals shared by the CUDA translation units of libeirene_b200.
#pragma once
#include <atomic>
#include <cstddef>
#include <cstdint>
#include <vector>

#include <cuda_runtime.h>

#include "bt_common.cuh"

namespace bt {

// process-wide count of kernels launched by this library (reported by the bench)
extern std::atomic<unsigned long long> g_launches;
inline void count_launch(unsigned n = 1) { g_launches.fetch_add(n, std::memory_order_relaxed); }

// phases timed with CUDA events when profiling is on (the reference's
// Time_Measure phases, src/gpu-stm-tree-v38/bpt-gpustm-kernel.cu:289-324)
enum Phase { kPhSort = 0, kPhMerge, kPhSearch, kPhInsert, kPhWriteback, kNumPhases };
// boundary events per batch: 0..kNumPhases in order, plus three for the
// other layouts (end of the touched sort on the side stream, end of the
// lookups on the main stream, start of the write-back before the leaf merge)
constexpr int kProfEvents = kNumPhases + 4;
constexpr int kEvSortEnd = kNumPhases + 1, kEvLookupEnd = kNumPhases + 2, kEvWbStart = kNumPhases + 3;
// per-batch event layout bits (prof_resolve)
constexpr int kLayoutOverlap = 1;  // sort and merge passes on the side stream, beside the lookups
constexpr int kLayoutEarly = 2;    // answers written back before the leaf merge

// ---- scan / sort (bt_sort.cu) ----
// layout of the radix sort's scratch: kSortMaxPasses digit histograms of
// kSortRadix counters, 64 tile counters, and one look-back table of
// kSortRadix words per pass and tile of kSortTileKeys keys
// (sort_scratch_words computes the same; bt_sort.cu checks the constants)
constexpr size_t kSortTileKeys = 2048;  // the smallest tile: scratch for every tile size
constexpr size_t kSortMaxPasses = 8;
constexpr size_t kSortRadix = 256;
constexpr size_t sort_scratch_words_for(size_t n) {
  return kSortMaxPasses * kSortRadix + 64 + kSortMaxPasses * ((n ? n : 1) + kSortTileKeys - 1) / kSortTileKeys * kSortRadix;
}
size_t scan_scratch_words(size_t n);
cudaError_t scan_exclusive_u32(const uint32_t* in, uint32_t* out, size_t n, uint32_t* total_dev, uint32_t* scratch,
                               cudaStream_t s,
                               const uint32_t* n_dev = nullptr);
// one-launch scan with decoupled look-back (status: scan_lb_words(n_upper)
// words; ctr: two words, zero before the first call; *epoch: the caller's
// call counter)
size_t scan_lb_words(size_t n_upper);
cudaError_t scan_exclusive_u32_lb(const uint32_t* in, uint32_t* out, size_t n_upper, const uint32_t* n_dev,
                                  uint32_t* total_dev, uint64_t* status, uint32_t* ctr, uint32_t* epoch,
                                  uint32_t* err, cudaStream_t s);
cudaError_t sort_prepare();
size_t sort_scratch_words(size_t n);
// tile_threads: 256, 512 or 1024 threads per onesweep tile of 8 items each
cudaError_t radix_sort_pairs(const uint64_t* keys_in, const uint32_t* vals_in, const uint8_t* ops, uint64_t* k_a,
                             uint32_t* v_a, uint64_t* k_b, uint32_t* v_b, size_t n, int begin_bit, int end_bit,
                             uint32_t* scratch, cudaStream_t s, uint64_t** k_out, uint32_t** v_out, uint32_t* err,
                             const uint32_t* n_dev = nullptr, int tile_threads = 512);

// Stable sort by key of (key, payload) pairs whose payload carries the
// request index in its low 30 bits, indices increasing in input order (the
// hash front end's touched requests): tile sort plus merge rounds; the
// result is always in (k_a, v_a).  n is the capacity, n_dev the count.
// touched counts up to which BT_OPT_TOUCH_SORT 2 takes the merge sort
// (2^18 touched requests: 92 against 126 us for the radix sort; the merge
// rounds grow with the count, the radix passes with its bytes)
constexpr uint32_t kMergeSortMax = 1u << 19;
cudaError_t merge_sort_pairs(const uint64_t* keys_in, const uint32_t* vals_in, uint64_t* k_a, uint32_t* v_a,
                             uint64_t* k_b, uint32_t* v_b, size_t n, const uint32_t* n_dev, int sm_count,
                             cudaStream_t s, uint64_t** k_out, uint32_t** v_out);

// ---- per-batch work buffers, sized for max_batch requests ----
struct BatchCounts {
  uint32_t n_unique;
  uint32_t n_ins;
  uint32_t n_get;
  uint32_t n_del;
  // hash front end (bt_front.cu)
  uint32_t n_ins_req;  // INSERT requests with a valid key
  uint32_t cap;        // hash table slots this batch (power of two)
  uint32_t n_touch;    // requests resolved through the sorted path
  uint32_t n_lookup;   // requests answered by a plain lookup
};

constexpr int kTopNodes = 256;  // nodes of the shared-memory top cache (384 B each)
struct TopInfo {
  uint32_t n_nodes;
  uint32_t n_levels;     // cached levels below and including the root (0: no cache)
  uint32_t below_level;  // level of the nodes the last cached level points to
  uint32_t pad;
};

struct TileSummary;  // bt_batch.cu

// The buffers the front part and the tree part of a hash-front-end batch
// share, and the merge passes' tile summaries, which either part may run
// (bt_batch.cu): a second set lets bt_execute_batches and the host batches
// run one batch's front part beside the previous batch's tree part.  Work's
// own fields hold the set in use; `alt` the other.
struct BatchSet {
  TileSummary* tiles = nullptr;
  BatchCounts* counts = nullptr;
  uint32_t* f_list = nullptr;
  uint64_t* f_lk = nullptr;
  uint64_t* ukeys = nullptr;
  uint64_t* uvals = nullptr;
  uint32_t* ins_list = nullptr;
  uint32_t* get_list = nullptr;
  uint32_t* del_list = nullptr;
  uint32_t* pend = nullptr;
  uint64_t* k_a = nullptr;
  uint64_t* k_b = nullptr;
  uint32_t* v_a = nullptr;
  uint32_t* v_b = nullptr;
};

struct Work {
  size_t cap = 0;  // requests
  uint64_t* k_a = nullptr;
  uint64_t* k_b = nullptr;
  uint32_t* v_a = nullptr;
  uint32_t* v_b = nullptr;
  uint32_t* sort_scratch = nullptr;
  uint64_t* ukeys = nullptr;
  uint64_t* uvals = nullptr;
  uint64_t* uans = nullptr;
  uint8_t* uans_st = nullptr;
  uint32_t* ins_list = nullptr;
  uint32_t* get_list = nullptr;
  uint32_t* del_list = nullptr;
  uint32_t* pend = nullptr;
  TileSummary* tiles = nullptr;
  uint64_t* tile_carry = nullptr;  // scratch for the tile pass
  BatchCounts* counts = nullptr;
  // segmented leaf merge (bt_merge.cu)
  uint32_t* m_path = nullptr;   // [cap][8] root-to-leaf path of each unique insert
  uint64_t* m_vpos = nullptr;   // [cap] value slot (node * 32 + slot) of an existing key, or ~0
  uint32_t* m_leaf = nullptr;
  uint32_t* m_isnew = nullptr;
  uint32_t* m_pos = nullptr;
  uint64_t* m_newk = nullptr;
  uint64_t* m_newv = nullptr;
  uint32_t* m_nq = nullptr;
  uint32_t* m_nleaf = nullptr;
  uint32_t* m_seg = nullptr;
  // delete phase (bt_delete.cu): leaf and slot of each unique DELETE key,
  // apart from the merge scratch so the two locates can run back to back
  uint32_t* d_leaf = nullptr;
  uint32_t* d_slot = nullptr;
  void* m_ent_a = nullptr;      // separator entries, 16 B each
  void* m_ent_b = nullptr;
  void* m_counts = nullptr;
  void* m_sync = nullptr;       // grid barrier + per-block partials of the inner merge
  // hash front end (bt_front.cu)
  void* f_tab = nullptr;         // 16 B slots
  size_t f_tab_cap = 0;          // slots allocated (power of two)
  uint32_t* f_flags = nullptr;   // [cap] words; the flag pass uses them as one "touched" byte per request
  uint32_t* f_pos = nullptr;     // [cap] per-tile touched counts, then the tiles' exclusive offsets
  uint32_t* f_list = nullptr;    // [cap] requests for the plain lookup, in input order
  uint64_t* f_lk = nullptr;      // [cap] their keys, in the same order
  uint64_t* f_tk = nullptr;      // [cap] keys of the touched requests, in input order
  uint32_t* f_tv = nullptr;      // [cap] index | op << 30 of the touched requests
  // all-INSERT op codes of bt_insert_batch
  uint8_t* ins_ops = nullptr;
  // look-back scan of the merge engine (scan_exclusive_u32_lb)
  uint64_t* lb_status = nullptr;
  uint32_t* lb_ctr = nullptr;
  uint32_t lb_epoch = 0;
  BatchSet alt;        // the second set (allocated by the first bt_execute_batches)
  bool alt_in = false; // Work's fields hold the second set
};
int work_alt_alloc(Work* w);
void work_swap_set(Work* w);  // exchange the fields' set with `alt`

// ---- host-buffer entry points (bt_api.cu) ----
// Three staging sets: batch i + 1's inputs are copied in and batch i - 1's
// answers copied out while batch i's kernels run.  With two, batch i + 1
// could be submitted only once batch i - 1's answers were out, so its copy-in
// started late in batch i's kernels and the GPU waited for it.
constexpr int kStagingSets = 3;
struct Staging {
  uint64_t* keys = nullptr;
  uint64_t* vals = nullptr;
  uint8_t* ops = nullptr;
  uint64_t* out_vals = nullptr;
  uint8_t* out_st = nullptr;
  uint64_t* packed = nullptr;  // packed INSERT values (allocated at the first packed batch)
  uint32_t* pack_scratch = nullptr;
  uint32_t* pack_err = nullptr;  // page-locked copy of the batch's count-mismatch flag
  bool packed_batch = false;     // the set's batch came with packed values
  cudaEvent_t in_ev = nullptr;    // keys and op codes are on the device
  cudaEvent_t vals_ev = nullptr;  // values are on the device
  cudaEvent_t ans_ev = nullptr;   // every answer is final in out_vals / out_st
  cudaEvent_t done_ev = nullptr;  // the answers are in host memory: the set is free
  uint64_t ticket = 0;            // the batch that last used the set (0: none)
};
struct HostPipe {
  size_t cap = 0;
  Staging set[kStagingSets];
  cudaStream_t in_stream = nullptr, out_stream = nullptr;
  uint64_t issued = 0;  // tickets handed out so far
  std::vector<uint64_t> refused;  // packed batches whose value count did not match (answered kRejected)
};

// ---- learned leaf predictor state (bt_learned.cu) ----
struct Learned {
  bool valid = false;
  uint32_t n_leaves = 0;
  uint32_t n_segments = 0;  // segments of the current model
  uint32_t seg_config = 0;  // segments asked for; 0: chosen at each full training (learned_retrain)
  uint32_t window = 64;
  uint64_t* leaf_low = nullptr;  // [n_leaves + 1] (sentinel at the end)
  uint32_t* leaf_id = nullptr;   // [n_leaves]
  size_t leaf_cap = 0;
  float* mlp = nullptr;          // 97 params
  float* mlp_grad = nullptr;     // 97 floats (device gradient buffer)
  double* seg = nullptr;         // SegParam[n_segments], 16 B each (bt_learned.cuh)
  uint32_t* seg_scratch = nullptr;
  uint32_t* seg_of = nullptr;    // [leaf_cap] segment of each leaf (training scratch)
  size_t seg_cap = 0;
  uint64_t kmin = 0, kmax = 0;
  int stage1 = 1;  // 1 = MLP root model, 0 = linear root model
  uint32_t train_steps = 300;
  uint32_t refit_steps = 0;  // warm-started Adam steps of stage 1 per refit
  uint32_t train_batch = 16384;
  float lr = 0.05f;
  bool trained = false;      // stage 1 and its key normalisation hold a full training
  uint64_t refits = 0;
  // page-locked host words written by the device after a (re)training:
  // [0] final training loss (float), [1] segments over the window
  uint32_t* host_words = nullptr;
  // requests the learned lookup leaves to the plain descent, and their count
  uint32_t* miss = nullptr;
  uint32_t* n_miss = nullptr;
  uint64_t* miss_keys = nullptr;  // their keys, compacted beside them
  size_t miss_cap = 0;
  // adaptive use (BT_OPT_LEARNED_POLICY): the device gate (LearnedGate,
  // bt_learned.cuh), and for policy 2 its stale word sampled into
  // page-locked memory on a side stream, read by a later batch once done
  int policy = 1;                       // 0 always, 1 plain once stale, 2 and refit
  struct LearnedGate* gate = nullptr;
  bool stale = false;                   // the sampled gate was closed
  uint32_t batches = 0;                 // batches since the last fit
  uint32_t* sample = nullptr;           // page-locked gate word
  bool pending = false;
  cudaEvent_t sample_ev = nullptr, lookups_ev = nullptr;
  cudaStream_t sample_stream = nullptr;
};

struct Handle {
  int device = 0;
  DevTree tree{};
  uint32_t leaf_fill = 24;
  uint32_t inner_fill = 24;
  uint32_t retry_limit = 1u << 16;
  int descent = 0;     // 0 plain, 1 learned
  uint32_t epoch = 0;  // tree epoch, bumped by every reset / bulk build
  int search_group = 4;  // lanes per request in the lock-free search
  int learned_group = 4;  // lanes per request in the learned search
  int learned_mode = 3;   // unsorted learned lookup: 1 one request per lane group, 2 two in lock step,
                          // 3 software-pipelined (up to five requests per group in successive rounds)
  int sorted_search = 1;  // batch GET phase: 1 = path-reusing search over the sorted keys
  int sorted_leaf_vals = 0;  // sorted search: load the leaf's values with its keys (1) or only the match (0)
  int sort_threads = 512;        // radix sort tile (x 8 items) for whole-batch sorts
  int sort_threads_touch = 512;  // ... for the hash front end's sort of the touched requests
  int batch_descent = -1;    // autotuned choice for the batch GET phase: -1 = follow `descent`
  int front_end = 1;         // sorted batches: 1 = hash front end (sort only INSERT-coupled requests), 0 = full sort
  int top_cache = 1;         // unsorted searches descend the upper levels from shared memory
  int search_pairs = 2;      // unsorted searches: 2 pairs of requests per lane group, child ids only; 1 pairs; 0 single
  bool pfx_valid = false;    // tree.pfx matches every inner row (false after bulk builds and STM writers)
  int use_pfx = 1;           // paired searches compare the separators' 32-bit prefixes first
  void* top = nullptr;       // top cache (kTopNodes nodes) + TopInfo
  TopInfo* top_info = nullptr;
  int sm_count = 148;
  Work w;
  Learned L;
  uint32_t* enum_a = nullptr;  // leaf enumeration buffers (node ids)
  uint32_t* enum_b = nullptr;
  uint32_t* enum_cnt = nullptr;
  uint32_t* enum_scan_scratch = nullptr;
  size_t enum_cap = 0;
  uint64_t level_counts[48] = {};  // filled by enumerate_leaves, leaf level first
  uint32_t n_levels = 0;
  cudaStream_t internal_stream = nullptr;
  // profiling: one event per phase boundary per batch, resolved on read
  bool prof = false;
  std::vector<cudaEvent_t> prof_ev;  // kProfEvents events per recorded batch
  std::vector<char> prof_layout;     // per recorded batch: kLayout* bits (see prof_resolve)
  size_t prof_batches = 0;
  // hash front end: the merge engine's locates and grouping (and, while the
  // values are still being copied in, the merge passes) run on a
  // high-priority side stream while the lookups run on the caller's stream
  cudaStream_t hi_stream = nullptr;
  cudaEvent_t fork_ev = nullptr, join_ev = nullptr;
  int overlap = 1;
  int lookup_reserve = 0;    // block slots the overlapped lookups leave free (set per batch)
  // bt_execute_batches and the host-buffer entry points: the front parts'
  // stream and its events
  cudaStream_t front_stream = nullptr;
  cudaEvent_t front_done[2] = {nullptr, nullptr}, tree_done[2] = {nullptr, nullptr};
  cudaEvent_t pipe_ev = nullptr;
  // host batches (batch_chained): the point of the caller's stream before
  // the last such batch's tree part, and whether no other call used the
  // handle since (the next front part may then start there)
  cudaEvent_t chain_gate = nullptr;
  bool chain_open = false;
  int chain_set = 0;
  int host_front_overlap = 1;  // BT_OPT_HOST_FRONT_OVERLAP
  // BT_OPT_TOUCH_SORT: 0 onesweep radix sort, 1 tile sort + merge rounds, 2 the
  // second while the touched count last seen (touch_hint, page-locked and
  // mapped, written by front_tile_scan_kernel) is at most kMergeSortMax
  int touch_sort = 2;
  uint32_t* touch_hint = nullptr;
  uint32_t* touch_hint_dev = nullptr;
  int overlap_reserve = 4;  // ... in the overlapped layout (measured, per 2^22 batch on 2^26 keys: 4 < 8 < 16 < 32 ms, 1.3 % from 4 to 16)
  // host-buffer entry points: staging sets and copy streams
  HostPipe hp;
  int stm_combine = 1;         // BT_MODE_STM batches combine the INSERTs of a key (BT_OPT_STM_COMBINE)
  int host_vals_in_place = 0;  // sorted host batches read page-locked values over the bus instead of copying
  // per-batch hooks of the sorted batch, set by the host-buffer entry points:
  // the stream that first reads `vals` waits for vals_wait; vals_remote says
  // that `vals` is page-locked host memory read over the bus (the merge
  // passes then run beside the lookups as when they wait for a copy);
  // ans_ready is recorded once every answer is in the output arrays
  cudaEvent_t vals_wait = nullptr;
  bool vals_remote = false;
  cudaEvent_t ans_ready = nullptr;
  // deferred write phase: a sorted batch (hash front end, merge engine)
  // completes on the caller's stream once its answers are final and leaves
  // the leaf/inner merge on tree_stream; tree_ev marks its end.  Every later
  // access to the tree or the merge scratch waits for tree_ev first
  // (tree_join on a stream, tree_sync on the host).
  cudaStream_t tree_stream = nullptr;
  cudaEvent_t tree_ev = nullptr;
  cudaEvent_t ans_ev = nullptr;
  bool tree_pending = false;
  int async_write = 1;
  double phase_ms[kNumPhases] = {};
  unsigned long long phase_batches = 0;
  unsigned long long phase_items[kNumPhases] = {};
};

// make stream `s` wait for the deferred write phase (no-op when none is pending)
cudaError_t tree_join(Handle* h, cudaStream_t s);
// block the host until the deferred write phase has finished
cudaError_t tree_sync(Handle* h);

// record the boundary event `which` (0..kProfEvents-1) of the current batch;
// event kNumPhases closes the batch, so the extra events come before it
void prof_mark(Handle* h, int which, cudaStream_t s);
void prof_set_layout(Handle* h, int layout);

// ---- tree kernels (bt_tree.cu) ----
// make tree.pfx match every inner row (a rebuild when stale), stream ordered
cudaError_t ensure_pfx(Handle* h, cudaStream_t s);
cudaError_t tree_reset(Handle* h, cudaStream_t s);
// header word of node rows [first, last) set to 0 (epoch 0: never written)
cudaError_t clear_headers(Handle* h, uint32_t first, uint32_t last, cudaStream_t s);
int tree_bulk_build(Handle* h, const uint64_t* keys, const uint64_t* vals, size_t n, cudaStream_t s);
// caller-provided scratch for the bulk build (used by the no-allocation entry point)
struct BuildScratch {
  uint64_t* ka;
  uint64_t* kb;
  uint32_t* va;
  uint32_t* vb;
  uint32_t* sort_scratch;  // sort_scratch_words(cap) words (>= scan_scratch_words(cap))
  uint32_t* pos;
  uint64_t* uv;
  uint32_t* tot;  // one word
  size_t cap;     // keys
};
int tree_bulk_build_scratch(Handle* h, const uint64_t* keys, const uint64_t* vals, size_t n, cudaStream_t s,
                            const BuildScratch& sc);
// ckeys (nullable): the keys of the listed requests compacted, ckeys[q] =
// qkeys[list[q]], read instead of the indirection where the kernel supports it
cudaError_t launch_search(Handle* h, const uint64_t* qkeys, const uint32_t* list, const uint32_t* n_dev, size_t n,
                          uint64_t* out_vals, uint8_t* out_st, cudaStream_t s, const uint64_t* ckeys = nullptr);
// range scan, one warp per query (bt_range_batch)
cudaError_t launch_range(Handle* h, const uint64_t* lo, const uint64_t* hi, size_t n, uint32_t max_per,
                         uint64_t* out_keys, uint64_t* out_vals, uint32_t* out_counts, cudaStream_t s);
// the same search with the tree's upper levels cached in shared memory
cudaError_t launch_search_top(Handle* h, const uint64_t* qkeys, const uint32_t* list, const uint32_t* n_dev,
                              size_t n, uint64_t* out_vals, uint8_t* out_st, cudaStream_t s);
// search over keys in ascending order (path reuse); needs root_level < 8
cudaError_t launch_search_sorted(Handle* h, const uint64_t* qkeys, const uint32_t* list, const uint32_t* n_dev,
                                 size_t n, uint64_t* out_vals, uint8_t* out_st, cudaStream_t s);
// ids of the leaves in key order; returns count (synchronises the stream)
int enumerate_leaves(Handle* h, cudaStream_t s, uint32_t** leaf_ids, size_t* n_leaves);
// leaf sizes in key order into a device buffer (after enumerate_leaves)
cudaError_t leaf_sizes_device(Handle* h, const uint32_t* leaves, size_t n, uint32_t* out, cudaStream_t s);
int tree_dump(Handle* h, uint64_t* out_keys, uint64_t* out_vals, size_t cap, size_t* n_out, cudaStream_t s);

// ---- serving loop (bt_stm.cu device side, bt_serve.cu host side) ----
constexpr int kServeChunk = 32;
constexpr int kServeWindow = 32;  // batches a warp considers under the fewest-unclaimed policy
struct ServeDesc {
  const uint64_t* keys;
  const uint64_t* vals;
  const uint8_t* ops;
  uint64_t* out_vals;
  uint8_t* out_st;
  uint32_t n;
  uint32_t seq;
};
struct ServeDev {
  const ServeDesc* desc;  // [cap]
  const uint32_t* tail;   // batches published
  uint32_t* cursor;       // oldest batch with unclaimed requests
  unsigned long long* claimed;  // [cap] per slot: batch seq << 32 | requests claimed
  uint32_t* done;         // [cap] requests finished per slot
  const uint32_t* stop;
  uint32_t* host_done;              // [cap] mapped host memory: seq of the finished batch
  unsigned long long* host_tend;    // [cap] mapped host memory: device clock at completion
  unsigned long long* host_tclaim;  // [cap] mapped host memory: device clock of the batch's first claim
  uint32_t cap;
  uint32_t policy;                  // 0 oldest batch first, 1 fewest unclaimed requests first
  unsigned long long idle_ns;
  unsigned long long* last_busy;  // device clock of the latest claim of work by any warp
  uint32_t* exiting;              // set by the warp that sees the idle timeout: every warp leaves
};
cudaError_t launch_serve(Handle* h, const ServeDev& S, cudaStream_t s);

// ---- STM kernels (bt_stm.cu) ----
cudaError_t launch_stm(Handle* h, const uint64_t* keys, const uint64_t* vals, const uint8_t* ops, uint8_t op_override,
                       const uint32_t* list, const uint32_t* n_dev, size_t n, uint64_t* out_vals, uint8_t* out_st,
                       cudaStream_t s, const uint8_t* skip = nullptr);

// ---- delete phase of the sorted batch (bt_delete.cu) ----
// locate: reads the tree only (answers the DELETE runs); apply: removes the keys
int delete_locate(Handle* h, size_t n_upper, cudaStream_t s);
int delete_apply(Handle* h, size_t n_upper, cudaStream_t s);

// ---- workload generators (bt_workload.cu) ----
// requests shaped like a key sample of any law (the node-fill tuner's batches)
cudaError_t gen_sample_requests(uint64_t seed, const uint64_t* sample, size_t n_sample, size_t n, uint32_t search_pct,
                                uint64_t* keys, uint64_t* vals, uint8_t* ops, cudaStream_t s);

// ---- hash front end of the sorted batch (bt_front.cu) ----
int front_classify(Handle* h, const uint64_t* keys, const uint8_t* ops, size_t n, cudaStream_t s);
// a whole BT_MODE_STM batch: its GETs first, by the lookup kernels, then its
// writes as STM transactions (bt_stm.cu)
int batch_stm(Handle* h, const uint64_t* keys, const uint64_t* vals, const uint8_t* ops, uint64_t* out_vals,
              uint8_t* out_st, size_t n, cudaStream_t s);
// BT_MODE_STM batch, split: the valid GETs to w.get_list (keys compacted in
// w.ukeys, count counts->n_lookup), every other request to w.ins_list
// (count counts->n_ins_req)
int stm_split(Handle* h, const uint64_t* keys, const uint8_t* ops, size_t n, cudaStream_t s);
// INSERT combining over the write list of stm_split: answers the INSERTs combined with
// an earlier one of their key and returns, per INSERT, a skip byte (1: answered
// already) and the value the STM kernel stores (in the front end's buffers);
// stm_combine_fixup after the kernel gives a chain the status of its
// representative when that did not commit
int stm_combine(Handle* h, const uint64_t* keys, const uint64_t* vals, const uint8_t* ops, size_t n,
                uint64_t* out_vals, uint8_t* out_st, cudaStream_t s, const uint8_t** skip, const uint64_t** cvals);
int stm_combine_fixup(Handle* h, const uint8_t* ops, size_t n, uint64_t* out_vals, uint8_t* out_st, cudaStream_t s);
// packed INSERT values (scratch sized by pack_scratch_words(n_cap), n <= n_cap):
// pack_check counts the INSERTs of ops per tile and, when their total is not
// n_packed, raises the word at pack_error_word and makes every op code
// invalid (the batch is then answered kRejected and applies nothing);
// pack_expand then puts packed[j], the value of the j-th INSERT in request
// order, at vals[r] of that INSERT's request r (other slots untouched:
// nothing reads them)
size_t pack_scratch_words(size_t n_cap);
uint32_t* pack_error_word(uint32_t* scratch, size_t n_cap);
cudaError_t pack_check(uint8_t* ops, size_t n, size_t n_packed, uint32_t* scratch, size_t n_cap, int sm_count,
                       cudaStream_t s);
cudaError_t pack_expand(const uint8_t* ops, size_t n, const uint64_t* packed, size_t n_packed, uint64_t* vals,
                        const uint32_t* scratch, size_t n_cap, cudaStream_t s);

// ---- key-range sharding (bt_shard.cu) ----
int route_batch(Handle* h, const uint64_t* splitters, int n_shards, const uint64_t* keys, const uint64_t* vals,
                const uint8_t* ops, size_t n, uint64_t* out_keys, uint64_t* out_vals, uint8_t* out_ops,
                uint32_t* out_perm, uint64_t* out_counts, cudaStream_t s);
int unroute_results(Handle* h, const uint32_t* perm, const uint64_t* in_vals, const uint8_t* in_st, size_t n,
                    uint64_t* out_vals, uint8_t* out_st, cudaStream_t s);

// ---- sorted-merge batch (bt_batch.cu) ----
int work_alloc(Work* w, size_t cap);
void work_free(Work* w);
int batch_sorted(Handle* h, const uint64_t* keys, const uint64_t* vals, const uint8_t* ops, uint64_t* out_vals,
                 uint8_t* out_st, size_t n, int engine, cudaStream_t s);
// several hash-front-end batches whose inputs are all ready on `s`: batch
// j + 1's front part beside batch j's tree part (bt_batch.cu)
int batches_pipelined(Handle* h, size_t count, const uint64_t* const* keys, const uint64_t* const* vals,
                      const uint8_t* const* ops, uint64_t* const* out_vals, uint8_t* const* out_st, const size_t* n,
                      int engine, cudaStream_t s);
// One hash-front-end batch of the host-buffer entry points, its op codes
// and keys ready at `in_ready` and its values at `vals_ready` (events of the
// copy-in stream; the merge passes wait for the values, and run in the tree
// part when `vals_late`): the front part on
// front_stream, the tree part on `s`, with buffer sets alternating from one
// such batch to the next.  While chain_open, the front part starts at
// chain_gate, beside the previous such batch's tree part; otherwise after
// everything queued on `s`.
int batch_chained(Handle* h, const uint64_t* keys, const uint64_t* vals, const uint8_t* ops, uint64_t* out_vals,
                  uint8_t* out_st, size_t n, int engine, cudaStream_t s, cudaEvent_t in_ready,
                  cudaEvent_t vals_ready, bool vals_late);

// ---- segmented leaf merge (bt_merge.cu) ----
int merge_engine(Handle* h, size_t n_upper, cudaStream_t s);
// the same in five parts:
//   locate   descents of the pre-batch tree, answers of the INSERT runs
//            (reads the tree only);
//   update   new values of the existing keys, in place (after the batch's
//            plain lookups, before its DELETE apply);
//   group    the new keys and their runs per leaf (no tree access);
//   reserve  pieces per touched leaf (reads leaf sizes: after the DELETE
//            apply), node reservation, kNoCapacity answers when it fails;
//   write    leaf merge and inner levels: reads only the merge scratch
//            (m_*), so the next batch's front end and sort may run beside it.
int merge_locate_phase(Handle* h, cudaStream_t s);
int merge_update_phase(Handle* h, size_t n_upper, cudaStream_t s);
int merge_group_phase(Handle* h, size_t n_upper, cudaStream_t s);
int merge_reserve_phase(Handle* h, size_t n_upper, cudaStream_t s);
int merge_write_phase(Handle* h, cudaStream_t s);

// device view of the learned model when the learned descent is on and trained
struct LearnedDev;
int learned_dev(Handle* h, LearnedDev* out);

// ---- autotuner (bt_tune.cu) ----
constexpr int kTuneReport = 24;  // doubles in bt_autotune's report (BT_AUTOTUNE_REPORT_LEN)
int autotune(Handle* h, const uint64_t* keys, size_t n, cudaStream_t s, double* rep);

// ---- learned predictor (bt_learned.cu) ----
int learned_retrain(Handle* h, cudaStream_t s, bool refit = false);
void learned_free(Learned* L);
// whether a batch's lookups use the learned descent (the handle's choice,
// then the adaptive policy; policy 2 may refit here), and the counter sample
// to take after them
bool batch_learned(Handle* h, int desc, cudaStream_t s);
void learned_sample(Handle* h, cudaStream_t s);
void learned_policy_free(Learned* L);
cudaError_t launch_learned_search(Handle* h, const uint64_t* qkeys, const uint32_t* list, const uint32_t* n_dev,
                                  size_t n, uint64_t* out_vals, uint8_t* out_st, cudaStream_t s, bool sorted);
// unsorted learned lookups (paired groups, misses deferred to a plain descent
// over a miss list); n <= max_batch when list or n_dev is given
cudaError_t launch_learned_lookup(Handle* h, const uint64_t* qkeys, const uint32_t* list, const uint32_t* n_dev,
                                  size_t n, uint64_t* out_vals, uint8_t* out_st, cudaStream_t s,
                                  const uint64_t* ckeys = nullptr, bool gated = false);
int learned_mlp_grad(Handle* h, const float* params, const float* x, const float* y, size_t n, float* grad_out,
                     float* loss_out, cudaStream_t s);

}  // namespace bt

// the opaque handle of the C ABI
struct bt_handle {
  bt::Handle h;
};
