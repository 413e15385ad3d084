/*
 * eirene_b200 -- C ABI of the B200 batched B+tree (bulk build, batched point
 * search, batched insert under warp-level STM, sort-based batch merge,
 * learned leaf predictor).
 *
 * The reference exposes this path as the C++ virtual class GPU_BTree
 * (src/tree.h:28-43) implemented by gpu_stm_nsp_39::GPU_STM_Tree and
 * gpu_stm_nsp_38::GPU_STM_Tree; there is no C ABI in the reference.  Each entry
 * point below names the reference member it replaces (paths are relative to
 * the reference project root).
 *
 * Conventions
 *   - Keys and values are uint64.  Key UINT64_MAX is reserved (the reference
 *     reserves INT_MAX as MAX_KEY, src/gpu-stm-tree-v39/bpt-gpustm.h:20).
 *   - Unless an entry point says "host", every pointer is a device pointer and
 *     the caller owns the buffer.  `stream` is a cudaStream_t (NULL = legacy
 *     default stream); calls are stream ordered and return before the work
 *     finishes unless documented as synchronous.
 *   - Every entry point returns BT_OK (0) or a negative BT_ERR_* code and
 *     never exits the process (the reference prints and calls exit(1),
 *     src/cuda_utils.h:3-12).  No C++ exception crosses this boundary.
 *   - A handle is not thread-safe; use one handle per host thread or lock.
 */
#ifndef EIRENE_B200_H
#define EIRENE_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes ---- */
#define BT_OK 0
#define BT_ERR_INVALID_ARG -1
#define BT_ERR_CUDA -2
#define BT_ERR_NO_MEMORY -3
#define BT_ERR_CAPACITY -4        /* node pool exhausted */
#define BT_ERR_RESERVED_KEY -5    /* UINT64_MAX given as a key to bt_bulk_build */
#define BT_ERR_BATCH_TOO_LARGE -6 /* n > bt_config.max_batch */
#define BT_ERR_NOT_TRAINED -7     /* learned descent requested before bt_retrain */
#define BT_ERR_STATIC_LIMIT -8    /* n > BT_STATIC_BUILD_MAX_KEYS in bt_bulk_build_static */
#define BT_ERR_BUSY -9            /* serving: no free slot or arena space now; retry after a completion */
#define BT_ERR_TIMEOUT -10        /* serving: bt_wait ran out of time */
#define BT_ERR_IO -11             /* snapshot file: cannot open / read / write, or not a valid snapshot */

/* ---- request op codes (same numbering as src/input-helper.h:14-17) ---- */
#define BT_OP_INSERT 0
#define BT_OP_GET 1
#define BT_OP_DELETE 2   /* src/input-helper.h:16 declares it; no reference version implements it.
                          * Answer: the previous value (FOUND) or ABSENT; the leaf shrinks in place
                          * (no merge with siblings). */

/* ---- per-request status byte written to out_status ---- */
#define BT_ST_ABSENT 0          /* key was not present (out_vals = 0) */
#define BT_ST_FOUND 1           /* key was present; out_vals = its (previous) value */
#define BT_ST_REJECTED 2        /* reserved key or unknown op; no effect */
#define BT_ST_RETRY_EXHAUSTED 3 /* STM insert could not commit within retry_limit; no effect */
#define BT_ST_NO_CAPACITY 4     /* node pool exhausted; no effect */

/* ---- batch modes (bt_execute_batch `mode`) ---- */
#define BT_MODE_SORTED 0      /* sort-based batch merge, deterministic (reference v38 meaning) */
#define BT_MODE_STM 1         /* unsorted warp-per-request STM (reference v39 meaning) */
#define BT_MODE_MERGE_ENGINE 0x10 /* with BT_MODE_SORTED: apply new keys by segmented leaf merge
                                      (needs leaf_fill >= 16 and inner_fill >= 16, else the STM engine runs) */

/* ---- descent (bt_set_descent) ---- */
#define BT_DESCENT_PLAIN 0
#define BT_DESCENT_LEARNED 1

typedef struct bt_config {
    uint64_t max_keys;     /* node pool sized for this many keys (default 1<<20) */
    uint64_t max_batch;    /* largest batch accepted (default 1<<22) */
    uint32_t leaf_fill;    /* keys per leaf for bulk build and merge splits (default 24) */
    uint32_t inner_fill;   /* keys per inner node for bulk build and merge splits (default 24) */
    uint32_t retry_limit;  /* STM attempts per request before BT_ST_RETRY_EXHAUSTED (default 65536) */
    int32_t device;        /* CUDA device ordinal (default 0) */
    uint32_t search_group; /* lanes per request in the search kernel: 4, 8, 16 or 32 (default 4; bt_autotune
                            * picks the fastest on the live tree) */
    uint32_t n_segments;   /* learned predictor: leaf segments (default 0: one per 64 leaves at each full
                            * training, a power of two, at least 4096; kept by bt_refit) */
    uint32_t window;       /* learned predictor: max error window in leaf slots (default 64) */
    uint32_t reserved[7];
} bt_config;

typedef struct bt_stats {
    uint64_t n_keys;
    uint64_t n_nodes;
    uint64_t n_leaves;        /* filled by bt_stats_get when with_leaves != 0 */
    uint32_t height;          /* levels including the leaf level, 0 when empty */
    uint32_t error;           /* sticky device error bits: 1 capacity, 2 retry limit */
    uint64_t commits;         /* STM commits */
    uint64_t aborts;          /* STM aborts (reference ABORT_COUNT roll_back_times) */
    uint64_t leaf_splits;
    uint64_t inner_splits;
    uint64_t new_roots;
    uint64_t retry_exhausted;
    uint64_t learned_hits;       /* learned descents that answered from the predicted leaf */
    uint64_t learned_fallbacks;  /* learned descents that fell back to the root descent */
    uint64_t learned_probe_sum;  /* sum of |predicted slot - true slot| over hits */
    uint64_t capacity_nodes;
} bt_stats;

typedef struct bt_handle bt_handle;

/* Fill `cfg` with defaults.  No reference counterpart (compile-time constants
 * in src/gpu-stm-tree-v39/bpt-gpustm.h:20-38). */
int bt_config_init(bt_config *cfg);

/* Allocate the node pool and batch work buffers on cfg->device.
 * Replaces GPU_STM_Tree::prepareGPU (src/gpu-stm-tree-v39/bpt-gpustm.cpp:14-28). */
int bt_create(const bt_config *cfg, bt_handle **out);

/* Free everything.  The reference never frees (~GPU_STM_Tree(){} ,
 * src/gpu-stm-tree-v39/bpt-gpustm.h:145). */
int bt_destroy(bt_handle *h);

/* Replace the tree contents with the n pairs (the last value wins for a repeated
 * key).  Synchronous.  The reference builds by running gpu_work() over a file of
 * P lines (src/main.cpp:21-25, src/gpu-stm-tree-v39/bpt-gpustm.cpp:67-132). */
int bt_bulk_build(bt_handle *h, const uint64_t *keys, const uint64_t *vals, size_t n, void *stream);

/* bt_bulk_build without any allocation, for callers that must not allocate GPU
 * memory while they load a tree: services whose device memory is reserved up
 * front by another allocator (a caching allocator or a start-up pool), where a
 * cudaMalloc at request time fails or fragments that pool, and latency-critical
 * threads, since cudaFree synchronises the whole device.  Same result as
 * bt_bulk_build.  Its scratch is a fixed device array inside the library
 * (about 2.6 MB, held on every GPU that loads the library until the process
 * exits), so n may be at most BT_STATIC_BUILD_MAX_KEYS, else
 * BT_ERR_STATIC_LIMIT.  All calls on a device share that array: calls that
 * overlap on the GPU race, so serialise them.  The first call on a device
 * looks up the array's device address; make that first call before any stream
 * capture on the device.  That address is kept for the process: calls after a
 * cudaDeviceReset of the device are not supported.  Synchronous.  This entry
 * point has no counterpart in the reference. */
#define BT_STATIC_BUILD_MAX_KEYS 65536
int bt_bulk_build_static(bt_handle *h, const uint64_t *keys, const uint64_t *vals, size_t n, void *stream);

/* Run one batch of n requests.  out_vals[i]/out_status[i] answer request i:
 * GET -> value or absent; INSERT -> previous value or absent, then insert or
 * update (src/input-helper.h:27-38).  Replaces gpu_work_main's per-batch
 * transferData/launchKernel/transferAns (src/gpu-stm-tree-v39/bpt-gpustm.cpp:78-105;
 * v38: src/gpu-stm-tree-v38/bpt-gpustm.cpp:88-112). */
int bt_execute_batch(bt_handle *h, const uint64_t *keys, const uint64_t *vals, const uint8_t *ops,
                     uint64_t *out_vals, uint8_t *out_status, size_t n, int mode, void *stream);

/* Same as bt_execute_batch with HOST buffers: copies in, runs, copies out and
 * synchronises `stream`.  Pinned buffers (bt_host_alloc) give full PCIe speed;
 * with BT_OPT_HOST_VALUES_IN_PLACE, BT_MODE_SORTED and a page-locked `vals`,
 * the value array is not copied: the kernels read the values of the batch's
 * writes from it over the bus.
 * Mirrors the reference's transferData -> kernel -> transferAns loop body
 * (src/gpu-stm-tree-v39/bpt-gpustm.cpp:78-105). */
int bt_execute_batch_host(bt_handle *h, const uint64_t *keys, const uint64_t *vals, const uint8_t *ops,
                          uint64_t *out_vals, uint8_t *out_status, size_t n, int mode, void *stream);
/* The same, asynchronous: queues the batch and returns a ticket (> 0; 0 for an
 * empty batch) that bt_host_wait redeems.  The handle keeps three staging
 * sets: a caller that keeps three batches in flight (submits batch i, then
 * waits for batch i - 2) gets the next batch's copy-in and the previous
 * batch's copy-out beside each batch's kernels; a fourth batch in flight
 * waits (on the host) until the first batch's answers are out.  Until its
 * ticket is redeemed, a batch's input buffers must stay unchanged and its
 * output buffers untouched.  Batches run in submission order, on `stream`.
 * The reference's loop is synchronous per batch
 * (src/gpu-stm-tree-v39/bpt-gpustm.cpp:67-132). */
int bt_execute_batch_host_async(bt_handle *h, const uint64_t *keys, const uint64_t *vals, const uint8_t *ops,
                                uint64_t *out_vals, uint8_t *out_status, size_t n, int mode, void *stream,
                                uint64_t *ticket);
/* The same with the values of the batch's INSERTs only: insert_vals[j] is the
 * value of the j-th INSERT request in request order, n_inserts of them (GET
 * and DELETE requests carry no value).  A read-mostly batch then copies 9 B
 * per request in (op code and key) plus 8 B per INSERT, instead of 17 B per
 * request.  n_inserts is checked against the op codes on the device, before
 * the batch's first kernel: on a mismatch every request of the batch is
 * answered BT_ST_REJECTED, nothing is applied, and bt_host_wait returns
 * BT_ERR_INVALID_ARG for its ticket (for the last 1024 such batches).  The
 * ticket is redeemed by bt_host_wait; the same staging sets, ordering and
 * buffer rules as bt_execute_batch_host_async.  No reference counterpart: the
 * reference copies a value slot for every request
 * (src/gpu-stm-tree-v39/bpt-gpustm.cpp:67-132). */
int bt_execute_batch_host_packed_async(bt_handle *h, const uint64_t *keys, const uint8_t *ops,
                                       const uint64_t *insert_vals, size_t n_inserts, uint64_t *out_vals,
                                       uint8_t *out_status, size_t n, int mode, void *stream, uint64_t *ticket);
/* Blocks until the batch of `ticket` has its answers in host memory
 * (its deferred leaf merge may still run; bt_sync orders after that). */
int bt_host_wait(bt_handle *h, uint64_t ticket);

/* `count` batches in order, their inputs all ready on `stream` (device
 * pointers in host arrays of `count`; batch j has n[j] requests and its own
 * output arrays).  Same answers and tree as `count` calls of
 * bt_execute_batch; with BT_MODE_SORTED and the hash front end, batch j + 1's
 * classification, sort and merge passes (which read no tree) run on an
 * internal stream beside batch j's lookups and writes, with a second set of
 * per-batch buffers (allocated at the first call, about 70 B per request of
 * capacity).  Other modes run the batches one by one.  Phases are not
 * recorded (bt_profile).  No reference counterpart: the reference runs its
 * batches one after another (src/gpu-stm-tree-v38/bpt-gpustm.cpp, gpu_work). */
int bt_execute_batches(bt_handle *h, size_t count, const uint64_t *const *keys, const uint64_t *const *vals,
                       const uint8_t *const *ops, uint64_t *const *out_vals, uint8_t *const *out_status,
                       const size_t *n, int mode, void *stream);

/* Convenience wrappers: all-GET and all-INSERT batches in BT_MODE_SORTED,
 * the reference's single-mission input (prepareInput(file, mission),
 * src/tree.h:34). */
int bt_search_batch(bt_handle *h, const uint64_t *keys, uint64_t *out_vals, uint8_t *out_status, size_t n,
                    void *stream);
int bt_insert_batch(bt_handle *h, const uint64_t *keys, const uint64_t *vals, uint64_t *out_vals,
                    uint8_t *out_status, size_t n, void *stream);

/* Range scan of n queries [lo[i], hi[i]] (both ends included, the reference's
 * "G start end" request, src/input-helper.h:177-185; op code RANGE = 3 is
 * declared there, src/input-helper.h:17, but no reference version implements
 * it).  Query i writes its first min(count, max_per) pairs in ascending key
 * order to out_keys/out_vals[i * max_per ...] and the full number of keys in
 * its range to out_counts[i] (a count above max_per means truncation).
 * Device buffers; stream ordered; must not overlap a batch that writes. */
int bt_range_batch(bt_handle *h, const uint64_t *lo, const uint64_t *hi, size_t n, uint32_t max_per,
                   uint64_t *out_keys, uint64_t *out_vals, uint32_t *out_counts, void *stream);

/* Number of keys (synchronous).  No reference counterpart. */
int bt_size(bt_handle *h, uint64_t *n_keys);

/* All pairs in ascending key order into device buffers of `cap` entries;
 * *n_out = number of pairs.  Synchronous.  Replaces the reference's -t answer
 * print (src/input-helper.h:205-218) as the parity format. */
int bt_dump_sorted(bt_handle *h, uint64_t *keys, uint64_t *vals, size_t cap, size_t *n_out, void *stream);

/* Host arrays: leaf sizes in key order (cap entries) and node counts per level
 * (leaf level first).  Synchronous.  Used to check split counts against the
 * oracle; no reference counterpart. */
int bt_leaf_sizes(bt_handle *h, uint32_t *sizes_host, size_t cap, size_t *n_leaves);
int bt_level_counts(bt_handle *h, uint64_t *counts_host, uint32_t cap, uint32_t *height);

/* Counters (synchronous).  with_leaves != 0 also enumerates the leaves.
 * Reference: ABORT_COUNT counters (src/gpu-stm-tree-v39/bpt-gpustm.cpp:111-129). */
int bt_stats_get(bt_handle *h, bt_stats *st, int with_leaves);
int bt_stats_reset(bt_handle *h);

/* Learned leaf predictor (no reference counterpart: the reference's closest
 * structure is v35's leaf array, src/gpu-stm-tree-v35/bpt-gpustm-kernel.cu:135-152).
 * bt_retrain rebuilds the leaf array and trains the model on the GPU
 * (synchronous); bt_set_descent picks plain or learned search. */
int bt_retrain(bt_handle *h, void *stream);
/* Incremental retraining after the tree has changed: rebuilds the leaf array
 * from the current leaves and re-fits the per-segment lines, keeping the
 * trained stage-1 model and its key normalisation (plus BT_OPT_REFIT_STEPS
 * warm-started Adam steps of it, default 0).  Stream ordered when `stream` is
 * given (its leaf enumeration synchronises the stream), synchronous with NULL.
 * BT_ERR_NOT_TRAINED before the first bt_retrain. */
int bt_refit(bt_handle *h, void *stream);
int bt_set_descent(bt_handle *h, int descent);
/* stage 1 root model: 1 = 1->32->1 MLP (default), 0 = linear */
int bt_set_root_model(bt_handle *h, int mlp);
/* lanes per request of the unsorted search (the reference fixes one warp per
 * request at compile time, src/gpu-stm-tree-v39/bpt-gpustm.h:25-38) */
int bt_set_search_group(bt_handle *h, uint32_t lanes);
/* Tuning options (bt_set_option); no reference counterpart (its variants are
 * compile-time, src/gpu-stm-tree-v39/bpt-gpustm.h:25-38). */
#define BT_OPT_SORTED_SEARCH 1 /* 1 (default): the batch's GET phase reuses the descent path across its
                                  ascending unique keys; 0: one root descent per key */
#define BT_OPT_RETRY_LIMIT 2   /* STM attempts per request */
#define BT_OPT_TRAIN_STEPS 3   /* Adam steps of the learned root model per bt_retrain */
#define BT_OPT_SORTED_LEAF_VALS 4 /* sorted search loads leaf values with the keys (1) or only the match (0) */
#define BT_OPT_BATCH_DESCENT 5 /* batch GET phase: -1 follow bt_set_descent (default), 0 plain, 1 learned */
#define BT_OPT_FRONT_END 6     /* BT_MODE_SORTED batches: 1 (default) hash front end - only requests whose key
                                * has an INSERT at or before them in the batch are sorted and merged, the rest
                                * are unsorted lookups of the pre-batch tree; 0 sort the whole batch (the
                                * reference's layout, v38 bpt-gpustm-kernel.cu:289-324).  Same answers. */
#define BT_OPT_TOP_CACHE 7     /* 1 (default): unsorted plain searches descend the tree's upper levels (up to
                                * 256 nodes) from a per-launch copy in shared memory; 0 all from global */
#define BT_OPT_OVERLAP 9       /* 1 (default): with the hash front end, the merge engine's locates and grouping of
                                * the touched requests run on a high-priority side stream while the lookups run
                                * (the lookups leave 4 block slots free; a value > 1 sets that to value - 1);
                                * 0 one after the other */
#define BT_OPT_SEARCH_PAIRS 8  /* unsorted plain searches: 2 (default) two requests per lane group in lock step,
                                * loading only the chosen child id at inner levels (half the bytes of a full
                                * row, one more dependent load); 1 the pairs with full rows; 0 one request
                                * per group.  Nonzero takes precedence over BT_OPT_TOP_CACHE */
#define BT_OPT_ASYNC_WRITE 10  /* 1 (default): a BT_MODE_SORTED | BT_MODE_MERGE_ENGINE batch with the hash front
                                * end completes on the caller's stream once its answers are final; its leaf and
                                * inner merge finish on an internal stream, beside the next batch's front end and
                                * sort.  Every later call on this handle, on any stream, waits for them before it
                                * touches the tree (bt_sync waits explicitly); 0 the merge runs on the caller's
                                * stream.  Same answers and tree. */
#define BT_OPT_REFIT_STEPS 11  /* warm-started Adam steps of the stage-1 model per bt_refit (default 0) */
#define BT_OPT_HOST_VALUES_IN_PLACE 13 /* host-buffer entry points, BT_MODE_SORTED: 1 reads the values of the
                                       * batch's writes from a page-locked value array over the bus instead of
                                       * copying the array (fewer bytes, but scattered reads; measured slower on
                                       * a 95/5 batch of 2^22); 0 (default) copies it */
#define BT_OPT_STM_COMBINE 15   /* BT_MODE_STM batches: 1 (default) combines the INSERTs of one key into one
                                 * transaction: the first to arrive stores the last one's value, each other is
                                 * answered FOUND with the value of the one before it (a serial order of the
                                 * concurrent requests, which is what the v39 meaning allows; keys the batch
                                 * also DELETEs are not combined); 0 runs every INSERT as its own transaction,
                                 * like the reference (src/gpu-stm-tree-v39/bpt-gpustm-kernel.cu:41-56) */
#define BT_OPT_LEARNED_POLICY 16 /* batches with the learned descent: 0 use it as chosen; 1 (default) the device
                                  * judges the miss rate after each batch's learned lookups and, once more than 5 %
                                  * of a window of 65536 fall back to the plain descent (leaves split since the fit),
                                  * the batches hand every lookup to the plain descent until the next bt_retrain /
                                  * bt_refit (in stream order: batches already queued follow it too); 2 the same,
                                  * and the library refits by itself once 8 batches have run since the last fit.
                                  * Answers are the same in every case; bt_search_batch keeps bt_set_descent's
                                  * choice */
#define BT_OPT_HOST_FRONT_OVERLAP 17 /* host-buffer entry points, BT_MODE_SORTED with the hash front end: 1
                                      * (default) a batch's classification, sort and merge passes (which read no
                                      * tree) run on an internal stream once its requests are copied in, beside
                                      * the previous host batch's lookups and writes, with a second set of
                                      * per-batch buffers (as bt_execute_batches); any other call on the handle
                                      * in between makes the next one wait for it.  0 runs each batch whole on
                                      * `stream`.  Same answers and tree */
#define BT_OPT_TOUCH_SORT 18 /* hash front end: the sort of the requests whose key a write touches.  1 sorts
                              * tiles of 2048 pairs on chip, then merges sorted runs pairwise (merge path)
                              * until one is left: a few rounds for the few hundred thousand such requests
                              * of a read-mostly batch; 0 the onesweep radix sort (eight passes of 8 bits,
                              * BT_OPT_SORT_TILE), better for many; 2 (default) the first while the touched
                              * count of the batch seen last was at most 2^19, else the second (the first
                              * batch: the second).  Same order in every case (by key, then request order) */
#define BT_OPT_SORT_TILE 14     /* radix sort tile of sorted batches: 256, 512 (default) or 1024 threads x 8 keys,
                                 * for whole batches and for the hash front end's touched requests alike
                                 * (bt_autotune picks the two separately) */
#define BT_OPT_LEARNED_MODE 12 /* unsorted learned lookups: 1 one request per lane group, 2 two requests per
                                * group in lock step, 3 (default) software-pipelined: a group carries up to five
                                * requests, one in each round of loads (list entry, key, leaf-table probe, leaf
                                * row, value); bt_autotune picks */
int bt_set_option(bt_handle *h, int option, int64_t value);
/* Orders work after every batch issued so far on this handle, its deferred
 * leaf/inner merge included (BT_OPT_ASYNC_WRITE): with a stream, the stream
 * waits; with NULL, the host blocks.  A CUDA stream sync or event on the
 * caller's stream covers a batch's answers but not its deferred merge; the
 * library's own calls need no bt_sync.  No reference counterpart (the
 * reference synchronises after every batch kernel, src/gpu-stm-tree-v38/
 * bpt-gpustm-kernel.cu:289-324). */
int bt_sync(bt_handle *h, void *stream);
/* Autotuner: times the lookup and sort configurations on this tree with n
 * sample keys (device pointer, n <= max_batch) and keeps the fastest: lanes
 * per request of the plain search, lanes per request and form of the learned
 * lookup, the sorted search's leaf-value load, the descent used by the batch
 * GET phase, and the radix sort's tile (256, 512 or 1024 threads x 8 keys) for
 * whole batches and for the hash front end's touched requests.  Read-only;
 * synchronous.
 * report (nullable, BT_AUTOTUNE_REPORT_LEN doubles): [0] plain lanes, [1]
 * learned lanes, [2] leaf values mode, [3] batch descent, [4..7] plain ms for
 * 4/8/16/32 lanes, [8..11] learned ms for 4 lanes pipelined, 2 lanes
 * pipelined, 4 lanes one request, 2 lanes one request, [12..13] sorted plain
 * ms (mode 0/1), [14] sorted learned ms, [15] learned mode
 * (BT_OPT_LEARNED_MODE), [16] sort tile threads (whole batch), [17] sort tile
 * threads (touched requests), [18..20] whole-sample sort ms for 256/512/1024,
 * [21..23] sixteenth-sample sort ms for 256/512/1024.  No reference counterpart (the reference's launch
 * shape is compile-time, src/gpu-stm-tree-v39/bpt-gpustm.h:25-38). */
#define BT_AUTOTUNE_REPORT_LEN 24
int bt_autotune(bt_handle *h, const uint64_t *sample_keys, size_t n, void *stream, double *report);
/* Node-fill autotuner (the fanout the merge engine and the bulk loader pack
 * to): builds a sample tree from the n sample keys (device pointer, n >= 64)
 * in a temporary handle for each leaf/inner fill of 16, 20, 24 and 28 keys,
 * times sorted 95/5 batches of n requests on it (merge engine), and keeps the
 * fastest fill for this handle's later bulk builds and merge splits (the
 * current leaves are not repacked).  Synchronous; allocates the temporary
 * trees.  report (nullable, 8 doubles): [0] leaf fill, [1] inner fill, [2..5]
 * ms per batch for fills 16/20/24/28.  The reference's fanout is the
 * compile-time ORDER (src/gpu-stm-tree-v39/bpt-gpustm.h:21-31). */
int bt_autotune_fill(bt_handle *h, const uint64_t *sample_keys, size_t n, void *stream, double *report);
/* Learned predictor settings and diagnostics (no reference counterpart: the
 * reference has no learned model).
 * Lanes per request in the learned search kernel: 2, 4, 8, 16 or 32 (default 4). */
int bt_set_learned_group(bt_handle *h, uint32_t lanes);
/* info[8]: valid, n_leaves, n_segments, segments over the window, window,
 * final training loss, root model (1 MLP, 0 linear), training steps */
int bt_learned_info(bt_handle *h, double *info);
/* Gradient of the mean-squared error of the 1->32->1 MLP (params packed
 * w1[32] b1[32] w2[32] b2) over n device pairs (x, y), computed by the same
 * kernels that train the model; grad_out[97] and *loss_out are device
 * pointers.  Used to check the training kernels against the CPU oracle. */
int bt_mlp_grad(bt_handle *h, const float *params, const float *x, const float *y, size_t n, float *grad_out,
                float *loss_out, void *stream);

/* Phase timing with CUDA events recorded on the batch's stream between the
 * phases of BT_MODE_SORTED (0 sort, 1 merge, 2 search, 3 insert, 4 writeback),
 * like the reference's Time_Measure (src/time_measure.cuh:14-42,
 * src/gpu-stm-tree-v38/bpt-gpustm-kernel.cu:289-324).  bt_profile_read
 * synchronises on the recorded events and returns summed milliseconds. */
int bt_profile(bt_handle *h, int enable);
int bt_profile_read(bt_handle *h, double *phase_ms /* [5] */, uint64_t *batches, int reset);
/* Kernels launched by this library in this process so far (no reference
 * counterpart). */
uint64_t bt_launch_count(void);

/* Pinned host memory helpers for bt_execute_batch_host callers (the
 * reference copies from pageable vectors, src/gpu-stm-tree-v39/bpt-gpustm.cpp:78-105). */
int bt_host_alloc(void **p, size_t bytes);
int bt_host_free(void *p);

/* ---- serving loop (continuous batching) ----
 * No reference counterpart: the reference runs batches one after another from
 * one host thread (src/gpu-stm-tree-v39/bpt-gpustm.cpp:78-105).
 * A server owns a device arena and a ring of batch slots.  bt_submit admits a
 * batch when a slot and enough arena bytes are free (else BT_ERR_BUSY), copies
 * it in and publishes it to a persistent kernel (graph-launched, relaunched on
 * demand) whose warps take chunks of the oldest unfinished batch, so batches
 * submitted while others run overlap on the device.  Requests run under the
 * STM meaning (BT_MODE_STM): batches in flight together may interleave on
 * shared keys; a batch whose keys no other in-flight batch touches gets the
 * answers it would get alone.  Host buffers: pageable inputs may be reused
 * when bt_submit returns, pinned inputs only after completion; output buffers
 * must stay valid until completion.  One server per handle; do not mix with
 * other batch calls on that handle while it runs. */
typedef struct bt_server bt_server;
typedef struct bt_serve_config {
    uint64_t arena_bytes;  /* device memory for batches in flight: 26 B per request (default 1 GiB) */
    uint32_t max_batches;  /* ring slots (default 256) */
    uint32_t idle_us;      /* the persistent kernel exits after this long without work (default 2000) */
    uint32_t policy;       /* which admitted batch a free warp takes work from: 0 (default) the oldest
                            * (first in, first out), 1 the one with the fewest unclaimed requests among the
                            * 32 oldest, so that small batches are not held behind a large one (measured:
                            * lower p50 but a p99 in the hundreds of ms for the large batches it holds back) */
    uint32_t reserved[5];
} bt_serve_config;
typedef struct bt_serve_stats {
    uint64_t batches;          /* completed since start / last reset */
    uint64_t requests;
    uint64_t kernel_launches;  /* persistent-kernel launches (graph replays) */
    uint64_t in_flight;
    double p50_ms, p99_ms, max_ms, mean_ms;  /* batch latency: submit -> answers in host memory */
    double mops;                             /* completed requests / (last completion - first submit) */
    double p50_service_ms, p99_service_ms;   /* device time from the batch's first claimed chunk to its
                                              * last finished one (the rest of the latency is waiting
                                              * for admission, the copies and the first claim) */
    double device_mops;                      /* completed requests / (latest completion - earliest first
                                              * claim), both on the device clock */
} bt_serve_stats;
int bt_serve_config_init(bt_serve_config *cfg);
int bt_serve_start(bt_handle *h, const bt_serve_config *cfg, bt_server **out);
int bt_submit(bt_server *s, const uint64_t *keys_host, const uint64_t *vals_host, const uint8_t *ops_host,
              size_t n, uint64_t *out_vals_host, uint8_t *out_status_host, uint64_t *ticket);
/* *done = 1 when the batch's answers are in its output buffers, 0 if not yet, -1 unknown ticket */
int bt_poll(bt_server *s, uint64_t ticket, int *done);
int bt_wait(bt_server *s, uint64_t ticket, uint32_t timeout_ms /* 0 = no limit */);
int bt_serve_get_stats(bt_server *s, bt_serve_stats *st, int reset);
/* Device clock (ns) of a finished batch's first claimed chunk and of its
 * completion; BT_ERR_INVALID_ARG for a batch that has not finished or whose
 * slot has been reused since.  Shows which batches ran on the device at the
 * same time. */
int bt_serve_batch_times(bt_server *s, uint64_t ticket, uint64_t *first_claim_ns, uint64_t *done_ns);
int bt_serve_stop(bt_server *s);

/* ---- benchmark input generators (seeded, counter based; device output) ----
 * dist: 0 uniform keys in [0, 2^63), 1 Zipf(0.99) ranks over 2^32 hashed to
 * uint64 (bt_gen_keys returns the n most popular ranks), 2 Normal(2^62, 2^58),
 * 3 Gamma(2, 2^56).  vals (nullable) receives key ^ 0x9E3779B97F4A7C15.
 * bt_gen_requests: search_pct % GETs, half of them keys of tree_keys; the rest
 * INSERTs of fresh keys.  These stand in for the reference's dataset files,
 * which are not shipped (evalutaion/random_testall_v39.sh:9-28). */
int bt_gen_keys(int dist, uint64_t seed, size_t n, uint64_t *keys, uint64_t *vals, void *stream);
int bt_gen_requests(int dist, uint64_t seed, const uint64_t *tree_keys, size_t n_tree, size_t n,
                    uint32_t search_pct, uint64_t *keys, uint64_t *vals, uint8_t *ops, void *stream);

/* ---- key-range sharding (one tree per GPU) ----
 * No counterpart in the reference, which runs one tree on one GPU
 * (src/gpu-stm-tree-v39/bpt-gpustm.cpp:14-28).  Shard s owns the keys in
 * [splitters[s-1], splitters[s]); splitters holds n_shards - 1 non-decreasing
 * keys (device memory; equal neighbours leave a shard empty),
 * 1 <= n_shards <= BT_MAX_SHARDS.
 *
 * bt_route_batch reorders a batch by owning shard, stably (each shard's run
 * keeps the input order): out_keys/out_vals/out_ops[i] = input[out_perm[i]],
 * out_counts[s] (device, uint64) = length of shard s's run.  vals and ops may
 * be NULL (their outputs are then not written).  n < 2^32.  Up to max_batch
 * requests it uses the handle's batch work buffers (stream-ordered with the
 * handle's other calls); larger inputs, such as the keys of a sharded bulk
 * build, take stream-ordered temporaries (cudaMallocAsync) for the call.
 *
 * bt_unroute_results scatters answers that came back in routed order to
 * input order: out_vals[perm[i]] = in_vals[i], out_status[perm[i]] = in_status[i]. */
#define BT_MAX_SHARDS 256
int bt_route_batch(bt_handle *h, const uint64_t *splitters, int n_shards, const uint64_t *keys,
                   const uint64_t *vals, const uint8_t *ops, size_t n, uint64_t *out_keys, uint64_t *out_vals,
                   uint8_t *out_ops, uint32_t *out_perm, uint64_t *out_counts, void *stream);
int bt_unroute_results(bt_handle *h, const uint32_t *perm, const uint64_t *in_vals, const uint8_t *in_status,
                       size_t n, uint64_t *out_vals, uint8_t *out_status, void *stream);

/* ---- snapshot (checkpoint / resume) ----
 * No counterpart in the reference, whose tree lives only as long as the
 * process (src/gpu-stm-tree-v39/bpt-gpustm.h:145).  bt_save writes the sorted
 * (key, value) pairs and a checksum to `path`; bt_load replaces h's contents
 * with a saved file by a bulk build (same contents and answers; the leaf
 * layout is a fresh bulk load with h's fill settings).  Both synchronous;
 * BT_ERR_IO for file errors, a bad magic, size, checksum or key order. */
int bt_save(bt_handle *h, const char *path);
int bt_load(bt_handle *h, const char *path);
/* Pool image: bt_save_image writes the node pool itself (every allocated
 * node's key and value rows, low fences, the control block and the handle's
 * leaf and inner fills); bt_load_image restores it into h, whose pool must
 * hold as many nodes (else BT_ERR_NO_MEMORY) and whose fills must equal the
 * saved ones (else BT_ERR_INVALID_ARG: later splits follow the fills), so the
 * loaded tree keeps the saved leaf layout and continues exactly as the saved
 * one would.  The loaded handle's counters and sticky error bits start at
 * zero.  Synchronous; BT_ERR_IO for file errors, a bad magic, size or
 * checksum. */
int bt_save_image(bt_handle *h, const char *path);
int bt_load_image(bt_handle *h, const char *path);

/* Static text for a status code. */
const char *bt_status_string(int code);

#ifdef __cplusplus
}
#endif
#endif /* EIRENE_B200_H */
