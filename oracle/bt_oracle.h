/*
 * CPU oracle for the batched B+tree path (TEST INFRASTRUCTURE ONLY).
 *
 * This is a plain-C restatement of the reference's algorithm, used by the
 * tests, the smoke check and the bench's CPU-baseline leg as the checker.
 * The product path (eirene_b200/csrc) never links or calls it.
 *
 * What it restates (paths relative to the reference project):
 *   - node layout and info encoding      src/gpu-stm-tree-v39/bpt-gpustm.h:41-60,
 *                                        src/gpu-stm-tree-v39/bpt-gpustm-kernel-tree.cuh:29-56
 *   - descent + early split of full inner nodes
 *                                        src/gpu-stm-tree-v39/bpt-gpustm-kernel.cu:136-190
 *   - inner split 15/15 around key[15]   src/gpu-stm-tree-v39/bpt-gpustm-kernel-tree.cuh:150-224
 *   - separator insert into a parent     src/gpu-stm-tree-v39/bpt-gpustm-kernel-tree.cuh:246-301
 *   - new root                           src/gpu-stm-tree-v39/bpt-gpustm-kernel-tree.cuh:307-344
 *   - leaf update / shift-insert / 16-16 split with right fence
 *                                        src/gpu-stm-tree-v39/bpt-gpustm-kernel-tree.cuh:348-467
 *   - answer rule (GET -> value or absent; INSERT -> previous value or absent)
 *                                        src/gpu-stm-tree-v39/bpt-gpustm-kernel.cu:197-213,
 *                                        src/input-helper.h:27-38
 *   - sort-based batch merge semantics   src/gpu-stm-tree-v38/bpt-gpustm-kernel.cu:289-324,
 *                                        src/gpu-stm-tree-v38/bpt-gpustm-kernel-aux.cuh:16-56
 * The bulk loader and the segmented leaf merge have no counterpart in the
 * reference (it builds by inserting); their deterministic packing rules are
 * defined here and restated bit-for-bit by the CUDA path.
 *
 * Keys and values are uint64; key UINT64_MAX is reserved as the padding
 * sentinel (the reference reserves INT_MAX the same way).
 */
#ifndef BT_ORACLE_H
#define BT_ORACLE_H
#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define BTO_ORDER 32
#define BTO_MAX_KEYS 31
#define BTO_KEY_MAX UINT64_MAX
#define BTO_NIL 0xFFFFFFFFu

/* operation codes: same numbering as the reference (src/input-helper.h:14-17) */
#define BTO_OP_INSERT 0
#define BTO_OP_GET 1
#define BTO_OP_DELETE 2 /* src/input-helper.h:16 (declared there, implemented by no reference version) */

/* per-request result status */
#define BTO_ABSENT 0
#define BTO_FOUND 1
#define BTO_REJECTED 2

/* insert engines for the merged batch */
#define BTO_ENGINE_STM 0   /* one-at-a-time insert (reference rules) */
#define BTO_ENGINE_MERGE 1 /* deterministic segmented leaf merge */

typedef struct bto_tree bto_tree;

typedef struct bto_stats {
    uint64_t n_keys;
    uint64_t n_nodes;
    uint64_t n_leaves;
    uint32_t height; /* levels including the leaf level; 0 for an empty tree */
    uint32_t root_level;
    uint64_t leaf_splits;  /* new leaves created by inserts */
    uint64_t inner_splits; /* new inner nodes created by inserts (new roots included) */
    uint64_t new_roots;
} bto_stats;

bto_tree *bto_create(uint32_t leaf_fill, uint32_t inner_fill);
void bto_destroy(bto_tree *t);
void bto_clear(bto_tree *t);

/* Replace the contents with the pairs (last value wins for repeated keys). */
int bto_bulk_build(bto_tree *t, const uint64_t *keys, const uint64_t *vals, size_t n);

/* Single-request operations (reference rules). Return BTO_FOUND/BTO_ABSENT/BTO_REJECTED. */
int bto_get(const bto_tree *t, uint64_t key, uint64_t *val);
int bto_insert(bto_tree *t, uint64_t key, uint64_t val, uint64_t *old_val);
/* Remove `key`; *old_val = its value.  The leaf shrinks in place: no merge
 * or redistribution with siblings, an emptied leaf stays in the tree (its
 * separators keep routing).  Returns BTO_FOUND or BTO_ABSENT. */
int bto_delete(bto_tree *t, uint64_t key, uint64_t *old_val);

/* Requests applied one at a time in input order (the serial meaning of the
 * unsorted STM batch). */
void bto_execute_serial(bto_tree *t, const uint64_t *keys, const uint64_t *vals,
                        const uint8_t *ops, size_t n, uint64_t *out_vals, uint8_t *out_status);

/* Sort-merged batch: per key, requests take effect in input order; across
 * keys every request sees the pre-batch tree.  engine picks how the unique
 * inserts are applied (BTO_ENGINE_STM: in ascending key order, one by one;
 * BTO_ENGINE_MERGE: segmented leaf merge).  n_threads > 1 runs the lookups
 * on that many host threads. */
void bto_execute_merged(bto_tree *t, const uint64_t *keys, const uint64_t *vals,
                        const uint8_t *ops, size_t n, uint64_t *out_vals, uint8_t *out_status,
                        int engine, int n_threads);

size_t bto_size(const bto_tree *t);
void bto_dump(const bto_tree *t, uint64_t *keys, uint64_t *vals);
/* sizes of the leaves in key order; returns the leaf count (writes at most cap) */
size_t bto_leaf_sizes(const bto_tree *t, uint32_t *sizes, size_t cap);
/* node counts per level, leaf level first; returns height */
uint32_t bto_level_counts(const bto_tree *t, uint64_t *counts, uint32_t cap);
/* (low key) of every leaf in key order, i.e. the learned predictor's training pairs */
size_t bto_leaf_lows(const bto_tree *t, uint64_t *lows, size_t cap);
void bto_get_stats(const bto_tree *t, bto_stats *s);
/* structural self-check: sorted keys, fences, separators, sizes. 0 = ok */
int bto_check(const bto_tree *t);

/* stable LSD radix sort of (key, index) pairs; idx_out[i] = input position */
void bto_sort_pairs(const uint64_t *keys, size_t n, uint64_t *keys_out, uint32_t *idx_out);

/* ---- learned leaf predictor reference (float math in double) ---- */
/* forward of the 1->32->1 MLP on normalised x; params packed [w1(32) b1(32) w2(32) b2] */
double bto_mlp_forward(const float *params, double x);
/* mean-squared-error gradient over a minibatch; grad packed like params */
double bto_mlp_grad(const float *params, const float *x, const float *y, size_t n, double *grad);

/* ---- workload generators (counter-based, seeded) ---- */
uint64_t bto_mix64(uint64_t x);
uint64_t bto_rand(uint64_t seed, uint64_t i, uint64_t j);
/* dist: 0 uniform [0,2^63), 1 zipf(0.99) over 2^32 ranks hashed, 2 normal(2^62, 2^58), 3 gamma(2, 2^56) */
void bto_gen_keys(int dist, uint64_t seed, size_t n, uint64_t *keys);
uint64_t bto_value_of(uint64_t key);
/* request batch: search_pct in [0,100]; searches are half existing keys (drawn from
 * tree_keys) and half drawn from dist; inserts draw fresh keys from dist with
 * value = bto_value_of(key). */
void bto_gen_requests(int dist, uint64_t seed, const uint64_t *tree_keys, size_t n_tree,
                      size_t n, uint32_t search_pct, uint64_t *keys, uint64_t *vals, uint8_t *ops);

#ifdef __cplusplus
}
#endif
#endif
