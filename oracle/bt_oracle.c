/*
 * CPU oracle for the batched B+tree path.  TEST INFRASTRUCTURE ONLY: the
 * tests, the smoke check and the bench's CPU-baseline leg use it as the
 * checker; the CUDA product path never links it.
 *
 * Parity is pinned against the reference binary itself (built from the
 * reference sources by oracle/build_ref.sh and run on 31-bit keys) because
 * the reference ships no golden vectors or tests of its own.
 *
 * Reference files cited below are relative to the reference project root.
 */
#include "bt_oracle.h"

#include <math.h>
#include <pthread.h>
#include <stdlib.h>
#include <string.h>

/* ------------------------------------------------------------------------ */
/* node pool: keys[n][32] (slot 31 = info), vals[n][32] (leaf slot 31 = right
 * fence), low[n] = low fence.  Mirrors the reference's keyArr_t/valArr_t
 * (src/gpu-stm-tree-v39/bpt-gpustm.h:41-51) widened to uint64.            */

typedef uint64_t node_row[BTO_ORDER];

struct bto_tree {
    node_row *keys;
    node_row *vals;
    uint64_t *low;
    uint32_t cap;
    uint32_t n_nodes;
    uint32_t root;
    uint32_t leaf_fill;
    uint32_t inner_fill;
    uint64_t n_keys;
    uint64_t leaf_splits, inner_splits, new_roots;
};

/* info word: size in bits 8..15, level in bits 0..7 (level 0 = leaf).  The
 * reference packs size<<5 | level (src/gpu-stm-tree-v39/bpt-gpustm-kernel-tree.cuh:29-56). */
static inline uint32_t n_size(const bto_tree *t, uint32_t n) { return (uint32_t)((t->keys[n][31] >> 8) & 0xff); }
static inline uint32_t n_level(const bto_tree *t, uint32_t n) { return (uint32_t)(t->keys[n][31] & 0xff); }
static inline void n_set_info(bto_tree *t, uint32_t n, uint32_t size, uint32_t level) {
    t->keys[n][31] = ((uint64_t)size << 8) | level;
}

static uint32_t alloc_node(bto_tree *t) {
    if (t->n_nodes == t->cap) {
        uint32_t nc = t->cap ? t->cap * 2 : 1024;
        t->keys = (node_row *)realloc(t->keys, sizeof(node_row) * nc);
        t->vals = (node_row *)realloc(t->vals, sizeof(node_row) * nc);
        t->low = (uint64_t *)realloc(t->low, sizeof(uint64_t) * nc);
        t->cap = nc;
    }
    uint32_t n = t->n_nodes++;
    for (int i = 0; i < BTO_ORDER; i++) {
        t->keys[n][i] = BTO_KEY_MAX;
        t->vals[n][i] = 0;
    }
    t->low[n] = 0;
    return n;
}

bto_tree *bto_create(uint32_t leaf_fill, uint32_t inner_fill) {
    bto_tree *t = (bto_tree *)calloc(1, sizeof(bto_tree));
    if (leaf_fill < 2 || leaf_fill > BTO_MAX_KEYS) leaf_fill = 24;
    if (inner_fill < 1 || inner_fill > BTO_MAX_KEYS) inner_fill = 24;
    t->leaf_fill = leaf_fill;
    t->inner_fill = inner_fill;
    t->root = BTO_NIL;
    return t;
}

void bto_clear(bto_tree *t) {
    t->n_nodes = 0;
    t->root = BTO_NIL;
    t->n_keys = 0;
    t->leaf_splits = t->inner_splits = t->new_roots = 0;
}

void bto_destroy(bto_tree *t) {
    if (!t) return;
    free(t->keys);
    free(t->vals);
    free(t->low);
    free(t);
}

/* number of keys[0..size) that are <= key: the child slot of an inner node.
 * Child i covers [key[i-1], key[i]) (src/tree.h:7-19). */
static inline uint32_t upper_slot(const uint64_t *k, uint32_t size, uint64_t key) {
    uint32_t lo = 0, hi = size;
    while (lo < hi) {
        uint32_t mid = (lo + hi) >> 1;
        if (k[mid] <= key) lo = mid + 1; else hi = mid;
    }
    return lo;
}
static inline uint32_t lower_slot(const uint64_t *k, uint32_t size, uint64_t key) {
    uint32_t lo = 0, hi = size;
    while (lo < hi) {
        uint32_t mid = (lo + hi) >> 1;
        if (k[mid] < key) lo = mid + 1; else hi = mid;
    }
    return lo;
}

static uint32_t find_leaf(const bto_tree *t, uint64_t key, uint32_t *path, uint32_t *slots) {
    uint32_t n = t->root;
    uint32_t lvl = n_level(t, n);
    while (lvl > 0) {
        uint32_t c = upper_slot(t->keys[n], n_size(t, n), key);
        if (path) { path[lvl] = n; slots[lvl] = c; }
        n = (uint32_t)t->vals[n][c];
        lvl--;
    }
    if (path) { path[0] = n; slots[0] = 0; }
    return n;
}

int bto_get(const bto_tree *t, uint64_t key, uint64_t *val) {
    if (key == BTO_KEY_MAX) return BTO_REJECTED;
    if (t->root == BTO_NIL) return BTO_ABSENT;
    uint32_t leaf = find_leaf(t, key, NULL, NULL);
    uint32_t sz = n_size(t, leaf);
    uint32_t p = lower_slot(t->keys[leaf], sz, key);
    if (p < sz && t->keys[leaf][p] == key) {
        if (val) *val = t->vals[leaf][p];
        return BTO_FOUND;
    }
    return BTO_ABSENT;
}

/* separator insert into an inner node: key at slot, new child at slot+1
 * (src/gpu-stm-tree-v39/bpt-gpustm-kernel-tree.cuh:232-301). */
static void insert_separator(bto_tree *t, uint32_t p, uint32_t slot, uint64_t sep, uint32_t child) {
    uint32_t sz = n_size(t, p);
    for (uint32_t i = sz; i > slot; i--) t->keys[p][i] = t->keys[p][i - 1];
    for (uint32_t i = sz + 1; i > slot + 1; i--) t->vals[p][i] = t->vals[p][i - 1];
    t->keys[p][slot] = sep;
    t->vals[p][slot + 1] = child;
    n_set_info(t, p, sz + 1, n_level(t, p));
}

/* new root with one key and two children (src/gpu-stm-tree-v39/bpt-gpustm-kernel-tree.cuh:307-344) */
static void new_root(bto_tree *t, uint32_t left, uint64_t sep, uint32_t right, uint32_t level) {
    uint32_t r = alloc_node(t);
    t->keys[r][0] = sep;
    t->vals[r][0] = left;
    t->vals[r][1] = right;
    t->low[r] = t->low[left];
    n_set_info(t, r, 1, level);
    t->root = r;
    t->new_roots++;
    t->inner_splits++;
}

/* early split of a full inner node: up = key[15]; left keeps keys 0..14 and
 * children 0..15, right gets keys 16..30 and children 16..31
 * (src/gpu-stm-tree-v39/bpt-gpustm-kernel-tree.cuh:150-224). */
static void split_inner(bto_tree *t, uint32_t n, uint32_t parent, uint32_t pslot) {
    const uint32_t mid = (BTO_ORDER - 2) / 2; /* 15 */
    uint32_t lvl = n_level(t, n);
    uint64_t up = t->keys[n][mid];
    uint32_t r = alloc_node(t);
    for (uint32_t i = 0; i < mid; i++) {
        t->keys[r][i] = t->keys[n][mid + 1 + i];
        t->keys[n][mid + 1 + i] = BTO_KEY_MAX;
    }
    for (uint32_t i = 0; i <= mid; i++) {
        t->vals[r][i] = t->vals[n][mid + 1 + i];
        t->vals[n][mid + 1 + i] = 0;
    }
    t->keys[n][mid] = BTO_KEY_MAX;
    n_set_info(t, n, mid, lvl);
    n_set_info(t, r, mid, lvl);
    t->low[r] = up;
    t->inner_splits++;
    if (parent == BTO_NIL) new_root(t, n, up, r, lvl + 1);
    else insert_separator(t, parent, pslot, up, r);
}

/* one insert under the reference's rules: descend, splitting every full inner
 * node on the way and restarting (src/gpu-stm-tree-v39/bpt-gpustm-kernel.cu:136-190),
 * then update in place / shift-insert / split 16-16
 * (src/gpu-stm-tree-v39/bpt-gpustm-kernel-tree.cuh:348-467). */
int bto_insert(bto_tree *t, uint64_t key, uint64_t val, uint64_t *old_val) {
    if (key == BTO_KEY_MAX) return BTO_REJECTED;
    if (t->root == BTO_NIL) { /* CREATE_NEW_TREE: empty leaf, fence MAX_KEY */
        uint32_t r = alloc_node(t);
        n_set_info(t, r, 0, 0);
        t->vals[r][31] = BTO_KEY_MAX;
        t->low[r] = 0;
        t->root = r;
    }
restart:;
    uint32_t parent = BTO_NIL, pslot = 0, n = t->root;
    for (;;) {
        uint32_t lvl = n_level(t, n), sz = n_size(t, n);
        if (lvl > 0 && sz == BTO_MAX_KEYS) {
            split_inner(t, n, parent, pslot);
            goto restart;
        }
        if (lvl == 0) break;
        uint32_t c = upper_slot(t->keys[n], sz, key);
        parent = n;
        pslot = c;
        n = (uint32_t)t->vals[n][c];
    }
    uint32_t sz = n_size(t, n);
    uint32_t p = lower_slot(t->keys[n], sz, key);
    if (p < sz && t->keys[n][p] == key) {
        if (old_val) *old_val = t->vals[n][p];
        t->vals[n][p] = val;
        return BTO_FOUND;
    }
    if (sz < BTO_MAX_KEYS) {
        for (uint32_t i = sz; i > p; i--) {
            t->keys[n][i] = t->keys[n][i - 1];
            t->vals[n][i] = t->vals[n][i - 1];
        }
        t->keys[n][p] = key;
        t->vals[n][p] = val;
        n_set_info(t, n, sz + 1, 0);
        t->n_keys++;
        return BTO_ABSENT;
    }
    /* full leaf: 31 keys + 1 -> 16 | 16, up = first key of the right half */
    uint64_t tk[BTO_ORDER], tv[BTO_ORDER];
    for (uint32_t i = 0, j = 0; i < BTO_ORDER; i++) {
        if (i == p) { tk[i] = key; tv[i] = val; }
        else { tk[i] = t->keys[n][j]; tv[i] = t->vals[n][j]; j++; }
    }
    const uint32_t half = BTO_ORDER / 2;
    uint64_t fence = t->vals[n][31];
    uint32_t r = alloc_node(t);
    for (uint32_t i = 0; i < BTO_ORDER - 1; i++) {
        t->keys[n][i] = i < half ? tk[i] : BTO_KEY_MAX;
        t->vals[n][i] = i < half ? tv[i] : 0;
        t->keys[r][i] = i < half ? tk[half + i] : BTO_KEY_MAX;
        t->vals[r][i] = i < half ? tv[half + i] : 0;
    }
    uint64_t up = tk[half];
    t->vals[n][31] = up;
    t->vals[r][31] = fence;
    n_set_info(t, n, half, 0);
    n_set_info(t, r, half, 0);
    t->low[r] = up;
    t->n_keys++;
    t->leaf_splits++;
    if (parent == BTO_NIL) new_root(t, n, up, r, 1);
    else insert_separator(t, parent, pslot, up, r);
    return BTO_ABSENT;
}

int bto_delete(bto_tree *t, uint64_t key, uint64_t *old_val) {
    if (key == BTO_KEY_MAX) return BTO_REJECTED;
    if (t->root == BTO_NIL) return BTO_ABSENT;
    uint32_t n = find_leaf(t, key, NULL, NULL);
    uint32_t sz = n_size(t, n);
    uint32_t p = lower_slot(t->keys[n], sz, key);
    if (p >= sz || t->keys[n][p] != key) return BTO_ABSENT;
    if (old_val) *old_val = t->vals[n][p];
    for (uint32_t i = p; i + 1 < sz; i++) {
        t->keys[n][i] = t->keys[n][i + 1];
        t->vals[n][i] = t->vals[n][i + 1];
    }
    t->keys[n][sz - 1] = BTO_KEY_MAX;
    t->vals[n][sz - 1] = 0;
    n_set_info(t, n, sz - 1, 0);
    t->n_keys--;
    return BTO_FOUND;
}

/* ------------------------------------------------------------------------ */
/* stable LSD radix sort, 8-bit digits, constant digits skipped */
void bto_sort_pairs(const uint64_t *keys, size_t n, uint64_t *keys_out, uint32_t *idx_out) {
    uint64_t *ka = (uint64_t *)malloc(sizeof(uint64_t) * (n ? n : 1));
    uint32_t *ia = (uint32_t *)malloc(sizeof(uint32_t) * (n ? n : 1));
    uint64_t *kb = keys_out;
    uint32_t *ib = idx_out;
    memcpy(ka, keys, sizeof(uint64_t) * n);
    for (size_t i = 0; i < n; i++) ia[i] = (uint32_t)i;
    size_t (*cnt)[256] = (size_t(*)[256])calloc(8, sizeof(size_t) * 256);
    for (size_t i = 0; i < n; i++)
        for (int d = 0; d < 8; d++) cnt[d][(ka[i] >> (8 * d)) & 0xff]++;
    int in_a = 1;
    for (int d = 0; d < 8; d++) {
        int trivial = 0;
        for (int b = 0; b < 256; b++) if (cnt[d][b] == n) trivial = 1;
        if (trivial) continue;
        size_t off[256], s = 0;
        for (int b = 0; b < 256; b++) { off[b] = s; s += cnt[d][b]; }
        uint64_t *sk = in_a ? ka : kb, *dk = in_a ? kb : ka;
        uint32_t *si = in_a ? ia : ib, *di = in_a ? ib : ia;
        for (size_t i = 0; i < n; i++) {
            size_t o = off[(sk[i] >> (8 * d)) & 0xff]++;
            dk[o] = sk[i];
            di[o] = si[i];
        }
        in_a = !in_a;
    }
    if (in_a) {
        memcpy(keys_out, ka, sizeof(uint64_t) * n);
        memcpy(idx_out, ia, sizeof(uint32_t) * n);
    }
    free(cnt);
    free(ka);
    free(ia);
}

/* ------------------------------------------------------------------------ */
/* Bulk loader (no counterpart in the reference, which builds by inserting).
 * Rule: n_leaves = ceil(m / leaf_fill) with the m keys spread evenly (the
 * first m % n_leaves leaves get one more); every inner level groups its
 * children the same way with inner_fill + 1 children per node, until one
 * node is left.  The leftmost node of each level has low fence 0.  Node ids:
 * leaves first, then each level bottom-up. */
static void build_levels(bto_tree *t, uint32_t first, uint32_t count, uint32_t level) {
    while (count > 1) {
        uint32_t per = t->inner_fill + 1;
        uint32_t nn = (count + per - 1) / per;
        uint32_t base = count / nn, rem = count % nn;
        uint32_t next_first = t->n_nodes;
        uint32_t c = first;
        for (uint32_t j = 0; j < nn; j++) {
            uint32_t k = base + (j < rem ? 1 : 0);
            uint32_t p = alloc_node(t);
            for (uint32_t i = 0; i < k; i++) {
                t->vals[p][i] = c + i;
                if (i > 0) t->keys[p][i - 1] = t->low[c + i];
            }
            t->low[p] = t->low[c];
            n_set_info(t, p, k - 1, level);
            c += k;
        }
        first = next_first;
        count = nn;
        level++;
    }
    t->root = first;
}

int bto_bulk_build(bto_tree *t, const uint64_t *keys, const uint64_t *vals, size_t n) {
    bto_clear(t);
    for (size_t i = 0; i < n; i++) if (keys[i] == BTO_KEY_MAX) return -1;
    if (n == 0) return 0;
    uint64_t *sk = (uint64_t *)malloc(sizeof(uint64_t) * n);
    uint32_t *si = (uint32_t *)malloc(sizeof(uint32_t) * n);
    bto_sort_pairs(keys, n, sk, si);
    /* dedupe: the last occurrence (largest input position) of each key wins */
    size_t m = 0;
    for (size_t i = 0; i < n; i++) {
        if (i + 1 < n && sk[i + 1] == sk[i]) continue;
        sk[m] = sk[i];
        si[m] = si[i];
        m++;
    }
    uint32_t nl = (uint32_t)((m + t->leaf_fill - 1) / t->leaf_fill);
    uint32_t base = (uint32_t)(m / nl), rem = (uint32_t)(m % nl);
    size_t pos = 0;
    for (uint32_t j = 0; j < nl; j++) {
        uint32_t k = base + (j < rem ? 1 : 0);
        uint32_t l = alloc_node(t);
        for (uint32_t i = 0; i < k; i++) {
            t->keys[l][i] = sk[pos + i];
            t->vals[l][i] = vals[si[pos + i]];
        }
        t->low[l] = j == 0 ? 0 : sk[pos];
        t->vals[l][31] = (j + 1 < nl) ? sk[pos + k] : BTO_KEY_MAX;
        n_set_info(t, l, k, 0);
        pos += k;
    }
    build_levels(t, 0, nl, 1);
    t->n_keys = m;
    free(sk);
    free(si);
    return 0;
}

/* ------------------------------------------------------------------------ */
/* segmented merge engine (deterministic batched insert; no counterpart in
 * the reference).  Inputs: unique new keys in ascending order that are all
 * absent from the tree, with their values.
 * Leaf rule: a leaf that would hold m > 31 keys is cut into
 * p = ceil(m / leaf_fill) leaves of even size (first m % p get one more);
 * the original leaf keeps the first piece.  For a single extra key on a full
 * leaf this is the reference's 16 | 16 split.
 * Inner rule: a node whose merged separator count s exceeds 31 is cut into
 * q = ceil((s+1) / (inner_fill+1)) nodes by children, spread evenly; the key
 * between two pieces moves up.  An overflowing root is rebuilt upward with
 * the bulk-level rule. */
typedef struct entry { uint64_t key; uint32_t child; uint32_t parent; uint32_t pslot; } entry;

static void merge_engine(bto_tree *t, const uint64_t *nk, const uint64_t *nv, size_t m) {
    if (m == 0) return;
    if (t->root == BTO_NIL) { /* an empty leaf root to merge into (CREATE_NEW_TREE) */
        uint32_t r = alloc_node(t);
        n_set_info(t, r, 0, 0);
        t->vals[r][31] = BTO_KEY_MAX;
        t->low[r] = 0;
        t->root = r;
    }
    uint32_t H = n_level(t, t->root) + 1;
    /* path of every new key: path[l] = node at level l, slots[l] = child slot */
    uint32_t *path = (uint32_t *)malloc(sizeof(uint32_t) * H * m);
    uint32_t *slot = (uint32_t *)malloc(sizeof(uint32_t) * H * m);
    for (size_t i = 0; i < m; i++) find_leaf(t, nk[i], path + i * H, slot + i * H);

    /* leaf level */
    entry *ent = (entry *)malloc(sizeof(entry) * (m + 1));
    size_t ne = 0;
    size_t i = 0;
    uint64_t *bk = NULL, *bv = NULL;
    size_t bcap = 0;
    while (i < m) {
        uint32_t leaf = path[i * H];
        size_t j = i;
        while (j < m && path[j * H] == leaf) j++;
        uint32_t sz = n_size(t, leaf);
        size_t tot = sz + (j - i);
        if (tot > bcap) {
            bcap = tot * 2;
            bk = (uint64_t *)realloc(bk, sizeof(uint64_t) * bcap);
            bv = (uint64_t *)realloc(bv, sizeof(uint64_t) * bcap);
        }
        size_t a = 0, b = i, o = 0;
        while (a < sz || b < j) {
            if (b >= j || (a < sz && t->keys[leaf][a] < nk[b])) { bk[o] = t->keys[leaf][a]; bv[o] = t->vals[leaf][a]; a++; }
            else { bk[o] = nk[b]; bv[o] = nv[b]; b++; }
            o++;
        }
        uint64_t fence = t->vals[leaf][31];
        if (tot <= BTO_MAX_KEYS) {
            for (uint32_t q = 0; q < BTO_MAX_KEYS; q++) {
                t->keys[leaf][q] = q < tot ? bk[q] : BTO_KEY_MAX;
                t->vals[leaf][q] = q < tot ? bv[q] : 0;
            }
            n_set_info(t, leaf, (uint32_t)tot, 0);
        } else {
            size_t p = (tot + t->leaf_fill - 1) / t->leaf_fill;
            size_t base = tot / p, rem = tot % p, s = 0;
            uint32_t prev = leaf;
            for (size_t c = 0; c < p; c++) {
                size_t k = base + (c < rem ? 1 : 0);
                uint32_t nd = c == 0 ? leaf : alloc_node(t);
                for (uint32_t q = 0; q < BTO_MAX_KEYS; q++) {
                    t->keys[nd][q] = q < k ? bk[s + q] : BTO_KEY_MAX;
                    t->vals[nd][q] = q < k ? bv[s + q] : 0;
                }
                n_set_info(t, nd, (uint32_t)k, 0);
                if (c > 0) {
                    t->low[nd] = bk[s];
                    t->vals[prev][31] = bk[s];
                    ent[ne].key = bk[s];
                    ent[ne].child = nd;
                    ent[ne].parent = H > 1 ? path[i * H + 1] : BTO_NIL;
                    ent[ne].pslot = 0;
                    ne++;
                    t->leaf_splits++;
                }
                prev = nd;
                s += k;
            }
            t->vals[prev][31] = fence;
        }
        i = j;
    }
    t->n_keys += m;

    /* inner levels */
    uint32_t level = 1;
    while (ne > 0) {
        if (level >= H) {
            /* the old root split: rebuild upward from [root pieces] */
            uint32_t cnt = (uint32_t)ne + 1;
            uint32_t *kids = (uint32_t *)malloc(sizeof(uint32_t) * cnt);
            kids[0] = t->root;
            for (size_t e = 0; e < ne; e++) kids[e + 1] = ent[e].child;
            /* build_levels needs contiguous ids: copy pieces into fresh contiguous nodes is
             * not needed; build with an explicit child list instead */
            uint32_t lvl = level;
            while (cnt > 1) {
                uint32_t per = t->inner_fill + 1;
                uint32_t nn = (cnt + per - 1) / per;
                uint32_t base = cnt / nn, rem = cnt % nn;
                uint32_t *up = (uint32_t *)malloc(sizeof(uint32_t) * nn);
                uint32_t c = 0;
                for (uint32_t q = 0; q < nn; q++) {
                    uint32_t k = base + (q < rem ? 1 : 0);
                    uint32_t p = alloc_node(t);
                    for (uint32_t x = 0; x < k; x++) {
                        t->vals[p][x] = kids[c + x];
                        if (x > 0) t->keys[p][x - 1] = t->low[kids[c + x]];
                    }
                    t->low[p] = t->low[kids[c]];
                    n_set_info(t, p, k - 1, lvl);
                    t->new_roots++;
                    t->inner_splits++;
                    up[q] = p;
                    c += k;
                }
                free(kids);
                kids = up;
                cnt = nn;
                lvl++;
            }
            t->root = kids[0];
            free(kids);
            break;
        }
        /* group entries by parent (entries are in key order, parents too) */
        entry *next = (entry *)malloc(sizeof(entry) * (ne + 1));
        size_t nn = 0, e = 0;
        while (e < ne) {
            uint32_t P = ent[e].parent;
            size_t f = e;
            while (f < ne && ent[f].parent == P) f++;
            uint32_t sz = n_size(t, P);
            size_t tot = sz + (f - e);
            size_t need = tot + 1;
            if (need > bcap) {
                bcap = need * 2;
                bk = (uint64_t *)realloc(bk, sizeof(uint64_t) * bcap);
                bv = (uint64_t *)realloc(bv, sizeof(uint64_t) * bcap);
            }
            /* merged keys bk[0..tot), children bv[0..tot] */
            size_t a = 0, b = e, o = 0;
            bv[0] = t->vals[P][0];
            while (a < sz || b < f) {
                if (b >= f || (a < sz && t->keys[P][a] < ent[b].key)) {
                    bk[o] = t->keys[P][a];
                    bv[o + 1] = t->vals[P][a + 1];
                    a++;
                } else {
                    bk[o] = ent[b].key;
                    bv[o + 1] = ent[b].child;
                    b++;
                }
                o++;
            }
            uint32_t lvl = n_level(t, P);
            if (tot <= BTO_MAX_KEYS) {
                for (uint32_t q = 0; q < BTO_MAX_KEYS; q++) t->keys[P][q] = q < tot ? bk[q] : BTO_KEY_MAX;
                for (uint32_t q = 0; q < BTO_ORDER; q++) t->vals[P][q] = q <= tot ? bv[q] : 0;
                n_set_info(t, P, (uint32_t)tot, lvl);
            } else {
                size_t ch = tot + 1;
                size_t per = t->inner_fill + 1;
                size_t q = (ch + per - 1) / per;
                size_t base = ch / q, rem = ch % q, s = 0;
                for (size_t c = 0; c < q; c++) {
                    size_t k = base + (c < rem ? 1 : 0);
                    uint32_t nd = c == 0 ? P : alloc_node(t);
                    for (uint32_t x = 0; x < BTO_ORDER; x++) t->vals[nd][x] = x < k ? bv[s + x] : 0;
                    for (uint32_t x = 0; x < BTO_MAX_KEYS; x++)
                        t->keys[nd][x] = (x + 1 < k) ? bk[s + x] : BTO_KEY_MAX;
                    n_set_info(t, nd, (uint32_t)(k - 1), lvl);
                    if (c > 0) {
                        uint64_t sep = bk[s - 1];
                        t->low[nd] = sep;
                        next[nn].key = sep;
                        next[nn].child = nd;
                        next[nn].parent = BTO_NIL;
                        next[nn].pslot = (uint32_t)(f - 1); /* any entry index of this group */
                        nn++;
                        t->inner_splits++;
                    }
                    s += k;
                }
            }
            e = f;
        }
        /* parents of the next level: look them up through the path of the entry's
         * original key (every entry at this level derived from some new key) */
        if (level + 1 < H) {
            /* find the grandparent by descending from the root to the level + 1 */
            for (size_t x = 0; x < nn; x++) {
                uint32_t n = t->root, l = n_level(t, n);
                uint64_t key = next[x].key;
                while (l > level + 1) {
                    uint32_t c = upper_slot(t->keys[n], n_size(t, n), key);
                    n = (uint32_t)t->vals[n][c];
                    l--;
                }
                next[x].parent = n;
            }
        }
        free(ent);
        ent = next;
        ne = nn;
        level++;
    }
    free(ent);
    free(path);
    free(slot);
    free(bk);
    free(bv);
}

/* ------------------------------------------------------------------------ */
/* batch execution */
void bto_execute_serial(bto_tree *t, const uint64_t *keys, const uint64_t *vals,
                        const uint8_t *ops, size_t n, uint64_t *out_vals, uint8_t *out_status) {
    for (size_t i = 0; i < n; i++) {
        uint64_t v = 0;
        int st;
        if (ops[i] == BTO_OP_GET) st = bto_get(t, keys[i], &v);
        else if (ops[i] == BTO_OP_INSERT) st = bto_insert(t, keys[i], vals[i], &v);
        else if (ops[i] == BTO_OP_DELETE) st = bto_delete(t, keys[i], &v);
        else st = BTO_REJECTED;
        out_vals[i] = st == BTO_FOUND ? v : 0;
        out_status[i] = (uint8_t)st;
    }
}

typedef struct lookup_job {
    const bto_tree *t;
    const uint64_t *ukeys;
    uint64_t *uval;
    uint8_t *ust;
    size_t lo, hi;
} lookup_job;

static void *lookup_worker(void *arg) {
    lookup_job *j = (lookup_job *)arg;
    for (size_t u = j->lo; u < j->hi; u++) {
        uint64_t v = 0;
        j->ust[u] = (uint8_t)bto_get(j->t, j->ukeys[u], &v);
        j->uval[u] = v;
    }
    return NULL;
}

/* v38 batch meaning (src/gpu-stm-tree-v38/bpt-gpustm-kernel-aux.cuh:16-56),
 * extended to DELETE: within a run of equal keys in stable order, each
 * request sees the tree's pre-batch state until the first write (INSERT or
 * DELETE), and afterwards the state the latest write before it left (the
 * value of an INSERT, or absent after a DELETE); the run collapses to its last
 * write, or to a GET.  The batch then applies its deletes, then its inserts. */
void bto_execute_merged(bto_tree *t, const uint64_t *keys, const uint64_t *vals,
                        const uint8_t *ops, size_t n, uint64_t *out_vals, uint8_t *out_status,
                        int engine, int n_threads) {
    if (n == 0) return;
    uint64_t *sk = (uint64_t *)malloc(sizeof(uint64_t) * n);
    uint32_t *si = (uint32_t *)malloc(sizeof(uint32_t) * n);
    bto_sort_pairs(keys, n, sk, si);
    /* unique keys */
    uint64_t *uk = (uint64_t *)malloc(sizeof(uint64_t) * n);
    size_t *ustart = (size_t *)malloc(sizeof(size_t) * (n + 1));
    size_t nu = 0;
    for (size_t i = 0; i < n; i++) {
        if (i == 0 || sk[i] != sk[i - 1]) { uk[nu] = sk[i]; ustart[nu] = i; nu++; }
    }
    ustart[nu] = n;
    uint64_t *uval = (uint64_t *)malloc(sizeof(uint64_t) * nu);
    uint8_t *ust = (uint8_t *)malloc(nu);
    if (n_threads < 1) n_threads = 1;
    if (n_threads == 1 || nu < 4096) {
        lookup_job j = {t, uk, uval, ust, 0, nu};
        lookup_worker(&j);
    } else {
        pthread_t *th = (pthread_t *)malloc(sizeof(pthread_t) * n_threads);
        lookup_job *jb = (lookup_job *)malloc(sizeof(lookup_job) * n_threads);
        for (int w = 0; w < n_threads; w++) {
            jb[w].t = t; jb[w].ukeys = uk; jb[w].uval = uval; jb[w].ust = ust;
            jb[w].lo = nu * w / n_threads; jb[w].hi = nu * (w + 1) / n_threads;
            pthread_create(&th[w], NULL, lookup_worker, &jb[w]);
        }
        for (int w = 0; w < n_threads; w++) pthread_join(th[w], NULL);
        free(th);
        free(jb);
    }
    /* resolve runs */
    uint64_t *ik = (uint64_t *)malloc(sizeof(uint64_t) * nu);
    uint64_t *iv = (uint64_t *)malloc(sizeof(uint64_t) * nu);
    uint64_t *nk = (uint64_t *)malloc(sizeof(uint64_t) * nu);
    uint64_t *nv = (uint64_t *)malloc(sizeof(uint64_t) * nu);
    uint64_t *dk = (uint64_t *)malloc(sizeof(uint64_t) * nu);
    size_t ni = 0, nnew = 0, nd = 0;
    for (size_t u = 0; u < nu; u++) {
        int have = 0, gone = 0;
        uint64_t cur = 0;
        int rejected_key = (uk[u] == BTO_KEY_MAX);
        for (size_t p = ustart[u]; p < ustart[u + 1]; p++) {
            uint32_t r = si[p];
            uint8_t op = ops[r];
            if (rejected_key || (op != BTO_OP_GET && op != BTO_OP_INSERT && op != BTO_OP_DELETE)) {
                out_status[r] = BTO_REJECTED;
                out_vals[r] = 0;
                continue;
            }
            if (!have) {
                out_status[r] = ust[u];
                out_vals[r] = ust[u] == BTO_FOUND ? uval[u] : 0;
            } else {
                out_status[r] = gone ? BTO_ABSENT : BTO_FOUND;
                out_vals[r] = gone ? 0 : cur;
            }
            if (op == BTO_OP_INSERT) { have = 1; gone = 0; cur = vals[r]; }
            else if (op == BTO_OP_DELETE) { have = 1; gone = 1; cur = 0; }
        }
        if (have && gone) {
            dk[nd++] = uk[u];
        } else if (have) {
            ik[ni] = uk[u]; iv[ni] = cur; ni++;
            if (ust[u] != BTO_FOUND) { nk[nnew] = uk[u]; nv[nnew] = cur; nnew++; }
        }
    }
    for (size_t x = 0; x < nd; x++) bto_delete(t, dk[x], NULL);
    free(dk);
    if (engine == BTO_ENGINE_MERGE) {
        /* updates in place, then the segmented merge of the new keys */
        for (size_t x = 0; x < ni; x++) {
            if (t->root != BTO_NIL) {
                uint32_t leaf = find_leaf(t, ik[x], NULL, NULL);
                uint32_t sz = n_size(t, leaf);
                uint32_t p = lower_slot(t->keys[leaf], sz, ik[x]);
                if (p < sz && t->keys[leaf][p] == ik[x]) t->vals[leaf][p] = iv[x];
            }
        }
        merge_engine(t, nk, nv, nnew);
    } else {
        for (size_t x = 0; x < ni; x++) bto_insert(t, ik[x], iv[x], NULL);
    }
    free(sk); free(si); free(uk); free(ustart); free(uval); free(ust);
    free(ik); free(iv); free(nk); free(nv);
}

/* ------------------------------------------------------------------------ */
/* inspection */
size_t bto_size(const bto_tree *t) { return (size_t)t->n_keys; }

typedef void (*leaf_fn)(const bto_tree *t, uint32_t leaf, void *ctx);
static void walk_leaves(const bto_tree *t, uint32_t n, leaf_fn fn, void *ctx) {
    if (n_level(t, n) == 0) { fn(t, n, ctx); return; }
    uint32_t sz = n_size(t, n);
    for (uint32_t c = 0; c <= sz; c++) walk_leaves(t, (uint32_t)t->vals[n][c], fn, ctx);
}

typedef struct dump_ctx { uint64_t *k, *v; size_t pos; uint32_t *sizes; uint64_t *lows; size_t cap; } dump_ctx;
static void dump_fn(const bto_tree *t, uint32_t leaf, void *c) {
    dump_ctx *d = (dump_ctx *)c;
    uint32_t sz = n_size(t, leaf);
    for (uint32_t i = 0; i < sz; i++) {
        if (d->k) d->k[d->pos + i] = t->keys[leaf][i];
        if (d->v) d->v[d->pos + i] = t->vals[leaf][i];
    }
    d->pos += sz;
}
void bto_dump(const bto_tree *t, uint64_t *keys, uint64_t *vals) {
    if (t->root == BTO_NIL) return;
    dump_ctx d = {keys, vals, 0, NULL, NULL, 0};
    walk_leaves(t, t->root, dump_fn, &d);
}
static void size_fn(const bto_tree *t, uint32_t leaf, void *c) {
    dump_ctx *d = (dump_ctx *)c;
    if (d->pos < d->cap) {
        if (d->sizes) d->sizes[d->pos] = n_size(t, leaf);
        if (d->lows) d->lows[d->pos] = t->low[leaf];
    }
    d->pos++;
}
size_t bto_leaf_sizes(const bto_tree *t, uint32_t *sizes, size_t cap) {
    if (t->root == BTO_NIL) return 0;
    dump_ctx d = {NULL, NULL, 0, sizes, NULL, cap};
    walk_leaves(t, t->root, size_fn, &d);
    return d.pos;
}
size_t bto_leaf_lows(const bto_tree *t, uint64_t *lows, size_t cap) {
    if (t->root == BTO_NIL) return 0;
    dump_ctx d = {NULL, NULL, 0, NULL, lows, cap};
    walk_leaves(t, t->root, size_fn, &d);
    return d.pos;
}

static void count_levels(const bto_tree *t, uint32_t n, uint64_t *counts, uint32_t cap) {
    uint32_t l = n_level(t, n);
    if (l < cap) counts[l]++;
    if (l == 0) return;
    uint32_t sz = n_size(t, n);
    for (uint32_t c = 0; c <= sz; c++) count_levels(t, (uint32_t)t->vals[n][c], counts, cap);
}
uint32_t bto_level_counts(const bto_tree *t, uint64_t *counts, uint32_t cap) {
    for (uint32_t i = 0; i < cap; i++) counts[i] = 0;
    if (t->root == BTO_NIL) return 0;
    count_levels(t, t->root, counts, cap);
    return n_level(t, t->root) + 1;
}

void bto_get_stats(const bto_tree *t, bto_stats *s) {
    memset(s, 0, sizeof(*s));
    s->n_keys = t->n_keys;
    s->n_nodes = t->n_nodes;
    s->leaf_splits = t->leaf_splits;
    s->inner_splits = t->inner_splits;
    s->new_roots = t->new_roots;
    if (t->root == BTO_NIL) return;
    s->root_level = n_level(t, t->root);
    s->height = s->root_level + 1;
    s->n_leaves = bto_leaf_sizes(t, NULL, 0);
}

static int check_node(const bto_tree *t, uint32_t n, uint64_t lo, uint64_t hi, uint32_t level, int is_root) {
    if (n_level(t, n) != level) return 1;
    uint32_t sz = n_size(t, n);
    if (sz > BTO_MAX_KEYS) return 2;
    if (t->low[n] != lo) return 3;
    for (uint32_t i = 0; i < sz; i++) {
        if (t->keys[n][i] < lo || t->keys[n][i] >= hi) return 4;
        if (i && t->keys[n][i - 1] >= t->keys[n][i]) return 5;
    }
    for (uint32_t i = sz; i < BTO_MAX_KEYS; i++) if (t->keys[n][i] != BTO_KEY_MAX) return 6;
    if (level == 0) {
        if (t->vals[n][31] != hi) return 7;
        return 0;
    }
    if (!is_root && sz == 0 && level > 0) return 8;
    for (uint32_t c = 0; c <= sz; c++) {
        uint64_t clo = c == 0 ? lo : t->keys[n][c - 1];
        uint64_t chi = c == sz ? hi : t->keys[n][c];
        int r = check_node(t, (uint32_t)t->vals[n][c], clo, chi, level - 1, 0);
        if (r) return r;
    }
    return 0;
}
int bto_check(const bto_tree *t) {
    if (t->root == BTO_NIL) return 0;
    return check_node(t, t->root, 0, BTO_KEY_MAX, n_level(t, t->root), 1);
}

/* ------------------------------------------------------------------------ */
/* learned predictor reference: 1 -> 32 (ReLU) -> 1 MLP, MSE loss */
double bto_mlp_forward(const float *p, double x) {
    double y = p[96];
    for (int j = 0; j < 32; j++) {
        double h = (double)p[j] * x + (double)p[32 + j];
        if (h > 0) y += (double)p[64 + j] * h;
    }
    return y;
}

double bto_mlp_grad(const float *p, const float *x, const float *y, size_t n, double *g) {
    for (int i = 0; i < 97; i++) g[i] = 0;
    double loss = 0;
    for (size_t i = 0; i < n; i++) {
        double xi = x[i];
        double h[32];
        double out = p[96];
        for (int j = 0; j < 32; j++) {
            double a = (double)p[j] * xi + (double)p[32 + j];
            h[j] = a > 0 ? a : 0;
            out += (double)p[64 + j] * h[j];
        }
        double d = out - (double)y[i];
        loss += d * d;
        double go = 2.0 * d / (double)n;
        g[96] += go;
        for (int j = 0; j < 32; j++) {
            g[64 + j] += go * h[j];
            if (h[j] > 0) {
                double gh = go * (double)p[64 + j];
                g[j] += gh * xi;
                g[32 + j] += gh;
            }
        }
    }
    return loss / (double)(n ? n : 1);
}

/* ------------------------------------------------------------------------ */
/* workload generators.  mix64 is the SplitMix64 output function (Steele,
 * Lea, Flood 2014; public-domain constants by S. Vigna). */
uint64_t bto_mix64(uint64_t z) {
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
}
uint64_t bto_rand(uint64_t seed, uint64_t i, uint64_t j) {
    return bto_mix64(bto_mix64(seed) + 0x9E3779B97F4A7C15ull * (i * 16 + j + 1));
}
uint64_t bto_value_of(uint64_t key) { return key ^ 0x9E3779B97F4A7C15ull; }

static double unit_open(uint64_t r) { /* (0, 1] */
    return ((double)(r >> 11) + 1.0) * (1.0 / 9007199254740992.0);
}

/* Zipf(s) over ranks 1..N by rejection-inversion (Hormann & Derflinger 1996). */
typedef struct zipf_t { double s, n, hx1, hn, sq; } zipf_t;
static double zh(const zipf_t *z, double x) { return exp(-z->s * log(x)); }
static double zhint(const zipf_t *z, double x) { /* integral of x^-s: (x^(1-s) - 1) / (1 - s) */
    double lx = log(x), t = (1.0 - z->s) * lx;
    double f = fabs(t) > 1e-8 ? expm1(t) / t : 1.0 + t * 0.5 * (1.0 + t / 3.0);
    return f * lx;
}
static double zhinv(const zipf_t *z, double x) {
    double t = x * (1.0 - z->s);
    if (t < -1.0) t = -1.0;
    double f = fabs(t) > 1e-8 ? log1p(t) / t : 1.0 - t * (0.5 - t / 3.0);
    return exp(f * x);
}
static void zipf_init(zipf_t *z, double s, double n) {
    z->s = s;
    z->n = n;
    z->hx1 = zhint(z, 1.5) - 1.0;
    z->hn = zhint(z, n + 0.5);
    z->sq = 2.0 - zhinv(z, zhint(z, 2.5) - zh(z, 2.0));
}
static uint64_t zipf_draw(const zipf_t *z, uint64_t seed, uint64_t i, uint64_t j0) {
    for (uint64_t a = 0; a < 64; a++) {
        double u01 = unit_open(bto_rand(seed, i, j0 + a));
        double u = z->hn + u01 * (z->hx1 - z->hn);
        double x = zhinv(z, u);
        double k = floor(x + 0.5);
        if (k < 1) k = 1;
        if (k > z->n) k = z->n;
        if (k - x <= z->sq || u >= zhint(z, k + 0.5) - zh(z, k)) return (uint64_t)k;
    }
    return 1;
}
static uint64_t rank_key(uint64_t rank) { return bto_mix64(rank ^ 0x2545F4914F6CDD1Dull) >> 1; }

static uint64_t clamp_key(double v) {
    if (!(v >= 0)) return 0;
    if (v >= 18446744073709549568.0) return 0xFFFFFFFFFFFFF7FFull;
    return (uint64_t)llround(v);
}

static uint64_t draw_key(int dist, const zipf_t *z, uint64_t seed, uint64_t i, uint64_t j0) {
    switch (dist) {
    case 1: return rank_key(zipf_draw(z, seed, i, j0));
    case 2: {
        double u1 = unit_open(bto_rand(seed, i, j0)), u2 = unit_open(bto_rand(seed, i, j0 + 1));
        double g = sqrt(-2.0 * log(u1)) * cos(6.283185307179586 * u2);
        return clamp_key(4611686018427387904.0 + 288230376151711744.0 * g);
    }
    case 3: {
        double u1 = unit_open(bto_rand(seed, i, j0)), u2 = unit_open(bto_rand(seed, i, j0 + 1));
        return clamp_key(72057594037927936.0 * (-log(u1) - log(u2)));
    }
    default: return bto_rand(seed, i, j0) >> 1;
    }
}

void bto_gen_keys(int dist, uint64_t seed, size_t n, uint64_t *keys) {
    zipf_t z;
    zipf_init(&z, 0.99, 4294967296.0);
    for (size_t i = 0; i < n; i++) {
        /* Zipf tree keys: the n most popular ranks, hashed */
        if (dist == 1) keys[i] = rank_key((uint64_t)i + 1);
        else keys[i] = draw_key(dist, &z, seed, i, 0);
    }
}

void bto_gen_requests(int dist, uint64_t seed, const uint64_t *tree_keys, size_t n_tree,
                      size_t n, uint32_t search_pct, uint64_t *keys, uint64_t *vals, uint8_t *ops) {
    zipf_t z;
    zipf_init(&z, 0.99, 4294967296.0);
    for (size_t i = 0; i < n; i++) {
        uint64_t r0 = bto_rand(seed, i, 0);
        if (r0 % 100 < search_pct) {
            ops[i] = BTO_OP_GET;
            vals[i] = 0;
            uint64_t r1 = bto_rand(seed, i, 1);
            if ((r1 & 1) && n_tree > 0) keys[i] = tree_keys[(r1 >> 1) % n_tree];
            else keys[i] = draw_key(dist, &z, seed, i, 2);
        } else {
            ops[i] = BTO_OP_INSERT;
            keys[i] = draw_key(dist, &z, seed ^ 0x5851F42D4C957F2Dull, i, 2);
            vals[i] = bto_value_of(keys[i]);
        }
    }
}
