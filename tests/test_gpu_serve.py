"""Serving loop (continuous batching): a batch's answers are the same alone and
in a mix of batches running together (bit-exact; the batches touch disjoint
keys), many batches overlap on the device, admission reports busy when the
arena is full, and the persistent kernel is relaunched after idling out."""
import time

import numpy as np
import pytest

import eirene_b200 as E
from oracle import oracle as O
from tests.helpers import dev, dump

pytestmark = pytest.mark.gpu

N_TREE = 200_000


def build(seed=1):
    keys = O.gen_keys("uniform", seed, N_TREE)
    vals = O.value_of(keys)
    t = E.BTree(max_keys=1 << 21, max_batch=1 << 16)
    t.bulk_build(dev(keys), dev(vals))
    return t, keys, vals


def make_batch(tree_keys, part, n, search_frac, seed):
    """Requests over a private key range: GETs of tree keys in `part`, GETs of
    absent keys and INSERTs of fresh keys, all distinct within the batch."""
    rng = np.random.default_rng(seed)
    lo, hi = part
    n_get_hit = int(n * search_frac / 2)
    n_get_miss = int(n * search_frac) - n_get_hit
    n_ins = n - n_get_hit - n_get_miss
    hits = rng.choice(tree_keys[lo:hi], n_get_hit, replace=False)
    fresh = (O.gen_keys("uniform", 10_000 + seed, n_get_miss + n_ins + 64))
    fresh = np.setdiff1d(fresh, tree_keys)[: n_get_miss + n_ins]
    fresh = rng.permutation(fresh)
    keys = np.concatenate([hits, fresh])
    ops = np.concatenate([np.ones(n_get_hit + n_get_miss, np.uint8), np.zeros(n_ins, np.uint8)])
    perm = rng.permutation(n)
    keys, ops = keys[perm], ops[perm]
    vals = np.where(ops == 0, keys * np.uint64(5) + np.uint64(seed), np.uint64(0)).astype(np.uint64)
    return keys, vals, ops


def oracle_answers(keys_tree, vals_tree, batches):
    o = O.OracleTree()
    o.bulk_build(keys_tree, vals_tree)
    outs = [o.execute_serial(*b) for b in batches]
    return outs, o


def serve_all(server, batches, timeout_s=120, tickets_out=None):
    outs = [(np.zeros(b[0].size, np.uint64), np.zeros(b[0].size, np.uint8)) for b in batches]
    tickets = [None] * len(batches)
    t0 = time.time()
    i = 0
    while i < len(batches):
        tk = server.submit(*batches[i], *outs[i])
        if tk is None:  # busy: wait for the oldest unfinished batch
            for j in range(i):
                if tickets[j] is not None and not server.poll(tickets[j]):
                    server.wait(tickets[j])
                    break
            assert time.time() - t0 < timeout_s
            continue
        tickets[i] = tk
        i += 1
    for tk in tickets:
        server.wait(tk)
    if tickets_out is not None:
        tickets_out.extend(tickets)
    return outs


def test_alone_equals_in_mix(gpu):
    t1, keys, vals = build()
    parts = [(0, 50_000), (50_000, 100_000), (100_000, 150_000), (150_000, 200_000)]
    A = make_batch(np.sort(keys), parts[0], 20_000, 0.7, seed=1)
    # the first batch of the mix is large, so the others arrive while it runs
    mix = [make_batch(np.sort(keys), parts[k], 90_000 if k == 1 else 30_000, 0.5 + 0.15 * k, seed=10 + k)
           for k in (1, 2, 3)]
    s1 = E.Server(t1)
    alone = serve_all(s1, [A])[0]
    s1.stop()
    t2, _, _ = build()
    s2 = E.Server(t2)
    batches = [mix[0], A, mix[1], mix[2]]
    tickets = []
    res = serve_all(s2, batches, tickets_out=tickets)
    st = s2.stats()
    # the batches were on the device together: A's span (first claimed chunk
    # to completion, device clock) overlaps another batch's span
    spans = [s2.batch_times(tk) for tk in tickets]
    s2.stop()
    a0, a1 = spans[1]
    assert all(s < e for s, e in spans)
    assert any(max(a0, s) < min(a1, e) for j, (s, e) in enumerate(spans) if j != 1), spans
    inmix = res[1]
    assert (alone[0] == inmix[0]).all() and (alone[1] == inmix[1]).all()
    ref, o = oracle_answers(keys, vals, batches)
    for (gv, gs), (ov, os_) in zip(res, ref):
        assert (gs == os_).all() and (gv == ov).all()
    gk, gvv = dump(t2)
    ok, ovv = o.dump()
    assert (gk == ok).all() and (gvv == ovv).all()
    assert st["batches"] == 4 and st["p99_ms"] >= st["p50_ms"] > 0


def test_many_overlapping_batches(gpu):
    t, keys, vals = build(seed=2)
    sk = np.sort(keys)
    rng = np.random.default_rng(3)
    batches = []
    for b in range(40):
        n = int(2 ** rng.uniform(10, 13))
        lo = b * 5000
        batches.append(make_batch(sk, (lo, lo + 5000), n, rng.uniform(0.5, 1.0), seed=100 + b))
    s = E.Server(t, arena_bytes=1 << 22, max_batches=16)
    res = serve_all(s, batches)
    st = s.stats()
    s.stop()
    ref, o = oracle_answers(keys, vals, batches)
    for (gv, gs), (ov, os_) in zip(res, ref):
        assert (gs == os_).all() and (gv == ov).all()
    assert st["batches"] == 40
    gk, gvv = dump(t)
    ok, ovv = o.dump()
    assert (gk == ok).all() and (gvv == ovv).all()


def test_admission_busy_when_arena_full(gpu):
    t, keys, vals = build(seed=4)
    sk = np.sort(keys)
    s = E.Server(t, arena_bytes=100_000, max_batches=8)
    b = [make_batch(sk, (i * 1000, i * 1000 + 1000), 1000, 0.9, seed=200 + i) for i in range(6)]
    outs = [(np.zeros(1000, np.uint64), np.zeros(1000, np.uint8)) for _ in b]
    tickets = []
    busy = False
    for i in range(6):
        tk = s.submit(*b[i], *outs[i])
        if tk is None:
            busy = True
            break
        tickets.append(tk)
    assert busy and 1 <= len(tickets) < 6
    for tk in tickets:
        s.wait(tk)
    tk = s.submit(*b[len(tickets)], *outs[len(tickets)])
    assert tk is not None
    s.wait(tk)
    s.stop()


def test_relaunch_after_idle(gpu):
    t, keys, vals = build(seed=5)
    sk = np.sort(keys)
    s = E.Server(t, idle_us=500)
    b1 = make_batch(sk, (0, 10_000), 5000, 0.8, seed=300)
    b2 = make_batch(sk, (10_000, 20_000), 5000, 0.8, seed=301)
    r1 = serve_all(s, [b1])
    time.sleep(0.05)  # the persistent kernel idles out
    r2 = serve_all(s, [b2])
    st = s.stats()
    s.stop()
    assert st["kernel_launches"] >= 2
    ref, _ = oracle_answers(keys, vals, [b1, b2])
    for (gv, gs), (ov, os_) in zip(r1 + r2, ref):
        assert (gs == os_).all() and (gv == ov).all()


def test_gets_beside_splitting_inserts(gpu):
    # reader batches run while writer batches split the leaves they read: a
    # GET of a key that is in the tree throughout must find it with its value
    # (the group lookup's seqlock check sends torn reads to the warp path),
    # and a GET of a key being inserted sees it absent or with its new value
    t, keys, vals = build(seed=7)
    rng = np.random.default_rng(8)
    fresh = np.setdiff1d(O.gen_keys("uniform", 777, 260_000), keys)[:240_000]
    fresh = rng.permutation(fresh)
    fval = fresh ^ np.uint64(0x5A5A)
    batches, kinds = [], []
    for b in range(8):
        w = fresh[b * 30_000:(b + 1) * 30_000]
        batches.append((w, fval[b * 30_000:(b + 1) * 30_000], np.zeros(w.size, np.uint8)))
        kinds.append(("w", b))
        old = rng.choice(keys, 20_000, replace=False)
        soon = fresh[rng.integers(0, (b + 1) * 30_000, 10_000)]
        rk = np.concatenate([old, soon])
        batches.append((rk, np.zeros(rk.size, np.uint64), np.ones(rk.size, np.uint8)))
        kinds.append(("r", old.size))
    srv = E.Server(t, arena_bytes=64 << 20, max_batches=64)
    try:
        outs = serve_all(srv, batches)
    finally:
        srv.stop()
    fmap = dict(zip(fresh.tolist(), fval.tolist()))
    vmap = dict(zip(keys.tolist(), vals.tolist()))
    for (kind, x), (rk, _, _), (ov, os_) in zip(kinds, batches, outs):
        if kind == "w":
            assert (os_ == E.ST_ABSENT).all()
            continue
        n_old = x
        assert (os_[:n_old] == E.ST_FOUND).all()
        assert all(int(v) == vmap[int(k)] for k, v in zip(rk[:n_old], ov[:n_old]))
        st = os_[n_old:]
        assert set(np.unique(st).tolist()) <= {E.ST_ABSENT, E.ST_FOUND}
        for k, v, s in zip(rk[n_old:], ov[n_old:], st):
            if s == E.ST_FOUND:
                assert int(v) == fmap[int(k)]
    gk, gv = dump(t)
    assert gk.size == keys.size + fresh.size
    assert (gk == np.union1d(keys, fresh)).all()
