"""INSERT combining in BT_MODE_STM batches (BT_OPT_STM_COMBINE, on by default).

The requests of an STM batch are concurrent transactions (the reference's v39
meaning), so the outcome must be that of some serial order of them.  With
combining, the INSERTs of one key run as one transaction that applies them
back to back: one of them sees the pre-batch state, every other one sees the
value of another INSERT of the key (each exactly once, one chain through all
of them), and the tree ends with the chain's last value.  GETs of the key see
the pre-batch value or the final one.  Keys the batch also DELETEs run
uncombined.  Every request carries its own value so the chain can be traced.
"""
import numpy as np
import pytest

import eirene_b200 as E
from oracle import oracle as O
from tests.helpers import dev, dump, run_batch

pytestmark = pytest.mark.gpu


def make_tree(n_tree, seed, **kw):
    keys = O.gen_keys("uniform", seed, n_tree)
    vals = O.value_of(keys)
    t = E.BTree(max_keys=1 << 20, max_batch=1 << 17, **kw)
    t.bulk_build(dev(keys), dev(vals))
    return t, dict(zip(keys.tolist(), vals.tolist())), keys


def hot_batch(keys, seed, n, n_hot, ins_frac, del_keys=0):
    """n requests on n_hot hot keys (half present in the tree, half fresh),
    Zipf-like popularity, ins_frac INSERTs, the rest GETs; the first del_keys
    hot keys also get a DELETE.  Values are distinct per request."""
    rng = np.random.default_rng(seed)
    fresh = (rng.choice(2**40, n_hot // 2, replace=False).astype(np.uint64) << np.uint64(1)) | np.uint64(1)
    hot = np.concatenate([rng.choice(keys, n_hot - n_hot // 2, replace=False), fresh])
    rng.shuffle(hot)
    w = 1.0 / np.arange(1, n_hot + 1)
    rk = hot[rng.choice(n_hot, n, p=w / w.sum())]
    ro = np.where(rng.random(n) < ins_frac, E.OP_INSERT, E.OP_GET).astype(np.uint8)
    for j in range(del_keys):
        at = np.flatnonzero(rk == hot[j])
        if at.size:
            ro[at[rng.integers(at.size)]] = E.OP_DELETE
    rv = (np.arange(n, dtype=np.uint64) + np.uint64(1 << 50)) * np.uint64(3)
    return rk, rv, ro, hot[:del_keys]


def check_chains(rk, rv, ro, gv, gs, pre, final, skip_keys=()):
    """Every INSERT key's answers form one chain; returns the number of keys
    with more than one INSERT."""
    skip = set(int(k) for k in skip_keys)
    multi = 0
    ins = np.flatnonzero(ro == E.OP_INSERT)
    uk, inv = np.unique(rk[ins], return_inverse=True)
    for j in range(uk.size):
        grp = ins[inv == j]
        k = int(rk[grp[0]])
        if k in skip:
            continue
        multi += grp.size > 1
        vals = {int(rv[i]): int(i) for i in grp}
        heads, preds = [], {}
        for i in grp:
            if gs[i] == E.ST_ABSENT or (gs[i] == E.ST_FOUND and int(gv[i]) == pre.get(k, -1) and k in pre):
                heads.append(int(i))
            else:
                assert gs[i] == E.ST_FOUND, (k, gs[i])
                p = vals.get(int(gv[i]))
                assert p is not None and p != int(i), (k, int(gv[i]))
                assert p not in preds.values(), k  # each INSERT is seen by at most one other
                preds[int(i)] = p
        assert len(heads) == 1, (k, heads)
        if k not in pre:
            assert gs[heads[0]] == E.ST_ABSENT
        # the tail is the INSERT no other one saw; walk back to the head
        seen = set(preds.values())
        tails = [int(i) for i in grp if int(i) not in seen]
        assert len(tails) == 1, k
        cur, steps = tails[0], 1
        while cur in preds:
            cur = preds[cur]
            steps += 1
        assert cur == heads[0] and steps == grp.size, k
        assert final[k] == int(rv[tails[0]]), k
    return multi


def split_commits(s0, s1):
    # a transaction that commits a split and goes on counts one commit more
    return sum(s1[f] - s0[f] for f in ("leaf_splits", "inner_splits", "new_roots"))


@pytest.mark.parametrize("learned", [False, True])
def test_combined_inserts_form_one_chain_per_key(gpu, learned):
    t, pre, keys = make_tree(60_000, 501)
    if learned:
        t.retrain()
        t.set_descent(True)
    rk, rv, ro, _ = hot_batch(keys, 502, 50_000, 600, 0.4)
    s0 = t.stats()
    gv, gs = run_batch(t, rk, rv, ro, E.MODE_STM)
    s1 = t.stats()
    gk, gval = dump(t)
    final = dict(zip(gk.tolist(), gval.tolist()))
    multi = check_chains(rk, rv, ro, gv, gs, pre, final)
    assert multi > 100
    # one transaction per INSERT key
    n_ins_keys = np.unique(rk[ro == E.OP_INSERT]).size
    assert n_ins_keys <= s1["commits"] - s0["commits"] <= n_ins_keys + split_commits(s0, s1)
    # GETs: the pre-batch state or the final one
    for i in np.flatnonzero(ro == E.OP_GET):
        k = int(rk[i])
        ok = [(E.ST_FOUND, pre[k])] if k in pre else [(E.ST_ABSENT, 0)]
        if k in final:
            ok.append((E.ST_FOUND, final[k]))
        assert (int(gs[i]), int(gv[i])) in ok, k
    # every other key is as it was
    ins_keys = set(rk[ro == E.OP_INSERT].tolist())
    assert set(final) == set(pre) | ins_keys
    assert all(final[k] == v for k, v in pre.items() if k not in ins_keys)


def test_keys_with_a_delete_are_not_combined(gpu):
    t, pre, keys = make_tree(60_000, 511)
    rk, rv, ro, dk = hot_batch(keys, 512, 30_000, 300, 0.4, del_keys=40)
    gv, gs = run_batch(t, rk, rv, ro, E.MODE_STM)
    gk, gval = dump(t)
    final = dict(zip(gk.tolist(), gval.tolist()))
    check_chains(rk, rv, ro, gv, gs, pre, final, skip_keys=dk)
    for k in dk.tolist():
        sel = rk == np.uint64(k)
        # run uncombined: a serial order of INSERTs and a DELETE; the key ends
        # absent or with one of the batch's values for it
        if k in final:
            assert final[k] in set(rv[sel & (ro == E.OP_INSERT)].tolist())
        ins_st = gs[sel & (ro == E.OP_INSERT)]
        assert set(np.unique(ins_st).tolist()) <= {E.ST_ABSENT, E.ST_FOUND}


def test_combining_off_runs_every_insert(gpu):
    t, pre, keys = make_tree(60_000, 521)
    t.set_option(E.OPT_STM_COMBINE, 0)
    rk, rv, ro, _ = hot_batch(keys, 522, 20_000, 200, 0.4)
    s0 = t.stats()
    gv, gs = run_batch(t, rk, rv, ro, E.MODE_STM)
    s1 = t.stats()
    n_ins = int((ro == E.OP_INSERT).sum())
    assert n_ins <= s1["commits"] - s0["commits"] <= n_ins + split_commits(s0, s1)
    gk, gval = dump(t)
    final = dict(zip(gk.tolist(), gval.tolist()))
    for k in np.unique(rk[ro == E.OP_INSERT]).tolist():
        assert final[k] in set(rv[(rk == np.uint64(k)) & (ro == E.OP_INSERT)].tolist())


def test_failed_representative_fails_its_chain(gpu):
    # full leaves and one attempt per transaction: an INSERT of a fresh key
    # needs a split, takes the validated path and runs out of attempts; the
    # INSERTs combined with it report the same status and nothing changes
    t, pre, keys = make_tree(20_000, 531, leaf_fill=31, inner_fill=31, retry_limit=1)
    rk, rv, ro, _ = hot_batch(keys, 532, 10_000, 100, 0.6)
    gv, gs = run_batch(t, rk, rv, ro, E.MODE_STM)
    fresh = np.array([int(k) not in pre for k in rk.tolist()])
    ins = ro == E.OP_INSERT
    assert (gs[ins & fresh] == E.ST_RETRY_EXHAUSTED).all()
    assert (gv[ins & fresh] == 0).all()
    gk, gval = dump(t)
    final = dict(zip(gk.tolist(), gval.tolist()))
    assert set(final) == set(pre)  # no fresh key got in
    assert t.stats()["error"] & 2
