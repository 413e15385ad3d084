"""The hash front end of sorted batches (only requests coupled by an INSERT of
their key are sorted; the rest are unsorted lookups of the pre-batch tree)
against the oracle's v38 meaning, on the cases that separate the two
classes: a GET before the first INSERT of its key, GETs and INSERTs after
it, repeated INSERTs, reserved keys and invalid op codes, batches that are
all INSERTs (the largest hash table), all GETs (no table), and the merge and
STM insert engines under both descents."""
import numpy as np
import pytest

import eirene_b200 as E
from oracle import oracle as O
from tests.helpers import dev, dump, run_batch

pytestmark = pytest.mark.gpu


def pair(n, seed, max_batch=1 << 18, dist="uniform"):
    keys = O.gen_keys(dist, seed, n)
    vals = O.value_of(keys)
    t = E.BTree(max_keys=1 << 21, max_batch=max_batch)
    t.bulk_build(dev(keys), dev(vals))
    o = O.OracleTree()
    o.bulk_build(keys, vals)
    return t, o, keys


def check(t, o, rk, rv, ro, mode=E.MODE_SORTED):
    ov, os_ = o.execute_merged(rk, rv, ro)
    gv, gs = run_batch(t, rk, rv, ro, mode)
    bad = np.nonzero((gs != os_) | (gv != ov))[0]
    assert bad.size == 0, (bad[:10], gs[bad[:10]], os_[bad[:10]], gv[bad[:10]], ov[bad[:10]])


def test_order_inside_a_key(gpu):
    t, o, keys = pair(10_000, 1)
    fresh = np.uint64(3)  # not in the tree (gen keys are large)
    old = keys[7]
    rk = np.array([fresh, fresh, fresh, fresh, old, old, old, old, old, keys[8]], np.uint64)
    ro = np.array([1, 0, 1, 0, 1, 1, 0, 1, 0, 1], np.uint8)
    rv = np.arange(rk.size, dtype=np.uint64) + 1000
    check(t, o, rk, rv, ro)
    assert (dump(t)[0] == o.dump()[0]).all()


def test_reserved_keys_and_invalid_ops(gpu):
    t, o, keys = pair(10_000, 2)
    rk = np.array([2**64 - 1, 2**64 - 1, keys[1], keys[1], keys[2], 5, 5], np.uint64)
    ro = np.array([0, 1, 9, 1, 2, 0, 200], np.uint8)
    rv = np.arange(rk.size, dtype=np.uint64)
    check(t, o, rk, rv, ro)


@pytest.mark.parametrize("engine", [E.MODE_MERGE_ENGINE, 0])
@pytest.mark.parametrize("learned", [False, True])
def test_all_inserts_all_gets_and_mixes(gpu, engine, learned):
    t, o, keys = pair(100_000, 3)
    if learned:
        t.retrain()
        t.set_descent(True)
    mode = E.MODE_SORTED | engine
    n = 1 << 18  # = max_batch: the hash table at its largest
    for b, mix in enumerate([0, 100, 95, 50, 5]):
        rk, rv, ro = O.gen_requests("uniform", 40 + b, keys, n, mix)
        check(t, o, rk, rv, ro, mode)
    gk, gv = dump(t)
    ok, ov = o.dump()
    assert (gk == ok).all() and (gv == ov).all()


def test_zipf_hot_keys_both_front_ends_agree(gpu):
    t1, o, keys = pair(50_000, 4, dist="zipf")
    t0, _, _ = pair(50_000, 4, dist="zipf")
    t0.set_option(E.OPT_FRONT_END, 0)
    for b in range(3):
        rk, rv, ro = O.gen_requests("zipf", 60 + b, keys, 100_000, [95, 50, 80][b])
        ov, os_ = o.execute_merged(rk, rv, ro)
        g1 = run_batch(t1, rk, rv, ro, E.MODE_SORTED | E.MODE_MERGE_ENGINE)
        g0 = run_batch(t0, rk, rv, ro, E.MODE_SORTED | E.MODE_MERGE_ENGINE)
        for gv, gs in (g1, g0):
            assert (gs == os_).all() and (gv == ov).all()
    for t in (t1, t0):
        gk, gv = dump(t)
        ok, ov = o.dump()
        assert (gk == ok).all() and (gv == ov).all()


@pytest.mark.parametrize("fills", [(24, 24), (16, 16)])
def test_search_top_cache_matches_global_descent(gpu, fills):
    # a taller tree (fill 16) has more cached levels; inserts between the
    # searches split nodes of the cached levels, and the cache is rebuilt
    keys = O.gen_keys("uniform", 70, 400_000)
    vals = O.value_of(keys)
    t = E.BTree(max_keys=1 << 22, max_batch=1 << 18, leaf_fill=fills[0], inner_fill=fills[1])
    t.bulk_build(dev(keys), dev(vals))
    o = O.OracleTree()
    o.bulk_build(keys, vals)
    for b in range(3):
        qk, _, _ = O.gen_requests("uniform", 80 + b, o.dump()[0], 150_000, 100)
        qk[:3] = [0, 2**64 - 1, 1]
        ov, os_ = o.execute_merged(qk, np.zeros_like(qk), np.ones(qk.size, np.uint8))
        for lanes in (4, 8, 16, 32):
            t.set_search_group(lanes)
            for cache in (1, 0):
                t.set_option(E.OPT_TOP_CACHE, cache)
                gv, gs = run_batch(t, qk, np.zeros_like(qk), np.ones(qk.size, np.uint8), E.MODE_SORTED)
                assert (gs == os_).all() and (gv == ov).all(), (b, lanes, cache)
        t.set_option(E.OPT_TOP_CACHE, 1)
        rk, rv, ro = O.gen_requests("uniform", 90 + b, keys, 200_000, 0)
        check(t, o, rk, rv, ro, E.MODE_SORTED | E.MODE_MERGE_ENGINE)
    assert t.stats()["inner_splits"] > 0


def test_unaligned_op_array_and_subranges(gpu):
    # op codes at an odd byte offset (a slice of a larger array): the front end
    # reads them one byte at a time
    import torch

    t, o, keys = pair(50_000, 5)
    rk, rv, ro = O.gen_requests("uniform", 95, keys, 30_001, 60)
    ov, os_ = o.execute_merged(rk, rv, ro)
    big = torch.from_numpy(np.concatenate([[7], ro]).astype(np.uint8)).cuda()
    gv = torch.zeros(rk.size, dtype=torch.int64, device="cuda")
    gs = torch.zeros(rk.size, dtype=torch.uint8, device="cuda")
    t.execute(dev(rk), dev(rv), big[1:], gv, gs, mode=E.MODE_SORTED)
    torch.cuda.synchronize()
    assert (gs.cpu().numpy() == os_).all() and (gv.cpu().numpy().view(np.uint64) == ov).all()
