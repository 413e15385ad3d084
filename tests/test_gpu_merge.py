"""Segmented leaf merge (BT_MODE_SORTED | BT_MODE_MERGE_ENGINE) against the
oracle's merge engine: answers, contents, and the exact tree shape (leaf
sizes in key order, nodes per level, split counts)."""
import numpy as np
import pytest

import eirene_b200 as E
from oracle import oracle as O
from tests.helpers import dev, dump, run_batch

pytestmark = pytest.mark.gpu
MERGE = E.MODE_SORTED | E.MODE_MERGE_ENGINE


def pair(keys, leaf_fill=24, inner_fill=24, max_batch=1 << 18):
    vals = O.value_of(keys)
    t = E.BTree(max_keys=max(8 * keys.size, 1 << 18), max_batch=max_batch, leaf_fill=leaf_fill,
                inner_fill=inner_fill)
    o = O.OracleTree(leaf_fill, inner_fill)
    if keys.size:
        t.bulk_build(dev(keys), dev(vals))
        o.bulk_build(keys, vals)
    return t, o


def check_same(t, o, splits=True):
    gk, gv = dump(t)
    ok, ov = o.dump()
    assert gk.size == ok.size and (gk == ok).all() and (gv == ov).all()
    assert (t.leaf_sizes() == o.leaf_sizes()).all()
    assert (t.level_counts() == o.level_counts()).all()
    if splits:
        gs, os_ = t.stats(), o.stats()
        for f in ("leaf_splits", "inner_splits", "new_roots"):
            assert gs[f] == os_[f], (f, gs[f], os_[f])


def run_both(t, o, rk, rv, ro):
    ov, os_ = o.execute_merged(rk, rv, ro, O.ENGINE_MERGE)
    gv, gs = run_batch(t, rk, rv, ro, MERGE)
    assert (gs == os_).all() and (gv == ov).all()


@pytest.mark.parametrize("mix", [95, 50, 0])
def test_merge_engine_matches_oracle_shape(gpu, mix):
    keys = O.gen_keys("uniform", 61, 120_000)
    t, o = pair(keys)
    for b in range(4):
        rk, rv, ro = O.gen_requests("uniform", 600 + b, keys, 100_000, mix)
        run_both(t, o, rk, rv, ro)
    check_same(t, o)
    if mix == 0:
        assert t.stats()["leaf_splits"] > 1000


def test_merge_engine_small_tree_many_inserts(gpu):
    # a 100-key tree takes 150k inserts in one batch: thousands of leaf splits,
    # inner splits and root rebuilds
    keys = O.gen_keys("uniform", 62, 100)
    t, o = pair(keys, max_batch=1 << 18)
    rk = O.gen_keys("uniform", 63, 150_000)
    run_both(t, o, rk, O.value_of(rk), np.zeros(rk.size, np.uint8))
    check_same(t, o)
    assert t.stats()["new_roots"] >= 1


@pytest.mark.parametrize("n", [1, 24, 25, 31, 32, 1000, 70_000])
def test_merge_engine_from_empty_tree(gpu, n):
    t, o = pair(np.zeros(0, np.uint64))
    rk = O.gen_keys("uniform", 64 + n, n)
    run_both(t, o, rk, O.value_of(rk), np.zeros(n, np.uint8))
    check_same(t, o)


@pytest.mark.parametrize("fills", [(24, 24), (16, 31), (31, 16), (16, 16)])
def test_merge_engine_fill_settings(gpu, fills):
    keys = O.gen_keys("uniform", 65, 20_000)
    t, o = pair(keys, *fills)
    for b in range(3):
        rk, rv, ro = O.gen_requests("uniform", 700 + b, keys, 30_000, 30)
        run_both(t, o, rk, rv, ro)
    check_same(t, o)


def test_merge_engine_zipf_duplicates_and_mixed_engines(gpu):
    keys = O.gen_keys("zipf", 66, 50_000)
    t, o = pair(keys)
    for b in range(4):
        rk, rv, ro = O.gen_requests("zipf", 800 + b, keys, 80_000, 50)
        if b % 2 == 0:
            run_both(t, o, rk, rv, ro)
        else:  # the STM engine in between: same answers and contents (shape may differ)
            ov, os_ = o.execute_merged(rk, rv, ro, O.ENGINE_STM)
            gv, gs = run_batch(t, rk, rv, ro, E.MODE_SORTED)
            assert (gs == os_).all() and (gv == ov).all()
    gk, gv = dump(t)
    ok, ov = o.dump()
    assert (gk == ok).all() and (gv == ov).all()


def test_merge_engine_learned_lookups_after_merge(gpu):
    keys = O.gen_keys("uniform", 67, 200_000)
    t, o = pair(keys)
    t.retrain()
    t.set_descent(True)
    for b in range(3):
        rk, rv, ro = O.gen_requests("uniform", 900 + b, keys, 120_000, 20)
        run_both(t, o, rk, rv, ro)
    check_same(t, o)
