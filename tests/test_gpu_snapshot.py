"""Snapshot save/load (bt_save / bt_load): a tree changed by batches is saved,
loaded into a fresh handle and must hold the same pairs and answer a new
batch exactly like the oracle; damaged files are refused with BT_ERR_IO."""
import os

import numpy as np
import pytest

import eirene_b200 as E
from oracle import oracle as O
from tests.helpers import dev, dump, run_batch

pytestmark = pytest.mark.gpu


def test_save_load_round_trip(gpu, tmp_path):
    keys = O.gen_keys("zipf", 41, 120_000)
    vals = O.value_of(keys)
    t = E.BTree(max_keys=1 << 20, max_batch=1 << 17)
    t.bulk_build(dev(keys), dev(vals))
    o = O.OracleTree()
    o.bulk_build(keys, vals)
    for b in range(3):
        rk, rv, ro = O.gen_requests("zipf", 42 + b, keys, 60_000, 60)
        o.execute_merged(rk, rv, ro)
        run_batch(t, rk, rv, ro, E.MODE_SORTED | E.MODE_MERGE_ENGINE)
    path = str(tmp_path / "tree.snap")
    t.save(path)
    assert os.path.getsize(path) == 32 + 16 * t.size()
    t2 = E.BTree(max_keys=1 << 20, max_batch=1 << 17, leaf_fill=20)
    t2.load(path)
    gk, gv = dump(t2)
    ok, ov = o.dump()
    assert (gk == ok).all() and (gv == ov).all()
    rk, rv, ro = O.gen_requests("zipf", 50, ok, 50_000, 70)
    ov2, os2 = o.execute_merged(rk, rv, ro)
    gv2, gs2 = run_batch(t2, rk, rv, ro, E.MODE_SORTED)
    assert (gs2 == os2).all() and (gv2 == ov2).all()


def test_empty_tree_and_damaged_files(gpu, tmp_path):
    t = E.BTree(max_keys=1 << 16, max_batch=1 << 12)
    p = str(tmp_path / "empty.snap")
    t.save(p)
    t.load(p)
    assert t.size() == 0
    keys = O.gen_keys("uniform", 3, 1000)
    t.bulk_build(dev(keys), dev(O.value_of(keys)))
    good = str(tmp_path / "good.snap")
    t.save(good)
    raw = bytearray(open(good, "rb").read())
    cases = {"truncated": raw[:-8], "flipped": raw[:40] + bytes([raw[40] ^ 1]) + raw[41:], "magic": b"X" + raw[1:]}
    for name, data in cases.items():
        bad = str(tmp_path / f"{name}.snap")
        open(bad, "wb").write(bytes(data))
        with pytest.raises(E.BTError) as ei:
            t.load(bad)
        assert ei.value.code == -11, name
    with pytest.raises(E.BTError) as ei:
        t.load(str(tmp_path / "missing.snap"))
    assert ei.value.code == -11
    # a failed load leaves the tree as it was
    assert t.size() == 1000


def test_pool_image_keeps_layout_and_continues(gpu, tmp_path):
    # the image holds the pool itself: the loaded tree has the saved leaf
    # layout, and the next merge-engine batch runs identically on both
    keys = O.gen_keys("gamma", 61, 100_000)
    vals = O.value_of(keys)
    t = E.BTree(max_keys=1 << 20, max_batch=1 << 17)
    t.bulk_build(dev(keys), dev(vals))
    o = O.OracleTree()
    o.bulk_build(keys, vals)
    for b in range(3):
        rk, rv, ro = O.gen_requests("gamma", 62 + b, keys, 60_000, 50)
        o.execute_merged(rk, rv, ro, engine=O.ENGINE_MERGE)
        run_batch(t, rk, rv, ro, E.MODE_SORTED | E.MODE_MERGE_ENGINE)
    path = str(tmp_path / "tree.img")
    t.save_image(path)
    n_nodes = t.stats()["n_nodes"]
    assert os.path.getsize(path) == 40 + 104 + 520 * n_nodes  # header, control block, rows and lows
    t2 = E.BTree(max_keys=1 << 20, max_batch=1 << 17)
    t2.load_image(path)
    ak, av = dump(t)
    bk, bv = dump(t2)
    assert (ak == bk).all() and (av == bv).all()
    assert (t.leaf_sizes() == t2.leaf_sizes()).all() and (t.level_counts() == t2.level_counts()).all()
    assert t2.size() == t.size() == o.size()
    rk, rv, ro = O.gen_requests("gamma", 70, keys, 60_000, 50)
    ov, os_ = o.execute_merged(rk, rv, ro, engine=O.ENGINE_MERGE)
    g1 = run_batch(t, rk, rv, ro, E.MODE_SORTED | E.MODE_MERGE_ENGINE)
    g2 = run_batch(t2, rk, rv, ro, E.MODE_SORTED | E.MODE_MERGE_ENGINE)
    assert (g2[1] == os_).all() and (g2[0] == ov).all()
    assert (g1[1] == g2[1]).all() and (g1[0] == g2[0]).all()
    assert (t.leaf_sizes() == t2.leaf_sizes()).all()
    assert (t2.leaf_sizes() == o.leaf_sizes()).all()
    # damaged image, and a pool too small for it
    raw = bytearray(open(path, "rb").read())
    raw[200] ^= 1
    bad = str(tmp_path / "bad.img")
    open(bad, "wb").write(bytes(raw))
    with pytest.raises(E.BTError) as ei:
        E.BTree(max_keys=1 << 20, max_batch=1 << 12).load_image(bad)
    assert ei.value.code == -11
    with pytest.raises(E.BTError) as ei:
        E.BTree(max_keys=0, max_batch=1 << 12).load_image(path)
    assert ei.value.code == -3  # BT_ERR_NO_MEMORY
    # a handle with other fills would split differently afterwards: refused
    with pytest.raises(E.BTError) as ei:
        E.BTree(max_keys=1 << 20, max_batch=1 << 12, leaf_fill=20).load_image(path)
    assert ei.value.code == -1  # BT_ERR_INVALID_ARG


def test_pool_image_starts_with_clean_counters(gpu, tmp_path):
    # counters of the saving handle do not come back with its tree
    keys = O.gen_keys("uniform", 71, 20_000)
    vals = O.value_of(keys)
    t = E.BTree(max_keys=1 << 18, max_batch=1 << 15)
    t.bulk_build(dev(keys), dev(vals))
    rk, rv, ro = O.gen_requests("uniform", 72, keys, 20_000, 0)
    run_batch(t, rk, rv, ro, E.MODE_SORTED | E.MODE_MERGE_ENGINE)
    assert t.stats()["leaf_splits"] > 0
    path = str(tmp_path / "c.img")
    t.save_image(path)
    t2 = E.BTree(max_keys=1 << 18, max_batch=1 << 15)
    t2.bulk_build(dev(keys[:5000]), dev(vals[:5000]))  # rows beyond the image's hold another tree
    t2.load_image(path)
    st = t2.stats()
    assert st["leaf_splits"] == 0 and st["error"] == 0 and st["n_keys"] == t.size()
    ak, av = dump(t)
    bk, bv = dump(t2)
    assert (ak == bk).all() and (av == bv).all()
