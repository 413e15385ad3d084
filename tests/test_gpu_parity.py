"""GPU parity: the CUDA path (through the C ABI) against the CPU oracle on the
same seeded inputs.  Everything here is integer work, so the bar is bit-exact:
answers (value + status byte) per request, final sorted contents, and for the
deterministic engines the leaf layout."""
import numpy as np
import pytest

import eirene_b200 as E
from oracle import oracle as O
from tests.helpers import dev, dump, empty_u64, empty_u8, host_u64, host_u8, run_batch

pytestmark = pytest.mark.gpu


def make_pair(n_keys, dist="uniform", seed=1, leaf_fill=24, inner_fill=24, max_batch=1 << 18, max_keys=None):
    keys = O.gen_keys(dist, seed, n_keys)
    vals = O.value_of(keys)
    t = E.BTree(max_keys=max_keys or max(4 * n_keys, 1 << 16), max_batch=max_batch, leaf_fill=leaf_fill,
                inner_fill=inner_fill)
    t.bulk_build(dev(keys), dev(vals))
    o = O.OracleTree(leaf_fill, inner_fill)
    o.bulk_build(keys, vals)
    return t, o, keys


def assert_same_contents(t, o):
    gk, gv = dump(t)
    ok, ov = o.dump()
    assert gk.size == ok.size
    assert (gk == ok).all() and (gv == ov).all()
    assert t.size() == o.size()


def test_bulk_build_layout_matches_oracle(gpu):
    for n in [1, 2, 23, 24, 25, 1000, 100_000]:
        t, o, _ = make_pair(n, seed=n)
        assert_same_contents(t, o)
        assert (t.leaf_sizes() == o.leaf_sizes()).all()
        assert (t.level_counts() == o.level_counts()).all()
        t.close()


def test_bulk_build_duplicates_last_wins(gpu):
    keys = np.array([9, 4, 9, 4, 1], np.uint64)
    vals = np.array([1, 2, 3, 4, 5], np.uint64)
    t = E.BTree(max_keys=1 << 12, max_batch=1 << 12)
    t.bulk_build(dev(keys), dev(vals))
    k, v = dump(t)
    assert k.tolist() == [1, 4, 9] and v.tolist() == [5, 4, 3]
    with pytest.raises(E.BTError) as ei:
        t.bulk_build(dev(np.array([3, 2**64 - 1], np.uint64)), dev(np.array([0, 0], np.uint64)))
    assert ei.value.code == -5


def test_search_matches_oracle(gpu):
    t, o, keys = make_pair(200_000, seed=5)
    rk, rv, ro = O.gen_requests("uniform", 6, keys, 100_000, 100)
    rk[7] = np.uint64(2**64 - 1)  # reserved key: rejected
    ov, os_ = o.execute_merged(rk, rv, ro)
    for lanes in [4, 8, 16, 32]:
        t.set_search_group(lanes)
        gv, gs = empty_u64(rk.size), empty_u8(rk.size)
        t.search(dev(rk), gv, gs)
        assert (host_u8(gs) == os_).all(), lanes
        assert (host_u64(gv) == ov).all(), lanes


@pytest.mark.parametrize("front", [1, 0])
@pytest.mark.parametrize("mix", [95, 50, 0])
def test_sorted_batch_uniform(gpu, mix, front):
    t, o, keys = make_pair(100_000, seed=11)
    t.set_option(E.OPT_FRONT_END, front)
    for b in range(3):
        rk, rv, ro = O.gen_requests("uniform", 100 + b, keys, 60_000, mix)
        ov, os_ = o.execute_merged(rk, rv, ro)
        gv, gs = run_batch(t, rk, rv, ro, E.MODE_SORTED)
        assert (gs == os_).all()
        assert (gv == ov).all()
    assert_same_contents(t, o)
    st = t.stats()
    assert st["error"] == 0 and st["retry_exhausted"] == 0


@pytest.mark.parametrize("front", [1, 0])
@pytest.mark.parametrize("dist", ["zipf", "normal", "gamma"])
def test_sorted_batch_skewed_duplicates(gpu, dist, front):
    t, o, keys = make_pair(50_000, dist=dist, seed=21)
    t.set_option(E.OPT_FRONT_END, front)
    for b in range(2):
        rk, rv, ro = O.gen_requests(dist, 200 + b, keys, 80_000, 95 if b == 0 else 50)
        ov, os_ = o.execute_merged(rk, rv, ro)
        gv, gs = run_batch(t, rk, rv, ro, E.MODE_SORTED)
        assert (gs == os_).all()
        assert (gv == ov).all()
    assert_same_contents(t, o)


@pytest.mark.parametrize("front", [1, 0])
def test_sorted_batch_edge_cases(gpu, front):
    t = E.BTree(max_keys=1 << 16, max_batch=1 << 15)
    t.set_option(E.OPT_FRONT_END, front)
    o = O.OracleTree()
    # empty tree: gets are absent, inserts build the tree through STM
    cases = [
        (np.array([5], np.uint64), np.array([50], np.uint64), np.array([1], np.uint8)),
        (np.array([5, 5, 5], np.uint64), np.array([50, 51, 0], np.uint64), np.array([0, 0, 1], np.uint8)),
        (np.array([2**64 - 1, 3, 3], np.uint64), np.array([1, 30, 0], np.uint64), np.array([0, 0, 7], np.uint8)),
        (np.arange(4000, dtype=np.uint64)[::-1].copy(), np.arange(4000, dtype=np.uint64),
         np.zeros(4000, np.uint8)),
    ]
    for rk, rv, ro in cases:
        ov, os_ = o.execute_merged(rk, rv, ro)
        gv, gs = run_batch(t, rk, rv, ro, E.MODE_SORTED)
        assert (gs == os_).all() and (gv == ov).all()
    assert_same_contents(t, o)
    # batch across tile boundaries with one long run of a single key
    n = 20_000
    rk = np.full(n, 77, np.uint64)
    rk[::3] = np.arange(0, n, 3, dtype=np.uint64) + 100_000
    ro = (np.arange(n) % 5 == 0).astype(np.uint8) ^ 1
    rv = np.arange(n, dtype=np.uint64) + 1
    ov, os_ = o.execute_merged(rk, rv, ro)
    gv, gs = run_batch(t, rk, rv, ro, E.MODE_SORTED)
    assert (gs == os_).all() and (gv == ov).all()
    assert_same_contents(t, o)


def test_stm_mode_matches_serial_without_duplicates(gpu):
    t, o, keys = make_pair(100_000, seed=31)
    rk, rv, ro = O.gen_requests("uniform", 32, keys, 50_000, 50)
    _, first = np.unique(rk, return_index=True)
    sel = np.sort(first)
    rk, rv, ro = rk[sel], rv[sel], ro[sel]
    ov, os_ = o.execute_serial(rk, rv, ro)
    gv, gs = run_batch(t, rk, rv, ro, E.MODE_STM)
    assert (gs == os_).all() and (gv == ov).all()
    assert_same_contents(t, o)


def test_stm_inserts_from_empty_tree_split_rules(gpu):
    # ascending single-warp-at-a-time inserts reproduce the reference split rules
    t = E.BTree(max_keys=1 << 14, max_batch=1 << 14)
    o = O.OracleTree()
    for i in range(0, 2000):
        k = np.array([i * 3], np.uint64)
        v = np.array([i], np.uint64)
        op = np.array([0], np.uint8)
        gv, gs = run_batch(t, k, v, op, E.MODE_STM)
        ov, os_ = o.execute_serial(k, v, op)
        assert gs[0] == os_[0]
    assert_same_contents(t, o)
    # one request at a time is a serial order: the shape matches the oracle exactly
    assert (t.leaf_sizes() == o.leaf_sizes()).all()
    assert (t.level_counts() == o.level_counts()).all()
    s = t.stats()
    os_ = o.stats()
    assert s["leaf_splits"] == os_["leaf_splits"] and s["new_roots"] == os_["new_roots"]


def test_stm_concurrent_random_inserts(gpu):
    # many warps inserting disjoint keys concurrently into a small tree (heavy splitting)
    t = E.BTree(max_keys=1 << 18, max_batch=1 << 17)
    o = O.OracleTree()
    rng = np.random.default_rng(5)
    rk = rng.choice(2**40, 100_000, replace=False).astype(np.uint64)
    rv = rk * np.uint64(3)
    ro = np.zeros(rk.size, np.uint8)
    ov, os_ = o.execute_serial(rk, rv, ro)
    gv, gs = run_batch(t, rk, rv, ro, E.MODE_STM)
    assert (gs == os_).all()
    assert_same_contents(t, o)
    st = t.stats()
    assert st["error"] == 0 and st["leaf_splits"] > 1000


def test_host_entry_point_matches_device(gpu):
    t, o, keys = make_pair(50_000, seed=41)
    rk, rv, ro = O.gen_requests("uniform", 42, keys, 30_000, 95)
    ov, os_ = o.execute_merged(rk, rv, ro)
    hv, hs = t.execute_host(rk, rv, ro, mode=E.MODE_SORTED)
    assert (hs == os_).all() and (hv == ov).all()
    assert_same_contents(t, o)


def test_batch_too_large_rejected(gpu):
    t = E.BTree(max_keys=1 << 12, max_batch=1024)
    rk = np.arange(2048, dtype=np.uint64)
    with pytest.raises(E.BTError) as ei:
        run_batch(t, rk, rk, np.ones(2048, np.uint8), E.MODE_SORTED)
    assert ei.value.code == -6


def test_pool_exhaustion_reports_status(gpu):
    # a pool too small for the inserts: requests report NO_CAPACITY, nothing corrupts
    t = E.BTree(max_keys=0, max_batch=1 << 16)  # pool = 4096 nodes, at most 4096 * 31 keys
    rk = np.arange(1, 4 * 65536 + 1, dtype=np.uint64) * np.uint64(7)
    st_all = []
    for c in range(0, rk.size, 16384):
        k = rk[c:c + 16384]
        gv, gs = run_batch(t, k, k, np.zeros(k.size, np.uint8), E.MODE_STM)
        st_all.append(gs)
    st_all = np.concatenate(st_all)
    assert set(np.unique(st_all).tolist()) <= {E.ST_ABSENT, E.ST_NO_CAPACITY}
    s = t.stats()
    assert s["error"] & 1
    # whatever was inserted is intact and searchable
    k, v = dump(t)
    assert (np.diff(k.astype(np.float64)) > 0).all()
    ins = rk[st_all == E.ST_ABSENT]
    assert np.isin(k, ins).all() and k.size == ins.size


@pytest.mark.parametrize("tile", [256, 512, 1024])
@pytest.mark.parametrize("front", [1, 0])
def test_sort_tiles_exact(gpu, tile, front):
    # every radix sort tile (threads x 8 keys) gives the oracle's answers,
    # through both front ends; batches large and skewed enough to span many
    # tiles and repeat keys
    t, o, keys = make_pair(150_000, dist="zipf", seed=41)
    t.set_option(E.OPT_FRONT_END, front)
    t.set_option(E.OPT_SORT_TILE, tile)
    for b in range(2):
        rk, rv, ro = O.gen_requests("zipf", 420 + b, keys, 90_000, [50, 80][b])
        ov, os_ = o.execute_merged(rk, rv, ro)
        gv, gs = run_batch(t, rk, rv, ro, E.MODE_SORTED)
        assert (gs == os_).all() and (gv == ov).all(), (tile, front, b)
    assert_same_contents(t, o)


def test_autotune_fill_then_exact(gpu):
    keys = O.gen_keys("uniform", 51, 200_000)
    vals = O.value_of(keys)
    t = E.BTree(max_keys=1 << 21, max_batch=1 << 18)
    rep = t.autotune_fill(dev(keys[:100_000]))
    f = rep["leaf_fill"]
    assert f in (16, 20, 24, 28) and rep["inner_fill"] == f
    assert all(v > 0 for v in rep["batch_ms"].values())
    # later builds and splits use the chosen fill: the layout equals the oracle's at that fill
    t.bulk_build(dev(keys), dev(vals))
    o = O.OracleTree(f, f)
    o.bulk_build(keys, vals)
    assert (t.leaf_sizes() == o.leaf_sizes()).all()
    rk, rv, ro = O.gen_requests("uniform", 52, keys, 60_000, 50)
    ov, os_ = o.execute_merged(rk, rv, ro, engine=O.ENGINE_MERGE)
    gv, gs = run_batch(t, rk, rv, ro, E.MODE_SORTED | E.MODE_MERGE_ENGINE)
    assert (gs == os_).all() and (gv == ov).all()
    assert (t.leaf_sizes() == o.leaf_sizes()).all()
