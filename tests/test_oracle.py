"""CPU tests of the oracle itself: structure invariants, reference rules,
batch semantics, generators.  The oracle is pinned against the reference
binary separately (tests/golden)."""
import numpy as np
import pytest

from oracle import oracle as O


def test_bulk_build_shape_and_lookup():
    keys = O.gen_keys("uniform", 1, 50000)
    t = O.OracleTree(24, 24)
    t.bulk_build(keys, O.value_of(keys))
    assert t.check() == 0
    sizes = t.leaf_sizes()
    n = np.unique(keys).size
    nl = -(-n // 24)
    assert sizes.size == nl and sizes.sum() == n and sizes.max() - sizes.min() <= 1
    st, v = t.get(int(keys[123]))
    assert st == O.FOUND and v == int(O.value_of(keys[123:124])[0])
    assert t.get(int(keys.max()) + 1)[0] == O.ABSENT


def test_bulk_build_last_value_wins_and_reserved_key():
    t = O.OracleTree()
    t.bulk_build(np.array([5, 3, 5], np.uint64), np.array([1, 2, 9], np.uint64))
    k, v = t.dump()
    assert k.tolist() == [3, 5] and v.tolist() == [2, 9]
    with pytest.raises(ValueError):
        t.bulk_build(np.array([2**64 - 1], np.uint64), np.array([0], np.uint64))


def test_reference_split_rules_sequential_keys():
    # ascending inserts into an empty tree: each leaf split is 16|16 and the
    # early inner split keeps 15|15 (src/gpu-stm-tree-v39/bpt-gpustm-kernel-tree.cuh:150-467)
    t = O.OracleTree()
    for i in range(32):
        assert t.insert(i, i * 10)[0] == O.ABSENT
    assert t.leaf_sizes().tolist() == [16, 16]
    s = t.stats()
    assert s["leaf_splits"] == 1 and s["new_roots"] == 1 and s["height"] == 2
    for i in range(32, 5000):
        t.insert(i, i)
    assert t.check() == 0
    # update returns the previous value
    st, old = t.insert(7, 1)
    assert st == O.FOUND and old == 70


def test_random_inserts_match_dict():
    rng = np.random.default_rng(3)
    t = O.OracleTree()
    d = {}
    for k in rng.integers(0, 2**20, 20000, dtype=np.uint64).tolist():
        st, old = t.insert(k, k + 1)
        assert (st == O.FOUND) == (k in d)
        d[k] = k + 1
    assert t.check() == 0
    k, v = t.dump()
    assert k.tolist() == sorted(d) and v.tolist() == [d[x] for x in sorted(d)]


def test_merged_equals_serial_without_duplicates():
    tk = O.gen_keys("uniform", 3, 20000)
    a, b = O.OracleTree(), O.OracleTree()
    a.bulk_build(tk, O.value_of(tk))
    b.bulk_build(tk, O.value_of(tk))
    rk, rv, ro = O.gen_requests("uniform", 4, tk, 20000, 50)
    v1, s1 = a.execute_serial(rk, rv, ro)
    v2, s2 = b.execute_merged(rk, rv, ro, O.ENGINE_STM, 3)
    assert (v1 == v2).all() and (s1 == s2).all()
    assert (a.dump()[0] == b.dump()[0]).all()


def test_merged_duplicate_semantics():
    # v38 meaning: per key, requests take effect in input order
    t = O.OracleTree()
    t.bulk_build(np.array([10, 20], np.uint64), np.array([100, 200], np.uint64))
    keys = np.array([10, 10, 10, 30, 30, 20, 10, 2**64 - 1], np.uint64)
    vals = np.array([0, 1, 0, 5, 0, 0, 7, 0], np.uint64)
    ops = np.array([1, 0, 1, 1, 0, 1, 0, 1], np.uint8)
    v, s = t.execute_merged(keys, vals, ops)
    assert s.tolist() == [1, 1, 1, 0, 0, 1, 1, 2]
    assert v.tolist() == [100, 100, 1, 0, 0, 200, 1, 0]
    k, vv = t.dump()
    assert k.tolist() == [10, 20, 30] and vv.tolist() == [7, 200, 0]


def test_merge_engine_contents_and_shape():
    tk = O.gen_keys("uniform", 7, 30000)
    a, b = O.OracleTree(), O.OracleTree()
    a.bulk_build(tk, O.value_of(tk))
    b.bulk_build(tk, O.value_of(tk))
    rk, rv, ro = O.gen_requests("uniform", 8, tk, 40000, 0)  # all inserts
    v1, s1 = a.execute_merged(rk, rv, ro, O.ENGINE_STM)
    v2, s2 = b.execute_merged(rk, rv, ro, O.ENGINE_MERGE)
    assert (v1 == v2).all() and (s1 == s2).all()
    assert b.check() == 0
    assert (a.dump()[0] == b.dump()[0]).all() and (a.dump()[1] == b.dump()[1]).all()
    # every merged leaf holds between ceil-split sizes and 31 keys
    assert b.leaf_sizes().max() <= 31


def test_generators_deterministic_and_ranges():
    for dist in ["uniform", "zipf", "normal", "gamma"]:
        a = O.gen_keys(dist, 11, 1000)
        b = O.gen_keys(dist, 11, 1000)
        assert (a == b).all()
        assert (a < np.uint64(2**64 - 1)).all()
    u = O.gen_keys("uniform", 1, 10000)
    assert (u < np.uint64(2**63)).all()
    rk, rv, ro = O.gen_requests("zipf", 2, O.gen_keys("zipf", 2, 1000), 20000, 95)
    assert abs((ro == 1).mean() - 0.95) < 0.01
    # zipf requests are duplicate heavy
    assert np.unique(rk).size < 0.7 * rk.size


def test_sort_pairs_stable():
    keys = np.array([5, 1, 5, 0, 1, 5], np.uint64)
    k, i = O.sort_pairs(keys)
    assert k.tolist() == [0, 1, 1, 5, 5, 5] and i.tolist() == [3, 1, 4, 0, 2, 5]


def test_mlp_gradient_finite_difference():
    rng = np.random.default_rng(0)
    p = rng.normal(0, 0.5, 97).astype(np.float32)
    x = rng.random(64).astype(np.float32)
    y = rng.random(64).astype(np.float32)
    loss, g = O.mlp_grad(p, x, y)
    eps = 1e-3
    for j in [0, 5, 40, 70, 96]:
        pp = p.astype(np.float64).copy()
        pp[j] += eps
        lp = np.mean([(O.mlp_forward(pp.astype(np.float32), xi) - yi) ** 2 for xi, yi in zip(x, y)])
        pm = p.astype(np.float64).copy()
        pm[j] -= eps
        lm = np.mean([(O.mlp_forward(pm.astype(np.float32), xi) - yi) ** 2 for xi, yi in zip(x, y)])
        assert abs((lp - lm) / (2 * eps) - g[j]) < 2e-3 * max(1.0, abs(g[j]))


def _with_deletes(keys, vals, ops, seed, frac=0.15):
    """Turn a share of the requests into DELETEs (op code 2)."""
    rng = np.random.default_rng(seed)
    ops = ops.copy()
    ops[rng.random(ops.size) < frac] = 2
    return keys, vals, ops


@pytest.mark.parametrize("engine", [O.ENGINE_STM, O.ENGINE_MERGE])
def test_merged_equals_serial_with_deletes(engine):
    # per key, the merged meaning is the serial meaning; keys are independent
    keys = O.gen_keys("zipf", 71, 20_000)
    vals = O.value_of(keys)
    a, b = O.OracleTree(), O.OracleTree()
    a.bulk_build(keys, vals)
    b.bulk_build(keys, vals)
    for i in range(4):
        rk, rv, ro = _with_deletes(*O.gen_requests("zipf", 72 + i, keys, 30_000, 60), seed=i)
        sv, ss = a.execute_serial(rk, rv, ro)
        mv, ms = b.execute_merged(rk, rv, ro, engine=engine)
        assert (ss == ms).all() and (sv == mv).all()
    ak, av = a.dump()
    bk, bv = b.dump()
    assert (ak == bk).all() and (av == bv).all()
    assert a.check() == 0 and b.check() == 0


def test_delete_basics():
    t = O.OracleTree()
    k = np.arange(1, 200, dtype=np.uint64) * np.uint64(10)
    t.bulk_build(k, k + np.uint64(1))
    rk = np.array([10, 10, 10, 15, 2**64 - 1, 20], np.uint64)
    ro = np.array([2, 1, 2, 2, 2, 3], np.uint8)
    v, s = t.execute_serial(rk, np.zeros_like(rk), ro)
    assert s.tolist() == [1, 0, 0, 0, 2, 2] and v.tolist() == [11, 0, 0, 0, 0, 0]
    assert t.size() == 198
    # empty leaves stay and keep routing: delete everything, then insert again
    v, s = t.execute_serial(k, np.zeros_like(k), np.full(k.size, 2, np.uint8))
    assert t.size() == 0 and t.check() == 0
    v, s = t.execute_serial(k, k, np.zeros(k.size, np.uint8))
    assert (s == 0).all() and t.size() == k.size and t.check() == 0
