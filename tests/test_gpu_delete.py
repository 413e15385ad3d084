"""DELETE (op code 2) on the GPU against the oracle: sorted batches with
repeated keys (every request's answer follows the serial order of its key:
state before the first write, then the latest write's), through both front
ends and both insert engines; STM batches of distinct keys; deleting a whole
tree and refilling it; and the serving loop."""
import numpy as np
import pytest

import eirene_b200 as E
from oracle import oracle as O
from tests.helpers import dev, dump, run_batch

pytestmark = pytest.mark.gpu


def with_deletes(k, v, o, seed, frac):
    rng = np.random.default_rng(seed)
    o = o.copy()
    o[rng.random(o.size) < frac] = 2
    return k, v, o


def pair(dist, seed, n=100_000, fills=(24, 24)):
    keys = O.gen_keys(dist, seed, n)
    vals = O.value_of(keys)
    t = E.BTree(max_keys=1 << 21, max_batch=1 << 18, leaf_fill=fills[0], inner_fill=fills[1])
    t.bulk_build(dev(keys), dev(vals))
    o = O.OracleTree(*fills)
    o.bulk_build(keys, vals)
    return t, o, keys


def same_contents(t, o):
    gk, gv = dump(t)
    ok, ov = o.dump()
    assert gk.size == ok.size and (gk == ok).all() and (gv == ov).all()
    assert t.size() == o.size()


@pytest.mark.parametrize("front", [1, 0])
@pytest.mark.parametrize("engine", [E.MODE_MERGE_ENGINE, 0])
@pytest.mark.parametrize("dist", ["uniform", "zipf"])
def test_sorted_batches_with_deletes(gpu, front, engine, dist):
    t, o, keys = pair(dist, 81)
    t.set_option(E.OPT_FRONT_END, front)
    for b, (mix, frac) in enumerate([(90, 0.05), (50, 0.3), (70, 0.6)]):
        rk, rv, ro = with_deletes(*O.gen_requests(dist, 82 + b, keys, 60_000, mix), seed=b, frac=frac)
        ov, os_ = o.execute_merged(rk, rv, ro, engine=O.ENGINE_MERGE if engine else O.ENGINE_STM)
        gv, gs = run_batch(t, rk, rv, ro, E.MODE_SORTED | engine)
        bad = np.nonzero((gs != os_) | (gv != ov))[0]
        assert bad.size == 0, (b, bad[:5], ro[bad[:5]], gs[bad[:5]], os_[bad[:5]])
        same_contents(t, o)
    if engine:  # the merge engine's shape is deterministic
        assert (t.leaf_sizes() == o.leaf_sizes()).all()


def test_stm_batches_with_deletes(gpu):
    t, o, keys = pair("gamma", 91)
    for b in range(3):
        rk, rv, ro = with_deletes(*O.gen_requests("gamma", 92 + b, keys, 50_000, 60), seed=10 + b, frac=0.3)
        _, first = np.unique(rk, return_index=True)
        sel = np.sort(first)
        rk, rv, ro = rk[sel], rv[sel], ro[sel]
        ov, os_ = o.execute_serial(rk, rv, ro)
        gv, gs = run_batch(t, rk, rv, ro, E.MODE_STM)
        assert (gs == os_).all() and (gv == ov).all()
    same_contents(t, o)


@pytest.mark.parametrize("mode", [E.MODE_SORTED | E.MODE_MERGE_ENGINE, E.MODE_STM])
def test_delete_all_then_refill(gpu, mode):
    t, o, keys = pair("uniform", 95, n=50_000)
    sk = np.sort(keys)
    gv, gs = run_batch(t, sk, sk, np.full(sk.size, 2, np.uint8), mode)
    assert (gs == 1).all() and (gv == O.value_of(sk)).all()
    assert t.size() == 0 and dump(t)[0].size == 0
    # searches in the emptied leaves find nothing; refilling works in both modes
    gv, gs = run_batch(t, sk[:1000], sk[:1000], np.ones(1000, np.uint8), E.MODE_SORTED)
    assert (gs == 0).all()
    rk = sk[::-1].copy()
    gv, gs = run_batch(t, rk, rk + np.uint64(3), np.zeros(rk.size, np.uint8), mode)
    assert (gs == 0).all()
    k, v = dump(t)
    assert (k == sk).all() and (v == sk + np.uint64(3)).all()


def test_serving_with_deletes(gpu):
    t, o, keys = pair("uniform", 97)
    rk, rv, ro = with_deletes(*O.gen_requests("uniform", 98, keys, 30_000, 70), seed=5, frac=0.3)
    _, first = np.unique(rk, return_index=True)
    sel = np.sort(first)
    rk, rv, ro = rk[sel], rv[sel], ro[sel]
    ov, os_ = o.execute_serial(rk, rv, ro)
    srv = E.Server(t)
    out_v = np.zeros(rk.size, np.uint64)
    out_s = np.zeros(rk.size, np.uint8)
    srv.wait(srv.submit(rk, rv, ro, out_v, out_s))
    srv.stop()
    assert (out_s == os_).all() and (out_v == ov).all()
    same_contents(t, o)
