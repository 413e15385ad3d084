"""The sort of the hash front end's touched requests (BT_OPT_TOUCH_SORT):
tile sort plus merge rounds, the onesweep radix sort and the choice between
them by the touched count seen last (default), against the oracle.  Touched counts from one tile to many merge rounds (a 50/50
batch of 2^20 has about 2^19 touched requests: eight rounds), repeated keys
with every op code in their runs, and keys that agree in their high bits."""
import numpy as np
import pytest

import eirene_b200 as E
from oracle import oracle as O
from tests.helpers import dev, dump, run_batch

pytestmark = pytest.mark.gpu
MERGE = E.MODE_SORTED | E.MODE_MERGE_ENGINE


@pytest.mark.parametrize("touch_sort", [2, 1, 0])
@pytest.mark.parametrize("n, pct, dfrac", [(1_000, 90, 0.0), (2_049, 50, 0.0), (60_000, 95, 0.02),
                                            (1 << 20, 50, 0.05)])
def test_touched_sort_matches_oracle(gpu, touch_sort, n, pct, dfrac):
    keys = O.gen_keys("uniform", 801, 200_000)
    vals = O.value_of(keys)
    t = E.BTree(max_keys=1 << 22, max_batch=1 << 20)
    t.set_option(E.OPT_TOUCH_SORT, touch_sort)
    t.bulk_build(dev(keys), dev(vals))
    o = O.OracleTree()
    o.bulk_build(keys, vals)
    rng = np.random.default_rng(802 + n)
    for b in range(3):
        rk, rv, ro = O.gen_requests("uniform", 810 + b + n, keys, n, pct)
        # runs of one key with INSERT, GET and DELETE requests in them
        hot = rk[rng.integers(0, n, max(1, n // 64))]
        at = rng.integers(0, n, n // 8)
        rk[at] = hot[rng.integers(0, hot.size, at.size)]
        if dfrac:
            ro[rng.random(n) < dfrac] = E.OP_DELETE
        ov, os_ = o.execute_merged(rk, rv, ro, engine=O.ENGINE_MERGE)
        gv, gs = run_batch(t, rk, rv, ro, MERGE)
        assert (gs == os_).all() and (gv == ov).all(), b
    t.sync()
    gk, gvv = dump(t)
    ok, ovv = o.dump()
    assert (gk == ok).all() and (gvv == ovv).all()


def test_touched_sort_high_bits_shared(gpu):
    # keys that share their high 40 bits: the order comes from the low bits
    base = np.uint64(0x5A5A5A5A5A) << np.uint64(24)
    rng = np.random.default_rng(811)
    keys = np.unique(base + rng.integers(0, 1 << 24, 30_000).astype(np.uint64))
    vals = O.value_of(keys)
    t = E.BTree(max_keys=1 << 20, max_batch=1 << 18)
    t.bulk_build(dev(keys), dev(vals))
    o = O.OracleTree()
    o.bulk_build(keys, vals)
    n = 150_000
    rk = base + rng.integers(0, 1 << 24, n).astype(np.uint64)
    ro = np.where(rng.random(n) < 0.4, E.OP_INSERT, E.OP_GET).astype(np.uint8)
    rv = rng.integers(0, 1 << 62, n).astype(np.uint64)
    ov, os_ = o.execute_merged(rk, rv, ro, engine=O.ENGINE_MERGE)
    gv, gs = run_batch(t, rk, rv, ro, MERGE)
    assert (gs == os_).all() and (gv == ov).all()
    t.sync()
    gk, gvv = dump(t)
    ok, ovv = o.dump()
    assert (gk == ok).all() and (gvv == ovv).all()
