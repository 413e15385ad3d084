"""The tree epoch (15 bits of the node header) wraps after 32767 bulk builds
on one handle.  At the wrap every row's header is cleared, so no row of an
earlier tree can pass the epoch check of the optimistic readers; the tree
built after the wrap answers exactly in every mode."""
import numpy as np
import pytest

import eirene_b200 as E
from oracle import oracle as O
from tests.helpers import dev, dump, empty_u64, empty_u8, host_u64, host_u8, run_batch

pytestmark = pytest.mark.gpu


def test_epoch_wrap_keeps_trees_exact(gpu):
    t = E.BTree(max_keys=1 << 14, max_batch=1 << 12)
    first = O.gen_keys("uniform", 90, 5000)
    t.bulk_build(dev(first), dev(O.value_of(first)))  # epoch 1, about 210 leaves
    one_k = dev(np.array([5], np.uint64))
    one_v = dev(np.array([6], np.uint64))
    for _ in range(0x7FFF - 1):  # epochs 2 .. 0x7fff
        t.bulk_build(one_k, one_v)
    assert t.size() == 1
    # the next build comes round to epoch 1 again
    keys = O.gen_keys("uniform", 91, 300)
    vals = O.value_of(keys)
    t.bulk_build(dev(keys), dev(vals))
    o = O.OracleTree()
    o.bulk_build(keys, vals)
    # STM inserts allocate the rows the first tree used, and the learned
    # guess and the optimistic descent check epochs
    t.retrain()
    t.set_descent(True)
    rk, rv, ro = O.gen_requests("uniform", 92, keys, 4000, 40)
    _, at = np.unique(rk, return_index=True)
    sel = np.sort(at)
    rk, rv, ro = rk[sel], rv[sel], ro[sel]
    ov, os_ = o.execute_serial(rk, rv, ro)
    gv, gs = run_batch(t, rk, rv, ro, E.MODE_STM)
    assert (gs == os_).all() and (gv == ov).all()
    rk, rv, ro = O.gen_requests("uniform", 93, keys, 4000, 60)
    ov, os_ = o.execute_merged(rk, rv, ro, engine=O.ENGINE_MERGE)
    gv, gs = run_batch(t, rk, rv, ro, E.MODE_SORTED | E.MODE_MERGE_ENGINE)
    assert (gs == os_).all() and (gv == ov).all()
    qk = o.dump()[0]
    v, s = empty_u64(qk.size), empty_u8(qk.size)
    t.search(dev(qk), v, s)
    assert (host_u8(s) == 1).all() and (host_u64(v) == o.dump()[1]).all()
    gk, gvv = dump(t)
    ok, ovv = o.dump()
    assert (gk == ok).all() and (gvv == ovv).all()
