"""bt_execute_batches: several batches in one call, batch j + 1's front part
(classification, sort, merge passes) beside batch j's lookups and writes,
with alternate buffer sets.  The answers of every batch and the final tree
must be those of the batches run one by one (the oracle), for both descents,
mixes with DELETE runs and repeated keys, an empty batch in the list, and
batches of different sizes; STM-mode lists run one by one."""
import numpy as np
import pytest

import eirene_b200 as E
from oracle import oracle as O
from tests.helpers import dev, dump, empty_u64, empty_u8, host_u64, host_u8

pytestmark = pytest.mark.gpu
MERGE = E.MODE_SORTED | E.MODE_MERGE_ENGINE


def with_deletes(k, v, o, seed, frac):
    rng = np.random.default_rng(seed)
    o = o.copy()
    o[rng.random(o.size) < frac] = E.OP_DELETE
    return k, v, o


@pytest.mark.parametrize("learned", [False, True])
def test_pipelined_batches_match_one_by_one(gpu, learned):
    keys = O.gen_keys("uniform", 601, 120_000)
    vals = O.value_of(keys)
    t = E.BTree(max_keys=1 << 21, max_batch=1 << 17)
    t.bulk_build(dev(keys), dev(vals))
    o = O.OracleTree()
    o.bulk_build(keys, vals)
    if learned:
        t.retrain()
        t.set_descent(True)
    shapes = [(60_000, 95, 0.0), (40_001, 50, 0.05), (0, 95, 0.0), (70_000, 80, 0.0), (9, 50, 0.0),
              (65_536, 95, 0.02), (33_333, 60, 0.0)]
    batches, outs, expect = [], [], []
    for b, (n, pct, dfrac) in enumerate(shapes):
        if n == 0:
            batches.append((empty_u64(0), empty_u64(0), empty_u8(0)))
            outs.append((empty_u64(0), empty_u8(0)))
            expect.append(None)
            continue
        rk, rv, ro = O.gen_requests("uniform", 610 + b, keys, n, pct)
        if b == 3:  # repeated keys inside the batch
            rk[1::7] = rk[::7][: rk[1::7].size]
        if dfrac:
            rk, rv, ro = with_deletes(rk, rv, ro, 620 + b, dfrac)
        expect.append(o.execute_merged(rk, rv, ro, engine=O.ENGINE_MERGE))
        batches.append((dev(rk), dev(rv), dev(ro)))
        outs.append((empty_u64(n), empty_u8(n)))
    t.execute_many(batches, outs, mode=MERGE)
    t.sync()
    for b, ex in enumerate(expect):
        if ex is None:
            continue
        ov, os_ = ex
        assert (host_u8(outs[b][1]) == os_).all(), b
        assert (host_u64(outs[b][0]) == ov).all(), b
    gk, gv = dump(t)
    ok, ovv = o.dump()
    assert (gk == ok).all() and (gv == ovv).all()
    # a one-by-one batch after the pipelined ones sees their tree
    rk, rv, ro = O.gen_requests("uniform", 640, keys, 50_000, 90)
    ov, os_ = o.execute_merged(rk, rv, ro, engine=O.ENGINE_MERGE)
    a, s = empty_u64(rk.size), empty_u8(rk.size)
    t.execute(dev(rk), dev(rv), dev(ro), a, s, mode=MERGE)
    assert (host_u8(s) == os_).all() and (host_u64(a) == ov).all()
    # and a second pipelined call after it
    more, mouts, mexp = [], [], []
    for b in range(3):
        rk, rv, ro = O.gen_requests("uniform", 650 + b, keys, 30_000 + b, 70)
        mexp.append(o.execute_merged(rk, rv, ro, engine=O.ENGINE_MERGE))
        more.append((dev(rk), dev(rv), dev(ro)))
        mouts.append((empty_u64(rk.size), empty_u8(rk.size)))
    t.execute_many(more, mouts, mode=MERGE)
    for b, (ov, os_) in enumerate(mexp):
        assert (host_u8(mouts[b][1]) == os_).all() and (host_u64(mouts[b][0]) == ov).all(), b
    t.sync()
    gk, gv = dump(t)
    ok, ovv = o.dump()
    assert (gk == ok).all() and (gv == ovv).all()


def test_pipelined_stm_runs_one_by_one(gpu):
    keys = O.gen_keys("uniform", 661, 80_000)
    vals = O.value_of(keys)
    t = E.BTree(max_keys=1 << 20, max_batch=1 << 16)
    t.bulk_build(dev(keys), dev(vals))
    o = O.OracleTree()
    o.bulk_build(keys, vals)
    batches, outs, expect = [], [], []
    for b in range(3):
        rk, rv, ro = O.gen_requests("uniform", 670 + b, keys, 30_000, 80)
        _, at = np.unique(rk, return_index=True)
        sel = np.sort(at)
        rk, rv, ro = rk[sel], rv[sel], ro[sel]
        expect.append(o.execute_serial(rk, rv, ro))
        batches.append((dev(rk), dev(rv), dev(ro)))
        outs.append((empty_u64(rk.size), empty_u8(rk.size)))
    t.execute_many(batches, outs, mode=E.MODE_STM)
    for b, (ov, os_) in enumerate(expect):
        assert (host_u8(outs[b][1]) == os_).all() and (host_u64(outs[b][0]) == ov).all(), b
