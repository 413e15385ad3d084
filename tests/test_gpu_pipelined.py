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


@pytest.mark.parametrize("learned", [False, True])
def test_host_batches_chain_beside_other_calls(gpu, learned):
    # host batches (BT_OPT_HOST_FRONT_OVERLAP on): each front part runs beside
    # the previous host batch's tree part.  Between them: device batches,
    # plain searches, bt_execute_batches, STM host batches, packed ones, the
    # option switched off and on; up to three host batches in flight.  Every
    # answer and the final tree against the oracle run in call order.
    import torch

    keys = O.gen_keys("uniform", 681, 100_000)
    vals = O.value_of(keys)
    t = E.BTree(max_keys=1 << 21, max_batch=1 << 17)
    t.bulk_build(dev(keys), dev(vals))
    o = O.OracleTree()
    o.bulk_build(keys, vals)
    if learned:
        t.retrain()
        t.set_descent(True)
    plan = ["host", "host", "host", "dev", "host", "host", "search", "host", "many", "host", "packed", "host",
            "off", "host", "host", "on", "host", "stm", "host", "host", "packed", "host"]
    keep, checks, inflight = [], [], []

    def host_tensors(rk, rv, ro):
        return [torch.from_numpy(rk.view(np.int64).copy()), torch.from_numpy(rv.view(np.int64).copy()),
                torch.from_numpy(ro.copy()), torch.zeros(rk.size, dtype=torch.int64),
                torch.zeros(rk.size, dtype=torch.uint8)]

    for i, what in enumerate(plan):
        if what == "off":
            t.set_option(E.OPT_HOST_FRONT_OVERLAP, 0)
            continue
        if what == "on":
            t.set_option(E.OPT_HOST_FRONT_OVERLAP, 1)
            continue
        n = 20_000 + 3_331 * (i % 5)
        rk, rv, ro = O.gen_requests("uniform", 690 + i, keys, n, 50 if i % 3 else 90)
        if what == "stm":
            _, at = np.unique(rk, return_index=True)
            sel = np.sort(at)
            rk, rv, ro = rk[sel], rv[sel], ro[sel]
            ex = o.execute_serial(rk, rv, ro)
        elif what == "search":
            ro = np.full(rk.size, E.OP_GET, dtype=np.uint8)
            ex = o.execute_merged(rk, rv, ro, engine=O.ENGINE_MERGE)
        else:
            ex = o.execute_merged(rk, rv, ro, engine=O.ENGINE_MERGE)
        if what in ("host", "stm"):
            hb = host_tensors(rk, rv, ro)
            tk = t.submit_host(*hb, mode=E.MODE_STM if what == "stm" else MERGE)
            keep.append(hb)
            checks.append((ex, hb[3], hb[4], True))
            inflight.append(tk)
        elif what == "packed":
            hb = host_tensors(rk, rv, ro)
            ins = torch.from_numpy(rv[ro == E.OP_INSERT].view(np.int64).copy())
            tk = t.submit_host_packed(hb[0], hb[2], ins, hb[3], hb[4], mode=MERGE)
            keep.append(hb + [ins])
            checks.append((ex, hb[3], hb[4], True))
            inflight.append(tk)
        elif what == "dev":
            a, s = empty_u64(rk.size), empty_u8(rk.size)
            d = (dev(rk), dev(rv), dev(ro))
            t.execute(*d, a, s, mode=MERGE)
            keep.append(d)
            checks.append((ex, a, s, False))
        elif what == "search":
            a, s = empty_u64(rk.size), empty_u8(rk.size)
            d = dev(rk)
            t.search(d, a, s)
            keep.append(d)
            checks.append((ex, a, s, False))
        elif what == "many":
            # this batch and a second one drawn after it
            rk2, rv2, ro2 = O.gen_requests("uniform", 790 + i, keys, 17_777, 70)
            ex2 = o.execute_merged(rk2, rv2, ro2, engine=O.ENGINE_MERGE)
            bs = [(dev(rk), dev(rv), dev(ro)), (dev(rk2), dev(rv2), dev(ro2))]
            outs = [(empty_u64(rk.size), empty_u8(rk.size)), (empty_u64(rk2.size), empty_u8(rk2.size))]
            t.execute_many(bs, outs, mode=MERGE)
            keep.append((bs, outs))
            checks.append((ex, outs[0][0], outs[0][1], False))
            checks.append((ex2, outs[1][0], outs[1][1], False))
        while len(inflight) > 2:
            t.wait_host(inflight.pop(0))
    for tk in inflight:
        t.wait_host(tk)
    t.sync()
    for j, ((ov, os_), a, s, host) in enumerate(checks):
        ga = a.numpy().view(np.uint64) if host else host_u64(a)
        gs = s.numpy() if host else host_u8(s)
        assert (gs == os_).all(), j
        assert (ga == ov).all(), j
    gk, gv = dump(t)
    ok, ovv = o.dump()
    assert (gk == ok).all() and (gv == ovv).all()
