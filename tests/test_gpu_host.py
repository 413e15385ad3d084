"""The host-buffer entry point (bt_execute_batch_host) against the oracle and
against the device-buffer entry point on a twin tree.  Sorted batches overlap
the value copy with the front end and the answer copy with the write phase;
these tests cover every layout of that pipeline: both front ends, both
insert engines, the side stream on and off, DELETE runs, repeated keys, and a
node pool that runs out (the kNoCapacity answers are rewritten after the
write phase and copied again)."""
import numpy as np
import pytest

import eirene_b200 as E
from oracle import oracle as O
from tests.helpers import dev, dump, run_batch

pytestmark = pytest.mark.gpu
MERGE = E.MODE_SORTED | E.MODE_MERGE_ENGINE


def with_deletes(k, v, o, seed, frac):
    rng = np.random.default_rng(seed)
    o = o.copy()
    o[rng.random(o.size) < frac] = E.OP_DELETE
    return k, v, o


def twins(dist, seed, n=80_000):
    keys = O.gen_keys(dist, seed, n)
    vals = O.value_of(keys)
    th = E.BTree(max_keys=1 << 21, max_batch=1 << 18)
    td = E.BTree(max_keys=1 << 21, max_batch=1 << 18)
    for t in (th, td):
        t.bulk_build(dev(keys), dev(vals))
    o = O.OracleTree()
    o.bulk_build(keys, vals)
    return th, td, o, keys


def same_contents(t, o):
    gk, gv = dump(t)
    ok, ov = o.dump()
    assert gk.size == ok.size and (gk == ok).all() and (gv == ov).all()


@pytest.mark.parametrize("overlap", [1, 0])
@pytest.mark.parametrize("front", [1, 0])
@pytest.mark.parametrize("engine", [E.MODE_MERGE_ENGINE, 0])
def test_host_batches_match_oracle_and_device(gpu, overlap, front, engine):
    th, td, o, keys = twins("zipf", 101)
    for t in (th, td):
        t.set_option(E.OPT_FRONT_END, front)
        t.set_option(E.OPT_OVERLAP, overlap)
    mode = E.MODE_SORTED | engine
    for b, (mix, frac) in enumerate([(95, 0.0), (50, 0.2), (80, 0.5), (0, 0.0)]):
        rk, rv, ro = with_deletes(*O.gen_requests("zipf", 102 + b, keys, 70_000, mix), seed=b, frac=frac)
        ov, os_ = o.execute_merged(rk, rv, ro, engine=O.ENGINE_MERGE if engine else O.ENGINE_STM)
        hv, hs = th.execute_host(rk, rv, ro, mode=mode)
        gv, gs = run_batch(td, rk, rv, ro, mode)
        bad = np.nonzero((hs != os_) | (hv != ov))[0]
        assert bad.size == 0, (b, bad[:5], ro[bad[:5]], hs[bad[:5]], os_[bad[:5]])
        assert (gs == hs).all() and (gv == hv).all()
        same_contents(th, o)
    if engine:
        assert (th.leaf_sizes() == o.leaf_sizes()).all()


def test_host_batches_from_empty_tree(gpu):
    # the first batch creates the root while the lookups of the same batch run
    t = E.BTree(max_keys=1 << 20, max_batch=1 << 16)
    o = O.OracleTree()
    rng = np.random.default_rng(7)
    for b in range(3):
        rk = rng.integers(1, 2**63, 40_000, dtype=np.uint64)
        rk[rng.random(rk.size) < 0.3] = rk[0]  # one hot key
        rv = rk ^ np.uint64(b + 1)
        ro = (rng.random(rk.size) < 0.4).astype(np.uint8)  # 60 % INSERT, 40 % GET
        ov, os_ = o.execute_merged(rk, rv, ro, engine=O.ENGINE_MERGE)
        hv, hs = t.execute_host(rk, rv, ro, mode=MERGE)
        assert (hs == os_).all() and (hv == ov).all()
    same_contents(t, o)


@pytest.mark.parametrize("host", [True, False])
def test_merge_engine_pool_exhaustion(gpu, host):
    # a pool too small for the batches: a batch whose new keys do not fit
    # answers kNoCapacity for every new key (all or nothing), updates of
    # existing keys still answer the old value, and the tree stays intact
    t = E.BTree(max_keys=0, max_batch=1 << 16)  # pool = 4096 nodes
    rng = np.random.default_rng(11)
    ins_ok = np.zeros(0, np.uint64)
    vals_now = {}
    failed = 0
    for b in range(12):
        new = rng.choice(2**40, 16384, replace=False).astype(np.uint64) + np.uint64(1)
        new = np.setdiff1d(new, ins_ok)
        old = ins_ok[rng.integers(0, ins_ok.size, 2048)] if ins_ok.size else np.zeros(0, np.uint64)
        old = np.unique(old)
        gets = ins_ok[rng.integers(0, ins_ok.size, 2048)] if ins_ok.size else np.zeros(0, np.uint64)
        gets = np.setdiff1d(gets, old)
        rk = np.concatenate([new, old, gets])
        rv = np.concatenate([new * np.uint64(3), old + np.uint64(b), gets])
        ro = np.concatenate([np.zeros(new.size + old.size, np.uint8), np.ones(gets.size, np.uint8)])
        perm = rng.permutation(rk.size)
        rk, rv, ro = rk[perm], rv[perm], ro[perm]
        if host:
            gv, gs = t.execute_host(rk, rv, ro, mode=MERGE)
        else:
            gv, gs = run_batch(t, rk, rv, ro, MERGE)
        is_new = np.isin(rk, new)
        st_new = np.unique(gs[is_new])
        assert st_new.size == 1 and st_new[0] in (E.ST_ABSENT, E.ST_NO_CAPACITY), st_new
        for i in np.nonzero(~is_new)[0]:
            assert gs[i] == E.ST_FOUND and gv[i] == vals_now[int(rk[i])]
        for i in np.nonzero(ro == 0)[0]:
            if not is_new[i] or st_new[0] == E.ST_ABSENT:
                vals_now[int(rk[i])] = int(rv[i])
        if st_new[0] == E.ST_ABSENT:
            ins_ok = np.union1d(ins_ok, new)
        else:
            failed += 1
    assert failed > 0 and ins_ok.size > 0
    assert t.stats()["error"] & 1
    k, v = dump(t)
    assert (k == ins_ok).all()
    assert all(int(vv) == vals_now[int(kk)] for kk, vv in zip(k[::97], v[::97]))


@pytest.mark.parametrize("pinned,in_place", [(True, 0), (True, 1), (False, 0), (False, 1)])
@pytest.mark.parametrize("mode", [MERGE, E.MODE_SORTED, E.MODE_STM])
def test_async_host_batches_in_flight(gpu, pinned, in_place, mode):
    # bt_execute_batch_host_async: four batches queued before the first wait
    # (the fourth submit waits for the first of the three staging sets), answers
    # request by request against the oracle.  With page-locked buffers and
    # OPT_HOST_VALUES_IN_PLACE the sorted modes read the values of the writes
    # over the bus instead of copying the value array; otherwise it is copied.
    import torch

    keys = O.gen_keys("uniform", 301, 60_000)
    vals = O.value_of(keys)
    t = E.BTree(max_keys=1 << 20, max_batch=1 << 16)
    t.bulk_build(dev(keys), dev(vals))
    t.set_option(E.OPT_HOST_VALUES_IN_PLACE, in_place)  # pageable values are copied either way
    o = O.OracleTree()
    o.bulk_build(keys, vals)
    bufs, pinned_bufs, expect = [], [], []
    for b in range(5):
        rk, rv, ro = O.gen_requests("uniform", 310 + b, keys, 40_000 + 997 * b, 80)
        if mode == E.MODE_STM:  # the v39 meaning: compare batches without repeated keys
            _, at = np.unique(rk, return_index=True)
            sel = np.sort(at)
            rk, rv, ro = rk[sel], rv[sel], ro[sel]
            expect.append(o.execute_serial(rk, rv, ro))
        else:
            expect.append(o.execute_merged(rk, rv, ro, engine=O.ENGINE_MERGE))
        n = rk.size
        if pinned:
            hb = [E.HostBuffer(n, d) for d in (torch.int64, torch.int64, torch.uint8, torch.int64, torch.uint8)]
            pinned_bufs += hb
            hb[0].tensor.numpy().view(np.uint64)[:] = rk
            hb[1].tensor.numpy().view(np.uint64)[:] = rv
            hb[2].tensor.numpy()[:] = ro
            bufs.append([x.tensor for x in hb])
        else:
            bufs.append([torch.from_numpy(rk.view(np.int64).copy()), torch.from_numpy(rv.view(np.int64).copy()),
                         torch.from_numpy(ro.copy()), torch.zeros(n, dtype=torch.int64),
                         torch.zeros(n, dtype=torch.uint8)])
    tickets = []
    for b in range(4):
        tickets.append(t.submit_host(*bufs[b], mode=mode))
    t.wait_host(tickets[2])  # out of order: batches run in submission order anyway
    t.wait_host(tickets[1])
    tickets.append(t.submit_host(*bufs[4], mode=mode))
    for tk in tickets[3:]:
        t.wait_host(tk)
    assert tickets == sorted(tickets) and len(set(tickets)) == 5
    t.wait_host(tickets[0])  # an old ticket: finished long ago
    with pytest.raises(E.BTError):
        t.wait_host(tickets[-1] + 1)  # never issued
    for b in range(5):
        ov, os_ = expect[b]
        gv = bufs[b][3].numpy().view(np.uint64)
        gs = bufs[b][4].numpy()
        assert (gs == os_).all(), b
        assert (gv == ov).all(), b
    t.sync()
    gk, gvv = dump(t)
    ok, ovv = o.dump()
    assert (gk == ok).all() and (gvv == ovv).all()
    del bufs
    for hbuf in pinned_bufs:
        hbuf.free()


@pytest.mark.parametrize("pinned", [True, False])
@pytest.mark.parametrize("mode", [MERGE, E.MODE_SORTED, E.MODE_STM])
def test_packed_insert_values(gpu, pinned, mode):
    # bt_execute_batch_host_packed_async: only the INSERTs' values cross the
    # bus, packed in request order.  Batches of 95/5, 50/50, all GETs (no
    # value at all) and DELETE runs, sizes that are not a multiple of the
    # eight-byte count step or of a tile, two in flight; answers request by
    # request and the final contents against the oracle.
    import torch

    keys = O.gen_keys("uniform", 401, 60_000)
    vals = O.value_of(keys)
    t = E.BTree(max_keys=1 << 20, max_batch=1 << 16)
    t.bulk_build(dev(keys), dev(vals))
    o = O.OracleTree()
    o.bulk_build(keys, vals)
    shapes = [(40_001, 95, 0.0), (33_333, 50, 0.0), (20_007, 100, 0.0), (45_555, 80, 0.1), (7, 50, 0.0)]
    bufs, keep, expect, n_ins = [], [], [], []
    for b, (n, pct, dfrac) in enumerate(shapes):
        rk, rv, ro = O.gen_requests("uniform", 410 + b, keys, n, pct)
        if dfrac:
            rk, rv, ro = with_deletes(rk, rv, ro, 420 + b, dfrac)
        if mode == E.MODE_STM:  # the v39 meaning: compare batches without repeated keys
            _, at = np.unique(rk, return_index=True)
            sel = np.sort(at)
            rk, rv, ro = rk[sel], rv[sel], ro[sel]
            expect.append(o.execute_serial(rk, rv, ro))
        else:
            expect.append(o.execute_merged(rk, rv, ro, engine=O.ENGINE_MERGE))
        iv = rv[ro == E.OP_INSERT].copy()
        n_ins.append(iv.size)
        m = rk.size
        if pinned:
            hb = [E.HostBuffer(m, torch.int64), E.HostBuffer(m, torch.uint8), E.HostBuffer(max(iv.size, 1), torch.int64),
                  E.HostBuffer(m, torch.int64), E.HostBuffer(m, torch.uint8)]
            keep += hb
            hb[0].tensor.numpy().view(np.uint64)[:] = rk
            hb[1].tensor.numpy()[:] = ro
            hb[2].tensor.numpy().view(np.uint64)[: iv.size] = iv
            ts = [x.tensor for x in hb]
            ts[2] = ts[2][: iv.size]
        else:
            ts = [torch.from_numpy(rk.view(np.int64).copy()), torch.from_numpy(ro.copy()),
                  torch.from_numpy(iv.view(np.int64).copy()), torch.zeros(m, dtype=torch.int64),
                  torch.zeros(m, dtype=torch.uint8)]
        bufs.append(ts)
    assert n_ins[2] == 0  # an all-GET batch sends no value
    tickets = []
    for b in range(len(shapes)):  # three in flight
        if b >= 3:
            t.wait_host(tickets[b - 3])
        tickets.append(t.submit_host_packed(*bufs[b], mode=mode))
    for tk in tickets[-3:]:
        t.wait_host(tk)
    for b in range(len(shapes)):
        ov, os_ = expect[b]
        assert (bufs[b][4].numpy() == os_).all(), b
        assert (bufs[b][3].numpy().view(np.uint64) == ov).all(), b
    t.sync()
    gk, gvv = dump(t)
    ok, ovv = o.dump()
    assert (gk == ok).all() and (gvv == ovv).all()
    # a count that does not match the op codes: every request rejected,
    # nothing applied, and the batch's wait reports it (also once its
    # staging set has been reused); the next batch runs normally
    rk, rv, ro = O.gen_requests("uniform", 430, keys, 1000, 50)
    iv = rv[ro == E.OP_INSERT]
    ok_, okv = o.dump()
    bad = []
    for wrong in (iv[:-1], np.concatenate([iv, iv[:1]])):
        st = torch.full((rk.size,), 9, dtype=torch.uint8)
        tk = t.submit_host_packed(torch.from_numpy(rk.view(np.int64).copy()), torch.from_numpy(ro.copy()),
                                  torch.from_numpy(wrong.view(np.int64).copy()), torch.zeros(rk.size, dtype=torch.int64),
                                  st, mode=mode)
        with pytest.raises(E.BTError) as ei:
            t.wait_host(tk)
        assert ei.value.code == -1  # BT_ERR_INVALID_ARG
        assert (st.numpy() == E.ST_REJECTED).all()
        bad.append(tk)
    good = [torch.zeros(rk.size, dtype=torch.int64), torch.zeros(rk.size, dtype=torch.uint8)]
    if mode == E.MODE_STM:
        _, at = np.unique(rk, return_index=True)
        sel = np.sort(at)
        rk, rv, ro = rk[sel], rv[sel], ro[sel]
        good = [g[: rk.size] for g in good]
        ov, os_ = o.execute_serial(rk, rv, ro)
    else:
        ov, os_ = o.execute_merged(rk, rv, ro, engine=O.ENGINE_MERGE)
    gk, gvv = dump(t)
    assert (gk == ok_).all() and (gvv == okv).all()  # the refused batches changed nothing
    iv = rv[ro == E.OP_INSERT]
    t.wait_host(t.submit_host_packed(torch.from_numpy(rk.view(np.int64).copy()), torch.from_numpy(ro.copy()),
                                     torch.from_numpy(iv.view(np.int64).copy()), *good, mode=mode))
    assert (good[1].numpy() == os_).all() and (good[0].numpy().view(np.uint64) == ov).all()
    # an all-GET batch (no values at all), then another: every staging set reused
    qk = ok_[:: max(1, ok_.size // 500)]
    qo = np.full(qk.size, E.OP_GET, np.uint8)
    gv_, gs_ = torch.zeros(qk.size, dtype=torch.int64), torch.zeros(qk.size, dtype=torch.uint8)
    for _ in range(2):
        t.wait_host(t.submit_host_packed(torch.from_numpy(qk.view(np.int64).copy()), torch.from_numpy(qo),
                                         torch.zeros(0, dtype=torch.int64), gv_, gs_, mode=mode))
    ek, ev = o.dump()
    assert (gs_.numpy() == 1).all() and (gv_.numpy().view(np.uint64) == ev[np.searchsorted(ek, qk)]).all()
    for tk in bad:  # both sets reused since: the refusals are still reported
        with pytest.raises(E.BTError):
            t.wait_host(tk)
    del bufs
    for hbuf in keep:
        hbuf.free()
