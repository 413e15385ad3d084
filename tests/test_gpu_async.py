"""Deferred write phase (OPT_ASYNC_WRITE): a sorted batch with the hash front
end and the merge engine completes on the caller's stream once its answers
are final, and its leaf/inner merge finishes on an internal stream.  Batches
issued back to back without a host sync, and every other call that reads the
tree right after such a batch, must see exactly what the synchronous order
gives: the same answers, contents and tree shape as the oracle."""
import numpy as np
import pytest

import eirene_b200 as E
from oracle import oracle as O
from tests.helpers import dev, dump, empty_u64, empty_u8, host_u64, host_u8, run_batch

pytestmark = pytest.mark.gpu
MERGE = E.MODE_SORTED | E.MODE_MERGE_ENGINE


def make(keys, async_write):
    t = E.BTree(max_keys=1 << 22, max_batch=1 << 18)
    t.bulk_build(dev(keys), dev(O.value_of(keys)))
    t.set_option(E.OPT_ASYNC_WRITE, async_write)
    return t


@pytest.mark.parametrize("overlap", [1, 0])
def test_back_to_back_batches_match_sync_and_oracle(gpu, overlap):
    import torch

    keys = O.gen_keys("uniform", 201, 200_000)
    ta, ts = make(keys, 1), make(keys, 0)
    for t in (ta, ts):
        t.set_option(E.OPT_OVERLAP, overlap)
    o = O.OracleTree()
    o.bulk_build(keys, O.value_of(keys))
    stream = torch.cuda.Stream()
    reqs, outs = [], []
    for b, mix in enumerate([95, 50, 5, 80, 95, 0]):
        rk, rv, ro = O.gen_requests("uniform", 210 + b, keys, 120_000, mix)
        ro = ro.copy()
        ro[np.random.default_rng(b).random(ro.size) < 0.05] = E.OP_DELETE
        reqs.append((rk, rv, ro))
    with torch.cuda.stream(stream):
        dreqs = [(dev(k), dev(v), dev(o_)) for (k, v, o_) in reqs]
        for t in (ta, ts):
            res = []
            for (k, v, o_) in dreqs:  # no host sync between the batches
                ov, ost = empty_u64(k.numel()), empty_u8(k.numel())
                t.execute(k, v, o_, ov, ost, mode=MERGE, stream=stream)
                res.append((ov, ost))
            outs.append(res)
    torch.cuda.synchronize()
    for b, (rk, rv, ro) in enumerate(reqs):
        ov, os_ = o.execute_merged(rk, rv, ro, engine=O.ENGINE_MERGE)
        av, ast = host_u64(outs[0][b][0]), host_u8(outs[0][b][1])
        sv, sst = host_u64(outs[1][b][0]), host_u8(outs[1][b][1])
        assert (ast == os_).all() and (av == ov).all(), b
        assert (sst == ast).all() and (sv == av).all(), b
    for t in (ta, ts):
        gk, gv = dump(t)
        ok, ov_ = o.dump()
        assert (gk == ok).all() and (gv == ov_).all()
        assert (t.leaf_sizes() == o.leaf_sizes()).all()
        assert (t.level_counts() == o.level_counts()).all()


def test_calls_after_a_deferred_batch_see_its_writes(gpu):
    # a lookup batch, a range scan, the size and bt_sync right after an
    # insert-heavy batch, on another stream than the batch's
    import torch

    keys = O.gen_keys("gamma", 301, 100_000)
    t = make(keys, 1)
    o = O.OracleTree()
    o.bulk_build(keys, O.value_of(keys))
    s1, s2 = torch.cuda.Stream(), torch.cuda.Stream()
    rng = np.random.default_rng(3)
    for b in range(4):
        new = rng.integers(1, 2**63, 50_000, dtype=np.uint64)
        rv = new ^ np.uint64(b + 7)
        ro = np.zeros(new.size, np.uint8)
        o.execute_merged(new, rv, ro, engine=O.ENGINE_MERGE)
        with torch.cuda.stream(s1):
            k, v, op = dev(new), dev(rv), dev(ro)
            ov, ost = empty_u64(new.size), empty_u8(new.size)
            t.execute(k, v, op, ov, ost, mode=MERGE, stream=s1)
        s1.synchronize()  # the answers only; the merge may still run
        with torch.cuda.stream(s2):
            qk = dev(new)
            qv, qs = empty_u64(new.size), empty_u8(new.size)
            t.search(qk, qv, qs, stream=s2)
        s2.synchronize()
        assert (host_u8(qs) == E.ST_FOUND).all() and (host_u64(qv) == rv).all()
        assert t.size() == o.size()
    t.sync()
    gk, gv = dump(t)
    ok, ov_ = o.dump()
    assert (gk == ok).all() and (gv == ov_).all()
    assert (t.leaf_sizes() == o.leaf_sizes()).all()


@pytest.mark.parametrize("overlap", [1, 0])
@pytest.mark.parametrize("async_write", [1, 0])
def test_lookup_before_first_write_sees_pre_batch_value(gpu, overlap, async_write):
    # GET k, then INSERT k, then GET k (and the same with DELETE): the first
    # GET is a plain lookup of the pre-batch tree and must not see the write,
    # which the merge engine locates while the lookups run
    keys = O.gen_keys("uniform", 401, 100_000)
    t = make(keys, async_write)
    t.set_option(E.OPT_OVERLAP, overlap)
    o = O.OracleTree()
    o.bulk_build(keys, O.value_of(keys))
    rng = np.random.default_rng(4)
    for b in range(3):
        k = rng.choice(keys, 30_000, replace=False)
        wr = np.where(rng.random(k.size) < 0.8, 0, E.OP_DELETE).astype(np.uint8)
        rk = np.concatenate([k, k, k])
        rv = np.concatenate([k, k ^ np.uint64(0xABC + b), k])
        ro = np.concatenate([np.ones(k.size, np.uint8), wr, np.ones(k.size, np.uint8)])
        ov, os_ = o.execute_merged(rk, rv, ro, engine=O.ENGINE_MERGE)
        gv, gs = run_batch(t, rk, rv, ro, MERGE)
        assert (gs == os_).all() and (gv == ov).all(), b
        assert (gv[: k.size] == O.value_of(k)).all() or b > 0
    gk, gv_ = dump(t)
    ok, ovv = o.dump()
    assert (gk == ok).all() and (gv_ == ovv).all()
