"""Key-range sharding on the GPU: the routing kernels against a stable
partition restated in numpy, and the whole sharded pipeline (route -> all-to-all
-> owner batch -> reverse all-to-all -> unroute) with 4 ranks emulated as host
threads on one GPU.  The threads' exchange is host barriers plus device
copies; no kernel waits on another, so the emulation runs on one GPU safely.
The answers and contents must equal ONE oracle tree over the concatenation of
the ranks' batches in rank order."""
import threading

import numpy as np
import pytest
import torch

import eirene_b200 as E
from eirene_b200.shard import ShardedBTree
from oracle import oracle as O
from tests.helpers import dev, empty_u64, empty_u8, host_u64, host_u8

pytestmark = pytest.mark.gpu


def np_route(spl, keys, n_shards):
    ids = np.searchsorted(spl, keys, side="right")
    perm = np.argsort(ids, kind="stable")
    return perm, np.bincount(ids, minlength=n_shards)


@pytest.mark.parametrize("n,n_shards,dup,cap", [(0, 4, False, 1), (1, 1, False, 1), (1, 8, False, 1),
                                                (4095, 8, False, 4095), (4096, 8, True, 4096),
                                                (100_000, 8, False, 100_000), (1 << 20, 256, True, 1 << 20),
                                                (77_777, 2, False, 77_777), (300_001, 5, False, 4096)])
def test_route_matches_stable_partition(gpu, n, n_shards, dup, cap):
    # cap < n: the input is larger than the handle's batch buffers (temporaries)
    rng = np.random.default_rng(n + n_shards)
    t = E.BTree(max_keys=1 << 12, max_batch=cap)
    keys = rng.integers(0, 2**64, n, dtype=np.uint64, endpoint=False)
    pool = keys if n else rng.integers(0, 2**64, 16, dtype=np.uint64)
    spl = np.sort(rng.choice(pool, n_shards - 1)) if n_shards > 1 else np.zeros(0, np.uint64)
    if dup and n_shards > 3:
        spl[1] = spl[2]  # an empty shard
    if n > 10:
        keys[:3] = spl[:3] if spl.size >= 3 else keys[:3]  # keys equal to splitters go right
        keys[5] = np.uint64(2**64 - 1)
    vals = rng.integers(0, 2**64, n, dtype=np.uint64)
    ops = rng.integers(0, 2, n).astype(np.uint8)
    rk, rv, ro = empty_u64(n), empty_u64(n), empty_u8(n)
    perm = torch.zeros(max(n, 1), dtype=torch.int32, device="cuda")[:n]
    counts = torch.zeros(n_shards, dtype=torch.int64, device="cuda")
    t.route(dev(spl) if spl.size else None, n_shards, dev(keys), dev(vals), dev(ops), rk, rv, ro, perm, counts)
    torch.cuda.synchronize()
    ep, ec = np_route(spl, keys, n_shards)
    assert (counts.cpu().numpy() == ec).all()
    assert (perm.cpu().numpy() == ep).all()
    assert (host_u64(rk) == keys[ep]).all() and (host_u64(rv) == vals[ep]).all() and (host_u8(ro) == ops[ep]).all()
    # answers in routed order scatter back to input order
    bv, bs = empty_u64(n), empty_u8(n)
    t.unroute(perm, rv, ro, bv, bs)
    torch.cuda.synchronize()
    assert (host_u64(bv) == vals).all() and (host_u8(bs) == ops).all()


class _Shared:
    def __init__(self, world):
        self.world = world
        self.barrier = threading.Barrier(world, timeout=300)
        self.slots = [None] * world


class ThreadComm:
    """The exchange between ranks that are threads of one process on one GPU."""

    def __init__(self, shared, rank):
        self.s, self.rank, self.world = shared, rank, shared.world

    def _sync(self):
        self.s.barrier.wait()

    def all_to_all_single(self, out, inp, out_splits=None, in_splits=None):
        w = self.world
        if in_splits is None:
            in_splits = [inp.numel() // w] * w
        self.s.slots[self.rank] = (inp, list(in_splits))
        self._sync()
        off = 0
        for src in range(w):
            sinp, ssp = self.s.slots[src]
            start, m = sum(ssp[: self.rank]), ssp[self.rank]
            out[off:off + m].copy_(sinp[start:start + m])
            off += m
        assert off == out.numel()
        torch.cuda.synchronize()
        self._sync()

    def all_gather(self, parts, t):
        self.s.slots[self.rank] = t
        self._sync()
        for i in range(self.world):
            parts[i].copy_(self.s.slots[i])
        torch.cuda.synchronize()
        self._sync()

    def all_reduce_sum(self, t):
        self.s.slots[self.rank] = t.clone()
        self._sync()
        total = sum(x.to(t.device) for x in self.s.slots)
        self._sync()
        t.copy_(total)


def _inputs(dist, rank, n_build, n_batch, steps, pct, distinct):
    keys = O.gen_keys(dist, 500 + rank, n_build)
    vals = O.value_of(keys) ^ np.uint64(rank + 1)
    out = []
    for i in range(steps):
        k, v, o = O.gen_requests(dist, 900 + 10 * i + rank, keys, n_batch, pct)
        if rank > 0 and not distinct:
            k0, _, _ = O.gen_requests(dist, 900 + 10 * i, O.gen_keys(dist, 500, n_build), n_batch, pct)
            m = n_batch // 10
            k[:m], o[:m] = k0[:m], 0
            v[:m] = np.arange(m, dtype=np.uint64) + np.uint64(7_000_000 * rank)
        if distinct:
            _, first = np.unique(k, return_index=True)
            sel = np.sort(first)
            k, v, o = k[sel], v[sel], o[sel]
        out.append((k, v, o))
    return keys, vals, out


@pytest.mark.parametrize("dist,mode,pct", [("uniform", E.MODE_SORTED, 80),
                                           ("zipf", E.MODE_SORTED | E.MODE_MERGE_ENGINE, 50),
                                           ("gamma", E.MODE_STM, 70)])
def test_four_thread_ranks_equal_one_tree(gpu, dist, mode, pct):
    world, n_build, n_batch, steps, max_batch = 4, 40_000, 8_000, 3, 8_192
    distinct = mode == E.MODE_STM
    inputs = [_inputs(dist, r, n_build, n_batch, steps, pct, distinct) for r in range(world)]
    shared = _Shared(world)
    results = [None] * world
    errors = []
    dev_id = torch.cuda.current_device()

    def rank_main(r):
        try:
            torch.cuda.set_device(dev_id)
            st = ShardedBTree.on_gpu(comm=ThreadComm(shared, r), sample_per_rank=512, max_keys=1 << 19,
                                     max_batch=max_batch)
            keys, vals, batches = inputs[r]
            st.bulk_build(dev(keys), dev(vals))
            outs = []
            for k, v, o in batches:
                ov, os_ = empty_u64(k.size), empty_u8(k.size)
                st.execute(dev(k), dev(v), dev(o), ov, os_, mode=mode)
                torch.cuda.synchronize()
                outs.append((host_u64(ov), host_u8(os_)))
            dk, dv = st.dump_local()
            results[r] = (outs, host_u64(dk), host_u64(dv), st.size(), st.owner_range())
            st.ops.tree.close()
        except BaseException as e:  # noqa: BLE001 - reported below
            errors.append((r, repr(e)))
            shared.barrier.abort()

    th = [threading.Thread(target=rank_main, args=(r,)) for r in range(world)]
    for x in th:
        x.start()
    for x in th:
        x.join(600)
    assert not errors, errors
    one = O.OracleTree()
    one.bulk_build(np.concatenate([x[0] for x in inputs]), np.concatenate([x[1] for x in inputs]))
    for i in range(steps):
        cat = [np.concatenate([x[2][i][j] for x in inputs]) for j in range(3)]
        ev, es = one.execute_serial(*cat) if distinct else one.execute_merged(*cat)
        off = 0
        for r in range(world):
            gv, gs = results[r][0][i]
            n = gv.size
            assert (gs == es[off:off + n]).all() and (gv == ev[off:off + n]).all(), (i, r)
            off += n
    ok, ov = one.dump()
    assert (np.concatenate([x[1] for x in results]) == ok).all()
    assert (np.concatenate([x[2] for x in results]) == ov).all()
    assert all(x[3] == ok.size for x in results)
    for r in range(world):
        lo, hi = results[r][4]
        if results[r][1].size:
            assert int(results[r][1][0]) >= lo and (hi is None or int(results[r][1][-1]) < hi)
