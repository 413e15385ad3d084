"""Key-range sharding on CPU: world_size 2 and 3 over gloo, the exchange logic
of eirene_b200.shard with each rank's tree and routing restated on the CPU by
the oracle.  The sharded answers and contents must equal ONE oracle tree
running the concatenation of all ranks' batches in rank order."""
import os
import socket
import sys

import numpy as np
import pytest
import torch
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

from eirene_b200.shard import pick_splitters  # noqa: E402
from oracle import oracle as O  # noqa: E402

MODE_SORTED, MODE_STM = 0, 1


class OracleShardOps:
    """CPU stand-in for DeviceShardOps: numpy routing, oracle tree."""

    def __init__(self, max_batch):
        self.max_batch = max_batch
        self.tree = O.OracleTree()
        self.device = torch.device("cpu")

    @staticmethod
    def _u64(t):
        return t.numpy().view(np.uint64)

    def empty(self, n, dtype):
        return torch.zeros(n, dtype=dtype)

    def from_numpy(self, a):
        a = np.ascontiguousarray(a)
        return torch.from_numpy(a.view(np.int64) if a.dtype == np.uint64 else a)

    def route(self, splitters, n_shards, keys, vals, ops):
        k = self._u64(keys)
        ids = np.searchsorted(self._u64(splitters), k, side="right")
        perm = np.argsort(ids, kind="stable")
        counts = np.bincount(ids, minlength=n_shards).astype(np.int64)
        rv = torch.from_numpy(vals.numpy()[perm].copy()) if vals is not None else None
        ro = torch.from_numpy(ops.numpy()[perm].copy()) if ops is not None else None
        return (torch.from_numpy(keys.numpy()[perm].copy()), rv, ro, torch.from_numpy(perm.astype(np.int32)),
                torch.from_numpy(counts))

    def unroute(self, perm, in_vals, in_status, out_vals, out_status):
        p = perm.numpy().astype(np.int64)
        out_vals.numpy()[p] = in_vals.numpy()
        out_status.numpy()[p] = in_status.numpy()

    def bulk_build(self, keys, vals):
        self.tree.bulk_build(self._u64(keys).copy(), self._u64(vals).copy())

    def execute(self, keys, vals, ops, out_vals, out_status, mode):
        assert keys.numel() <= self.max_batch
        args = (self._u64(keys).copy(), self._u64(vals).copy(), ops.numpy().astype(np.uint8))
        if mode == MODE_STM:
            v, s = self.tree.execute_serial(*args)
        else:
            v, s = self.tree.execute_merged(*args)
        out_vals.numpy()[:] = v.view(np.int64)
        out_status.numpy()[:] = s

    def size(self):
        return self.tree.size()

    def dump(self):
        k, v = self.tree.dump()
        return torch.from_numpy(k.view(np.int64)), torch.from_numpy(v.view(np.int64))


def rank_inputs(case, rank, world):
    """Seeded build keys and batches of one rank."""
    dist_name, n_build, n_batch, n_steps, pct, mode = case
    keys = O.gen_keys(dist_name, 100 + rank, n_build)
    if rank == 1 and n_build > 10:
        keys[:5] = O.gen_keys(dist_name, 100, n_build)[:5]  # keys built on two ranks: later rank wins
    vals = O.value_of(keys) ^ np.uint64(rank)
    steps = []
    for i in range(n_steps):
        nb = 0 if (rank == world - 1 and i == 1) else n_batch  # one empty batch
        k, v, o = O.gen_requests(dist_name, 1000 * i + rank, keys, nb, pct)
        if mode == MODE_SORTED and rank > 0 and nb:
            # a tenth of the batch re-inserts keys that rank 0 touches in the
            # same step: the owner must order them by source rank
            k0, _, _ = O.gen_requests(dist_name, 1000 * i, O.gen_keys(dist_name, 100, n_build), n_batch, pct)
            m = min(nb, k0.size) // 10
            k[:m] = k0[:m]
            o[:m] = 0
            v[:m] = np.arange(m, dtype=np.uint64) + np.uint64(10_000 * rank)
        if mode == MODE_STM and nb:
            _, first = np.unique(k, return_index=True)
            sel = np.sort(first)
            k, v, o = k[sel], v[sel], o[sel]
        steps.append((k, v, o))
    return keys, vals, steps


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, case, out_dir, max_batch):
    import torch.distributed as dist

    from eirene_b200.shard import ShardedBTree

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    import datetime

    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        mode = case[5]
        keys, vals, steps = rank_inputs(case, rank, world)
        st = ShardedBTree(OracleShardOps(max_batch), sample_per_rank=256)
        st.bulk_build(torch.from_numpy(keys.view(np.int64)), torch.from_numpy(vals.view(np.int64)))
        outs = {}
        for i, (k, v, o) in enumerate(steps):
            ov = torch.zeros(k.size, dtype=torch.int64)
            os_ = torch.zeros(k.size, dtype=torch.uint8)
            st.execute(torch.from_numpy(k.view(np.int64)), torch.from_numpy(v.view(np.int64)),
                       torch.from_numpy(o.astype(np.uint8)), ov, os_, mode=mode)
            outs[f"v{i}"] = ov.numpy().view(np.uint64)
            outs[f"s{i}"] = os_.numpy()
        dk, dv = st.dump_local()
        lo, hi = st.owner_range()
        np.savez(os.path.join(out_dir, f"rank{rank}.npz"), dk=dk.numpy().view(np.uint64),
                 dv=dv.numpy().view(np.uint64), lo=np.uint64(lo), hi=np.uint64(hi if hi is not None else 0),
                 last=hi is None, size=st.size(), spl=st.splitters_host, **outs)
    finally:
        dist.destroy_process_group()


CASES = {
    "uniform_sorted_w2": (("uniform", 20_000, 6_000, 3, 80, MODE_SORTED), 2, 4096),
    "zipf_sorted_w3_chunked": (("zipf", 30_000, 5_000, 3, 50, MODE_SORTED), 3, 1500),
    "gamma_stm_w2": (("gamma", 20_000, 4_000, 2, 70, MODE_STM), 2, 8192),
    "tiny_w3": (("uniform", 7, 20, 3, 50, MODE_SORTED), 3, 8),
}


@pytest.mark.parametrize("name", list(CASES))
def test_sharded_equals_one_tree(name, tmp_path):
    case, world, max_batch = CASES[name]
    mp.start_processes(_rank_main, args=(world, _free_port(), case, str(tmp_path), max_batch), nprocs=world,
                       join=True, start_method="spawn")
    res = [dict(np.load(tmp_path / f"rank{r}.npz")) for r in range(world)]
    inputs = [rank_inputs(case, r, world) for r in range(world)]
    mode = case[5]
    one = O.OracleTree()
    one.bulk_build(np.concatenate([inp[0] for inp in inputs]), np.concatenate([inp[1] for inp in inputs]))
    for i in range(case[3]):
        ks = [inp[2][i] for inp in inputs]
        cat = [np.concatenate([x[j] for x in ks]) for j in range(3)]
        if mode == MODE_STM:
            ev, es = one.execute_serial(*cat)
        else:
            ev, es = one.execute_merged(*cat)
        off = 0
        for r in range(world):
            n = ks[r][0].size
            assert (res[r][f"s{i}"] == es[off:off + n]).all(), (name, i, r)
            assert (res[r][f"v{i}"] == ev[off:off + n]).all(), (name, i, r)
            off += n
    ok, ov = one.dump()
    gk = np.concatenate([r["dk"] for r in res])
    gv = np.concatenate([r["dv"] for r in res])
    assert (gk == ok).all() and (gv == ov).all()
    for r in res:
        assert int(r["size"]) == ok.size
        if r["dk"].size:
            assert r["dk"][0] >= r["lo"]
            if not r["last"]:
                assert r["dk"][-1] < r["hi"]


def test_pick_splitters():
    assert pick_splitters(np.zeros(0, np.uint64), 1).size == 0
    e = pick_splitters(np.full(5, 2**64 - 1, np.uint64), 4)
    assert e.size == 3 and (np.diff(e.astype(object)) > 0).all()
    s = np.arange(1000, dtype=np.uint64) * np.uint64(3) + np.uint64(2**63)  # above 2^63: uint64 order
    spl = pick_splitters(s[::-1], 4)
    assert spl.tolist() == [int(s[250]), int(s[500]), int(s[750])]
    d = pick_splitters(np.array([5, 5, 5], np.uint64), 4)
    assert d.size == 3 and (np.diff(d.astype(np.int64)) >= 0).all()
