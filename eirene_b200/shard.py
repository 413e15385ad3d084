"""Key-range-sharded tree over the ranks of a process group (one GPU per rank).

Each rank holds one tree.  Shard s owns the keys in [splitter[s-1],
splitter[s]); the splitters are equal-count quantiles of a sample of every
rank's build keys.  A batch submitted on any rank takes one exchange step:

  1. route: stable partition of the batch by owning shard on the GPU
     (bt_route_batch), with the per-shard run lengths;
  2. all-to-all of the run lengths, then of keys, values and op codes
     (NCCL over NVLink/NVSwitch for the GPU path);
  3. the owner runs everything it received as one batch, in source-rank
     order (in pieces of max_batch when more arrives than that);
  4. reverse all-to-all of answers and statuses, scattered back to input
     order (bt_unroute_results).

Because every request for a key goes to the same owner and keeps its input
order there, the answers and the final contents equal those of ONE tree that
runs the concatenation of all ranks' batches in rank order (for both batch
meanings: per key, the sorted-merge meaning depends only on that key's
requests in order, and the STM meaning on distinct keys is order free).  The
reference is single-GPU only (one GPU_STM_Tree, src/gpu-stm-tree-v39/
bpt-gpustm.cpp:14-28): this layer has no counterpart there.

The per-rank work (route, local batch, unroute, buffers) is behind a small
ops object, `DeviceShardOps` on the GPU, and the collectives behind a comm
object, `DistComm` (torch.distributed: NCCL between GPUs, gloo on CPU
tensors); the exchange logic between them is the same for both.
"""
from __future__ import annotations

import numpy as np
import torch
import torch.distributed as dist

from . import MAX_SHARDS, MODE_SORTED, BTree

KEY_MAX_U64 = np.uint64(0xFFFFFFFFFFFFFFFF)


def pick_splitters(sample: np.ndarray, n_shards: int) -> np.ndarray:
    """n_shards - 1 non-decreasing splitters (uint64) at equal-count quantiles
    of the distinct keys in `sample`; an empty sample splits the key space
    into equal-width ranges.  Equal neighbours leave a shard with no keys."""
    u = np.unique(np.asarray(sample, dtype=np.uint64))
    u = u[u != KEY_MAX_U64]
    if n_shards <= 1:
        return np.zeros(0, np.uint64)
    if u.size == 0:
        step = (1 << 64) // n_shards
        return np.array([s * step for s in range(1, n_shards)], dtype=np.uint64)
    idx = (np.arange(1, n_shards, dtype=np.int64) * u.size) // n_shards
    return u[idx]


class DeviceShardOps:
    """This rank's tree and routing kernels on its GPU (the library path)."""

    def __init__(self, tree: BTree):
        self.tree = tree
        self.device = torch.device("cuda", tree.device)
        self.max_batch = tree.max_batch

    def _s(self):
        return torch.cuda.current_stream(self.device)

    def empty(self, n: int, dtype) -> torch.Tensor:
        return torch.empty(max(n, 1), dtype=dtype, device=self.device)[:n]

    def from_numpy(self, a: np.ndarray) -> torch.Tensor:
        a = np.ascontiguousarray(a)
        if a.dtype == np.uint64:
            a = a.view(np.int64)
        return torch.from_numpy(a).to(self.device)

    def route(self, splitters, n_shards, keys, vals, ops):
        n = keys.numel()
        rk = self.empty(n, torch.int64)
        rv = self.empty(n, torch.int64) if vals is not None else None
        ro = self.empty(n, torch.uint8) if ops is not None else None
        perm = self.empty(n, torch.int32)
        counts = self.empty(n_shards, torch.int64)
        self.tree.route(splitters if splitters.numel() else None, n_shards, keys, vals, ops, rk, rv, ro, perm,
                        counts, stream=self._s())
        return rk, rv, ro, perm, counts

    def unroute(self, perm, in_vals, in_status, out_vals, out_status):
        self.tree.unroute(perm, in_vals, in_status, out_vals, out_status, stream=self._s())

    def bulk_build(self, keys, vals):
        self.tree.bulk_build(keys, vals, stream=self._s())

    def execute(self, keys, vals, ops, out_vals, out_status, mode):
        self.tree.execute(keys, vals, ops, out_vals, out_status, mode=mode, stream=self._s())

    def size(self) -> int:
        return self.tree.size()

    def dump(self):
        return self.tree.dump()


class DistComm:
    """The exchange over torch.distributed (NCCL between GPUs, gloo on CPU)."""

    def __init__(self, group=None):
        self.group = group
        init = dist.is_available() and dist.is_initialized()
        self.rank = dist.get_rank(group) if init else 0
        self.world = dist.get_world_size(group) if init else 1

    def all_to_all_single(self, out, inp, out_splits=None, in_splits=None):
        dist.all_to_all_single(out, inp, out_splits, in_splits, group=self.group)

    def all_gather(self, parts, t):
        dist.all_gather(parts, t, group=self.group)

    def all_reduce_sum(self, t):
        dist.all_reduce(t, group=self.group)


class ShardedBTree:
    """One logical tree, key-range-partitioned over the ranks of `group`."""

    def __init__(self, ops, group=None, sample_per_rank: int = 4096, comm=None):
        self.ops = ops
        self.comm = comm if comm is not None else DistComm(group)
        self.rank = self.comm.rank
        self.world = self.comm.world
        if self.world > MAX_SHARDS:
            raise ValueError(f"at most {MAX_SHARDS} shards")
        self.sample_per_rank = sample_per_rank
        self.splitters = None  # on the ops device, world - 1 keys (int64 bit patterns)
        self.splitters_host = np.zeros(0, np.uint64)

    @classmethod
    def on_gpu(cls, group=None, sample_per_rank: int = 4096, comm=None, **tree_kw) -> "ShardedBTree":
        return cls(DeviceShardOps(BTree(**tree_kw)), group=group, sample_per_rank=sample_per_rank, comm=comm)

    # ---- exchange helpers (every rank calls these in the same order) ----
    def _counts(self, counts: torch.Tensor):
        if self.world == 1:
            c = counts.cpu().tolist()
            return c, c
        recv = torch.empty_like(counts)
        self.comm.all_to_all_single(recv, counts)
        both = torch.stack([counts, recv]).cpu()
        return both[0].tolist(), both[1].tolist()

    def _a2a(self, send: torch.Tensor, send_counts, recv_counts) -> torch.Tensor:
        if self.world == 1:
            return send
        recv = self.ops.empty(int(sum(recv_counts)), send.dtype)
        self.comm.all_to_all_single(recv, send, recv_counts, send_counts)
        return recv

    def owner_range(self, shard: int | None = None):
        """[lo, hi) of the keys shard `shard` (default: this rank) owns; hi is
        None for the last shard (up to the largest key)."""
        s = self.rank if shard is None else shard
        lo = 0 if s == 0 else int(self.splitters_host[s - 1])
        hi = None if s == self.world - 1 else int(self.splitters_host[s])
        return lo, hi

    # ---- tree operations ----
    def bulk_build(self, keys: torch.Tensor, vals: torch.Tensor):
        """Build the global tree from every rank's (keys, vals); a key given
        more than once keeps the value that comes last in rank order."""
        n = keys.numel()
        k = min(n, self.sample_per_rank)
        samp = np.full(self.sample_per_rank, KEY_MAX_U64, np.uint64)
        if k:
            idx = (np.arange(k, dtype=np.int64) * n) // k
            samp[:k] = keys[torch.from_numpy(idx).to(keys.device)].cpu().numpy().view(np.uint64)
        st = torch.from_numpy(samp.view(np.int64)).to(keys.device)
        if self.world > 1:
            parts = [torch.empty_like(st) for _ in range(self.world)]
            self.comm.all_gather(parts, st)
            allsamp = torch.cat(parts).cpu().numpy().view(np.uint64)
        else:
            allsamp = samp
        self.splitters_host = pick_splitters(allsamp, self.world)
        self.splitters = self.ops.from_numpy(self.splitters_host)
        if self.world == 1:
            self.ops.bulk_build(keys, vals)
            return
        rk, rv, _, _, counts = self.ops.route(self.splitters, self.world, keys, vals, None)
        cs, cr = self._counts(counts)
        self.ops.bulk_build(self._a2a(rk, cs, cr), self._a2a(rv, cs, cr))

    def execute(self, keys, vals, ops, out_vals, out_status, mode: int = MODE_SORTED):
        """Run this rank's batch against the global tree (collective: every
        rank of the group calls it, with its own batch, possibly empty)."""
        if self.splitters is None:
            raise RuntimeError("bulk_build first: the splitters come from the build keys")
        if self.world == 1:
            self._local(keys, vals, ops, out_vals, out_status, mode)
            return
        rk, rv, ro, perm, counts = self.ops.route(self.splitters, self.world, keys, vals, ops)
        cs, cr = self._counts(counts)
        qk, qv, qo = self._a2a(rk, cs, cr), self._a2a(rv, cs, cr), self._a2a(ro, cs, cr)
        m = qk.numel()
        av, ast = self.ops.empty(m, torch.int64), self.ops.empty(m, torch.uint8)
        self._local(qk, qv, qo, av, ast, mode)
        bv, bs = self._a2a(av, cr, cs), self._a2a(ast, cr, cs)
        self.ops.unroute(perm, bv, bs, out_vals, out_status)

    def _local(self, keys, vals, ops, out_vals, out_status, mode):
        m, b = keys.numel(), self.ops.max_batch
        for c0 in range(0, m, b):
            c1 = min(m, c0 + b)
            self.ops.execute(keys[c0:c1], vals[c0:c1], ops[c0:c1], out_vals[c0:c1], out_status[c0:c1], mode)

    def local_size(self) -> int:
        return self.ops.size()

    def size(self) -> int:
        """Keys in the global tree (collective)."""
        t = torch.tensor([self.local_size()], dtype=torch.int64, device=self.ops.empty(0, torch.int64).device)
        if self.world > 1:
            self.comm.all_reduce_sum(t)
        return int(t.item())

    def dump_local(self):
        """This shard's (keys, values) in key order; the global sorted contents
        are the shards' dumps concatenated in rank order."""
        return self.ops.dump()
