"""Shared helpers for the GPU parity tests (numpy <-> torch CUDA tensors)."""
import numpy as np


def dev(a: np.ndarray):
    import torch

    a = np.ascontiguousarray(a)
    if a.dtype == np.uint64:
        return torch.from_numpy(a.view(np.int64)).cuda()
    return torch.from_numpy(a).cuda()


def empty_u64(n: int):
    import torch

    return torch.zeros(max(n, 1), dtype=torch.int64, device="cuda")[:n]


def empty_u8(n: int):
    import torch

    return torch.zeros(max(n, 1), dtype=torch.uint8, device="cuda")[:n]


def host_u64(t) -> np.ndarray:
    return t.cpu().numpy().view(np.uint64)


def host_u8(t) -> np.ndarray:
    return t.cpu().numpy().astype(np.uint8)


def run_batch(tree, keys, vals, ops, mode):
    k, v, o = dev(keys), dev(vals), dev(ops.astype(np.uint8))
    ov, os_ = empty_u64(keys.size), empty_u8(keys.size)
    tree.execute(k, v, o, ov, os_, mode=mode)
    import torch

    torch.cuda.synchronize()
    return host_u64(ov), host_u8(os_)


def dump(tree):
    k, v = tree.dump()
    return host_u64(k), host_u64(v)
