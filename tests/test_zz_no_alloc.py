"""bt_bulk_build_static: the bulk build for callers that must not allocate GPU
memory while loading a tree (device memory reserved up front by another
allocator, or latency-critical threads where cudaFree would synchronise the
whole device).  Its scratch is a fixed array inside the library, so the call
must give exactly what the allocating bt_bulk_build gives, call after call,
even though the array keeps the previous call's contents.

This file is named so that pytest collects it last."""
import ctypes

import numpy as np
import pytest

import eirene_b200 as E
from oracle import oracle as O
from tests.helpers import dev, dump

pytestmark = pytest.mark.gpu


def static_build(tree, keys_t, vals_t, n):
    return E.lib().bt_bulk_build_static(tree._h, keys_t.data_ptr(), vals_t.data_ptr(), n, None)


def test_static_build_matches_allocating_build_twice(gpu):
    import torch

    ref = E.BTree(max_keys=1 << 18, max_batch=1 << 12)
    sta = E.BTree(max_keys=1 << 18, max_batch=1 << 12)
    # two calls in a row; the second is smaller and has repeated keys, so any
    # scratch left over from the first call would show in the result
    cases = [(E.STATIC_BUILD_MAX_KEYS, 3), (40_009, 4)]
    for n, seed in cases:
        keys = O.gen_keys("uniform", seed, n)
        if seed == 4:
            keys[::7] = keys[1::7][: keys[::7].size]  # repeated keys: last value wins
        vals = np.arange(n, dtype=np.uint64) * np.uint64(3) + np.uint64(seed)
        kt, vt = dev(keys), dev(vals)
        ref.bulk_build(kt, vt)
        rc = static_build(sta, kt, vt, n)
        torch.cuda.synchronize()
        assert rc == E.BT_OK, E.lib().bt_status_string(rc)
        rk, rv = dump(ref)
        sk, sv = dump(sta)
        assert sk.size == rk.size and (sk == rk).all() and (sv == rv).all()
        assert sta.size() == ref.size()
        assert (sta.leaf_sizes() == ref.leaf_sizes()).all()
        assert (sta.level_counts() == ref.level_counts()).all()


def test_static_build_rejects_more_than_the_limit(gpu):
    t = E.BTree(max_keys=1 << 18, max_batch=1 << 12)
    n = E.STATIC_BUILD_MAX_KEYS + 1
    keys = np.arange(n, dtype=np.uint64)
    kt = dev(keys)
    assert static_build(t, kt, kt, n) == -8
    # the handle still works afterwards
    assert static_build(t, kt, kt, 1000) == E.BT_OK
    assert t.size() == 1000


def test_static_build_edge_calls(gpu):
    # an empty build, a build on a non-default stream, and a build straight
    # after a batch whose deferred leaf/inner merge may still be running:
    # each gives what the allocating bt_bulk_build gives
    import torch

    ref = E.BTree(max_keys=1 << 18, max_batch=1 << 15)
    sta = E.BTree(max_keys=1 << 18, max_batch=1 << 15)
    keys = O.gen_keys("uniform", 5, 30_000)
    vals = O.value_of(keys)
    kt, vt = dev(keys), dev(vals)
    for t in (ref, sta):
        t.bulk_build(kt, vt)
    # empty build
    ref.bulk_build(kt[:0], vt[:0])
    assert E.lib().bt_bulk_build_static(sta._h, kt.data_ptr(), vt.data_ptr(), 0, None) == E.BT_OK
    assert sta.size() == 0 == ref.size()
    # on a side stream
    side = torch.cuda.Stream()
    ref.bulk_build(kt, vt)
    rc = E.lib().bt_bulk_build_static(sta._h, kt.data_ptr(), vt.data_ptr(), keys.size, side.cuda_stream)
    side.synchronize()
    assert rc == E.BT_OK
    rk, rv = dump(ref)
    sk, sv = dump(sta)
    assert (sk == rk).all() and (sv == rv).all()
    # right after a batch with the deferred write phase on (the default)
    qk, qv, qo = O.gen_requests("uniform", 6, keys, 20_000, 0)
    q = (dev(qk), dev(qv), dev(qo))
    for t in (ref, sta):
        t.set_option(E.OPT_ASYNC_WRITE, 1)
        ov = torch.empty(qk.size, dtype=torch.int64, device="cuda")
        os_ = torch.empty(qk.size, dtype=torch.uint8, device="cuda")
        t.execute(*q, ov, os_, mode=E.MODE_SORTED | E.MODE_MERGE_ENGINE)
    k2 = O.gen_keys("uniform", 7, 25_000)
    v2 = O.value_of(k2)
    k2t, v2t = dev(k2), dev(v2)
    ref.bulk_build(k2t, v2t)
    assert static_build(sta, k2t, v2t, k2.size) == E.BT_OK
    torch.cuda.synchronize()
    rk, rv = dump(ref)
    sk, sv = dump(sta)
    assert (sk == rk).all() and (sv == rv).all()
    assert (sta.leaf_sizes() == ref.leaf_sizes()).all()
