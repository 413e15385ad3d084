"""Lookups that compare the separators' 32-bit prefixes first: keys whose
high halves collide (every comparison of such a key falls back to the full
keys) and mixes of colliding and spread keys, after a bulk build, after
merge-engine batches (which keep the prefixes) and after STM batches (after
which the prefixes are rebuilt from the rows), against the oracle."""
import numpy as np
import pytest

import eirene_b200 as E
from oracle import oracle as O
from tests.helpers import dev, empty_u64, empty_u8, host_u64, host_u8, run_batch

pytestmark = pytest.mark.gpu
MERGE = E.MODE_SORTED | E.MODE_MERGE_ENGINE


def colliding_keys(seed, n, n_prefixes):
    rng = np.random.default_rng(seed)
    hi = rng.integers(0, 2**32 - 1, n_prefixes, dtype=np.uint64)
    k = (hi[rng.integers(0, n_prefixes, n)] << np.uint64(32)) | rng.integers(0, 2**32, n, dtype=np.uint64)
    return np.unique(k)


def lookups_match(t, o, q):
    import torch

    ov, os_ = empty_u64(q.size), empty_u8(q.size)
    t.search(dev(q), ov, os_)
    torch.cuda.synchronize()
    gv, gs = host_u64(ov), host_u8(os_)
    rv, rs = o.execute_merged(q, np.zeros(q.size, np.uint64), np.ones(q.size, np.uint8))
    assert (gs == rs).all() and (gv == rv).all()


@pytest.mark.parametrize("n_prefixes", [1, 3, 1000])
def test_prefix_collisions(gpu, n_prefixes):
    rng = np.random.default_rng(n_prefixes)
    keys = colliding_keys(10 + n_prefixes, 150_000, n_prefixes)
    spread = O.gen_keys("uniform", 20 + n_prefixes, 50_000)
    keys = np.union1d(keys, spread)
    vals = O.value_of(keys)
    t = E.BTree(max_keys=1 << 21, max_batch=1 << 18)
    t.bulk_build(dev(keys), dev(vals))
    o = O.OracleTree()
    o.bulk_build(keys, vals)
    probe = np.concatenate([rng.choice(keys, 40_000), colliding_keys(30 + n_prefixes, 20_000, n_prefixes),
                            O.gen_keys("uniform", 40 + n_prefixes, 10_000)])
    lookups_match(t, o, probe)
    # merge-engine batches split leaves and inner nodes (prefixes kept in place)
    for b in range(3):
        new = colliding_keys(50 + 10 * b + n_prefixes, 60_000, n_prefixes)
        rk = np.concatenate([new, rng.choice(keys, 20_000)])
        rv = rk ^ np.uint64(b + 1)
        ro = np.concatenate([np.zeros(new.size, np.uint8), np.ones(20_000, np.uint8)])
        ov, os_ = o.execute_merged(rk, rv, ro, engine=O.ENGINE_MERGE)
        gv, gs = run_batch(t, rk, rv, ro, MERGE)
        assert (gs == os_).all() and (gv == ov).all(), b
        lookups_match(t, o, np.concatenate([probe, new[::7]]))
    # an STM batch of distinct fresh keys (prefixes rebuilt before the next lookups)
    fresh = np.setdiff1d(colliding_keys(99 + n_prefixes, 30_000, n_prefixes), o.dump()[0])
    sv_, ss_ = o.execute_serial(fresh, fresh, np.zeros(fresh.size, np.uint8))
    gv, gs = run_batch(t, fresh, fresh, np.zeros(fresh.size, np.uint8), E.MODE_STM)
    assert (gs == ss_).all()
    lookups_match(t, o, np.concatenate([probe, fresh[::5]]))
