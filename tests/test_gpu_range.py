"""Range scan (bt_range_batch): every query [lo, hi] must return exactly the
oracle's keys in that closed range, in ascending order, with their values,
its full count, and the first max_per of them when it is truncated."""
import numpy as np
import pytest

import eirene_b200 as E
from oracle import oracle as O
from tests.helpers import dev, run_batch

pytestmark = pytest.mark.gpu

U64MAX = np.uint64(2**64 - 1)


@pytest.mark.parametrize("dist,fills", [("uniform", (24, 24)), ("zipf", (16, 16)), ("gamma", (31, 31))])
def test_range_matches_oracle(gpu, dist, fills):
    import torch

    keys = O.gen_keys(dist, 61, 150_000)
    vals = O.value_of(keys)
    t = E.BTree(max_keys=1 << 20, max_batch=1 << 17, leaf_fill=fills[0], inner_fill=fills[1])
    t.bulk_build(dev(keys), dev(vals))
    o = O.OracleTree(*fills)
    o.bulk_build(keys, vals)
    rk, rv, ro = O.gen_requests(dist, 62, keys, 60_000, 50)  # inserts split leaves before the scans
    o.execute_merged(rk, rv, ro)
    run_batch(t, rk, rv, ro, E.MODE_SORTED | E.MODE_MERGE_ENGINE)
    ok, ov = o.dump()
    rng = np.random.default_rng(63)
    n_q = 3000
    a = ok[rng.integers(0, ok.size, n_q)]
    span = rng.integers(0, 400, n_q)
    b = ok[np.minimum(np.searchsorted(ok, a) + span, ok.size - 1)]
    lo, hi = a.copy(), b.copy()
    lo[::7] -= np.uint64(1)                      # bounds between keys
    hi[::5] += np.uint64(1)
    lo[:4] = [0, 0, 5, ok[-1]]
    hi[:4] = [U64MAX, 0, 4, U64MAX]              # everything, nothing, lo > hi, the last key
    lo[4], hi[4] = U64MAX, U64MAX                # the reserved key: empty
    max_per = 128
    counts, gk, gv = t.range(dev(lo), dev(hi), max_per)
    torch.cuda.synchronize()
    counts = counts.cpu().numpy()
    gk = gk.cpu().numpy().view(np.uint64)
    gv = gv.cpu().numpy().view(np.uint64)
    s = np.searchsorted(ok, lo, side="left")
    e = np.searchsorted(ok, hi, side="right")
    want = np.where(lo <= hi, e - s, 0)
    want[4] = 0
    assert (counts == want).all()
    assert counts[0] == ok.size
    for i in range(n_q):
        m = min(int(want[i]), max_per)
        assert (gk[i, :m] == ok[s[i]:s[i] + m]).all(), i
        assert (gv[i, :m] == ov[s[i]:s[i] + m]).all(), i
    assert (counts > max_per).any() and (counts == 0).any()
