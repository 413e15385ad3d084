"""Learned leaf predictor on the GPU: gradient check of the training kernels
against the CPU oracle, bit-exact lookups versus plain descent (and the
oracle), behaviour after splits, and what the trained MLP root gains over a
linear root."""
import numpy as np
import pytest

import eirene_b200 as E
from oracle import oracle as O
from tests.helpers import dev, dump, empty_u64, empty_u8, host_u64, host_u8, run_batch

pytestmark = pytest.mark.gpu

# float32 accumulation over n samples vs a double CPU reference
GRAD_RTOL = 2e-3
GRAD_ATOL = 1e-6


def test_mlp_gradient_matches_oracle(gpu):
    import torch

    t = E.BTree(max_keys=1 << 14, max_batch=1 << 12)
    rng = np.random.default_rng(1)
    for n in [1, 97, 5000, 65536]:
        p = rng.normal(0, 0.7, 97).astype(np.float32)
        x = rng.random(n).astype(np.float32)
        y = rng.random(n).astype(np.float32)
        g = torch.zeros(97, dtype=torch.float32, device="cuda")
        loss = torch.zeros(1, dtype=torch.float32, device="cuda")
        t.mlp_grad(torch.from_numpy(p).cuda(), torch.from_numpy(x).cuda(), torch.from_numpy(y).cuda(), g, loss)
        torch.cuda.synchronize()
        ref_loss, ref_g = O.mlp_grad(p, x, y)
        gg = g.cpu().numpy().astype(np.float64)
        scale = np.abs(ref_g).max()
        assert np.allclose(gg, ref_g, rtol=GRAD_RTOL, atol=GRAD_ATOL + GRAD_RTOL * scale), (n, np.abs(gg - ref_g).max())
        assert abs(float(loss.item()) - ref_loss) <= GRAD_RTOL * max(1.0, ref_loss)


def lookups(t, keys):
    v, s = empty_u64(keys.size), empty_u8(keys.size)
    t.search(dev(keys), v, s)
    return host_u64(v), host_u8(s)


@pytest.mark.parametrize("dist", ["uniform", "normal", "gamma", "zipf"])
def test_learned_lookup_bit_exact(gpu, dist):
    keys = O.gen_keys(dist, 3, 300_000)
    vals = O.value_of(keys)
    t = E.BTree(max_keys=1 << 20, max_batch=1 << 18)
    t.bulk_build(dev(keys), dev(vals))
    o = O.OracleTree()
    o.bulk_build(keys, vals)
    qk, _, _ = O.gen_requests(dist, 4, keys, 200_000, 100)
    qk[5] = np.uint64(2**64 - 1)
    qk[6] = np.uint64(0)
    ov, os_ = o.execute_merged(qk, np.zeros_like(qk), np.ones(qk.size, np.uint8))
    t.set_descent(False)
    pv, ps = lookups(t, qk)
    t.retrain()
    info = t.learned_info()
    assert info["valid"] == 1
    t.set_descent(True)
    t.reset_stats()
    lv, ls = lookups(t, qk)
    assert (ps == os_).all() and (pv == ov).all()
    assert (ls == ps).all() and (lv == pv).all()
    st = t.stats()
    assert st["learned_hits"] > 0.5 * qk.size, (st, info)


def test_learned_after_splits_and_sorted_batches(gpu):
    keys = O.gen_keys("uniform", 8, 200_000)
    vals = O.value_of(keys)
    t = E.BTree(max_keys=1 << 21, max_batch=1 << 18)
    t.bulk_build(dev(keys), dev(vals))
    o = O.OracleTree()
    o.bulk_build(keys, vals)
    t.retrain()
    t.set_descent(True)
    # insert-heavy batches split many leaves after training: lookups must stay exact
    for b in range(4):
        rk, rv, ro = O.gen_requests("uniform", 50 + b, keys, 100_000, 50)
        ov, os_ = o.execute_merged(rk, rv, ro)
        gv, gs = run_batch(t, rk, rv, ro, E.MODE_SORTED)
        assert (gs == os_).all() and (gv == ov).all()
    st = t.stats()
    assert st["leaf_splits"] > 0 and st["learned_fallbacks"] > 0 and st["learned_hits"] > 0
    qk, _, _ = O.gen_requests("uniform", 99, o.dump()[0], 100_000, 100)
    ov, os_ = o.execute_merged(qk, np.zeros_like(qk), np.ones(qk.size, np.uint8))
    lv, ls = lookups(t, qk)
    assert (ls == os_).all() and (lv == ov).all()
    # retraining restores the hit rate
    t.reset_stats()
    t.retrain()
    lookups(t, qk)
    st2 = t.stats()
    assert st2["learned_fallbacks"] < st["learned_fallbacks"]


def test_trained_mlp_root_beats_linear_root(gpu):
    # skewed keys and few segments: a linear root cuts the key range into
    # equal-width segments, so the dense part of the distribution falls into a
    # few segments whose lines span long curved stretches of the CDF; their
    # errors exceed the window and lookups miss the probe and fall back.  The
    # trained MLP root follows the CDF and gives every segment the same share
    # of leaves.
    keys = O.gen_keys("gamma", 11, 400_000)
    vals = O.value_of(keys)
    qk, _, _ = O.gen_requests("gamma", 12, keys, 200_000, 100)
    res = {}
    for mlp in (False, True):
        t = E.BTree(max_keys=1 << 21, max_batch=1 << 18, n_segments=64, window=16)
        t.bulk_build(dev(keys), dev(vals))
        t.set_root_model(mlp)
        t.retrain()
        t.set_descent(True)
        t.reset_stats()
        lv, ls = lookups(t, qk)
        st = t.stats()
        info = t.learned_info()
        res[mlp] = (st["learned_fallbacks"] / qk.size, st["learned_probe_sum"] / max(1, st["learned_hits"]),
                    info["segments_over_window"], info["loss"])
        t.set_descent(False)
        pv, ps = lookups(t, qk)
        assert (lv == pv).all() and (ls == ps).all()
        t.close()
    lin, mlp = res[False], res[True]
    assert mlp[0] < lin[0], res
    assert mlp[2] <= lin[2], res


def test_autotune_then_batches_stay_exact(gpu):
    keys = O.gen_keys("uniform", 21, 300_000)
    vals = O.value_of(keys)
    t = E.BTree(max_keys=1 << 21, max_batch=1 << 18)
    t.bulk_build(dev(keys), dev(vals))
    o = O.OracleTree()
    o.bulk_build(keys, vals)
    t.retrain()
    t.set_descent(True)
    rk, rv, ro = O.gen_requests("uniform", 22, keys, 100_000, 95)
    rep = t.autotune(dev(rk))
    assert rep["plain_lanes"] in (4, 8, 16, 32) and rep["learned_lanes"] in (2, 4) and rep["learned_mode"] in (1, 2, 3)
    assert rep["sort_threads"] in (256, 512, 1024) and rep["sort_threads_touched"] in (256, 512, 1024)
    assert all(v > 0 for v in rep["plain_ms"].values())
    for desc in (0, 1, -1):
        t.set_option(E.OPT_BATCH_DESCENT, desc)
        for lv in (0, 1):
            t.set_option(E.OPT_SORTED_LEAF_VALS, lv)
            rk, rv, ro = O.gen_requests("uniform", 30 + desc * 2 + lv, keys, 50_000, 95)
            ov, os_ = o.execute_merged(rk, rv, ro)
            gv, gs = run_batch(t, rk, rv, ro, E.MODE_SORTED)
            assert (gs == os_).all() and (gv == ov).all()


def test_learned_in_stm_mode_and_serving(gpu):
    # the learned model proposes leaves in the STM fast path; answers and
    # contents must equal the serial oracle
    keys = O.gen_keys("uniform", 31, 200_000)
    vals = O.value_of(keys)
    t = E.BTree(max_keys=1 << 21, max_batch=1 << 17)
    t.bulk_build(dev(keys), dev(vals))
    o = O.OracleTree()
    o.bulk_build(keys, vals)
    t.retrain()
    t.set_descent(True)
    rk, rv, ro = O.gen_requests("uniform", 32, keys, 60_000, 70)
    _, first = np.unique(rk, return_index=True)
    sel = np.sort(first)
    rk, rv, ro = rk[sel], rv[sel], ro[sel]
    ov, os_ = o.execute_serial(rk, rv, ro)
    gv, gs = run_batch(t, rk, rv, ro, E.MODE_STM)
    assert (gs == os_).all() and (gv == ov).all()
    srv = E.Server(t)
    qk, qv, qo = O.gen_requests("uniform", 33, keys, 30_000, 90)
    _, first = np.unique(qk, return_index=True)
    sel = np.sort(first)
    qk, qv, qo = qk[sel], qv[sel], qo[sel]
    ov2, os2 = o.execute_serial(qk, qv, qo)
    out_v = np.zeros(qk.size, np.uint64)
    out_s = np.zeros(qk.size, np.uint8)
    srv.wait(srv.submit(qk, qv, qo, out_v, out_s))
    srv.stop()
    assert (out_s == os2).all() and (out_v == ov2).all()
    gk, gvv = dump(t)
    ok, ovv = o.dump()
    assert (gk == ok).all() and (gvv == ovv).all()


@pytest.mark.parametrize("lanes,mode", [(2, 3), (2, 1), (4, 3), (8, 3), (16, 3), (4, 2), (4, 1), (8, 2), (8, 1),
                                        (16, 1), (32, 1)])
def test_learned_lookup_shapes_bit_exact(gpu, lanes, mode):
    # every lane-group shape of the unsorted learned lookup against the plain
    # descent and the oracle: present, absent, reserved and extreme keys, and a
    # search larger than the miss list (it runs in pieces)
    keys = O.gen_keys("normal", 41, 120_000)
    vals = O.value_of(keys)
    t = E.BTree(max_keys=1 << 19, max_batch=1 << 12)
    t.bulk_build(dev(keys), dev(vals))
    o = O.OracleTree()
    o.bulk_build(keys, vals)
    qk, _, _ = O.gen_requests("normal", 42, keys, 150_000, 100)
    qk[:4] = np.array([0, 1, 2**64 - 1, 2**64 - 2], np.uint64)
    qk[4] = keys.min()
    qk[5] = keys.max()
    ov, os_ = o.execute_merged(qk, np.zeros_like(qk), np.ones(qk.size, np.uint8))
    t.retrain()
    t.set_descent(True)
    t.set_learned_group(lanes)
    t.set_option(E.OPT_LEARNED_MODE, mode)
    t.reset_stats()
    lv, ls = lookups(t, qk)
    assert (ls == os_).all() and (lv == ov).all()
    st = t.stats()
    assert st["learned_hits"] + st["learned_fallbacks"] == qk.size - 1  # the reserved key is neither
    assert st["learned_hits"] > 0.8 * qk.size, st


def test_refit_follows_splits_and_deletes(gpu):
    # after insert batches split leaves and delete batches empty some, a refit
    # (stage 1 kept) restores the hit rate; answers stay exact throughout
    keys = O.gen_keys("uniform", 51, 200_000)
    vals = O.value_of(keys)
    t = E.BTree(max_keys=1 << 21, max_batch=1 << 17)
    t.bulk_build(dev(keys), dev(vals))
    o = O.OracleTree()
    o.bulk_build(keys, vals)
    with pytest.raises(E.BTError):
        t.refit()
    t.retrain()
    t.set_descent(True)
    for b in range(3):
        rk, rv, ro = O.gen_requests("uniform", 60 + b, keys, 80_000, 50)
        ov, os_ = o.execute_merged(rk, rv, ro)
        gv, gs = run_batch(t, rk, rv, ro, E.MODE_SORTED | E.MODE_MERGE_ENGINE)
        assert (gs == os_).all() and (gv == ov).all()
    # delete a contiguous run of keys: whole leaves empty and keep routing
    cur = o.dump()[0]
    dk = cur[1000:3000]
    ops = np.full(dk.size, E.OP_DELETE, np.uint8)
    ov, os_ = o.execute_merged(dk, np.zeros_like(dk), ops)
    gv, gs = run_batch(t, dk, np.zeros_like(dk), ops, E.MODE_SORTED | E.MODE_MERGE_ENGINE)
    assert (gs == os_).all() and (gv == ov).all()
    qk, _, _ = O.gen_requests("uniform", 70, o.dump()[0], 100_000, 100)
    qk[:2000] = dk  # deleted keys, in emptied leaves
    ov, os_ = o.execute_merged(qk, np.zeros_like(qk), np.ones(qk.size, np.uint8))
    t.reset_stats()
    lv, ls = lookups(t, qk)
    assert (ls == os_).all() and (lv == ov).all()
    before = t.stats()["learned_fallbacks"]
    loss0 = t.learned_info()["loss"]
    t.refit()
    info = t.learned_info()
    assert info["valid"] == 1 and info["loss"] == loss0  # stage 1 untouched
    t.reset_stats()
    lv, ls = lookups(t, qk)
    assert (ls == os_).all() and (lv == ov).all()
    after = t.stats()["learned_fallbacks"]
    assert after < before, (before, after)
    # a refit with warm-started steps trains stage 1 further and stays exact
    t.set_option(E.OPT_REFIT_STEPS, 20)
    t.refit()
    lv, ls = lookups(t, qk)
    assert (ls == os_).all() and (lv == ov).all()


def test_segment_count_follows_the_leaves(gpu):
    # default (n_segments 0): one segment line per 64 leaves at each full
    # training, a power of two, at least 4096; a refit keeps the count; an
    # explicit count is used as given.  Lookups stay exact either way.
    for n_keys in (200_000, 12_000_000):
        keys = O.gen_keys("uniform", 61, n_keys)
        vals = O.value_of(keys)
        t = E.BTree(max_keys=1 << 25, max_batch=1 << 18)
        t.bulk_build(dev(keys), dev(vals))
        t.retrain()
        info = t.learned_info()
        leaves = int(info["n_leaves"])
        want = 4096
        while want < (leaves + 63) // 64:
            want *= 2
        assert int(info["n_segments"]) == want, (leaves, info["n_segments"])
        rk, rv, ro = O.gen_requests("uniform", 62, keys, 100_000, 50)
        run_batch(t, rk, rv, ro, E.MODE_SORTED | E.MODE_MERGE_ENGINE)
        t.refit()
        assert int(t.learned_info()["n_segments"]) == want
        qk, _, _ = O.gen_requests("uniform", 63, keys, 200_000, 100)
        t.set_descent(True)
        lv, ls = lookups(t, qk)
        t.set_descent(False)
        pv, ps = lookups(t, qk)
        assert (lv == pv).all() and (ls == ps).all()
        t.close()
    t = E.BTree(max_keys=1 << 21, max_batch=1 << 18, n_segments=512)
    keys = O.gen_keys("uniform", 64, 300_000)
    t.bulk_build(dev(keys), dev(O.value_of(keys)))
    t.retrain()
    assert int(t.learned_info()["n_segments"]) == 512


@pytest.mark.parametrize("policy", [0, 1, 2])
def test_learned_policy_on_a_fast_growing_tree(gpu, policy):
    # 50/50 batches of 120 K requests on a 150 K-key tree: leaves split in
    # every batch and the learned lookups of a batch miss more and more.
    # Policy 0 keeps the learned descent; policy 1 answers with the plain
    # descent once the sampled miss rate passes 5 %, until bt_refit; policy 2
    # refits by itself 8 batches after the last fit.  Every batch is exact.
    keys = O.gen_keys("uniform", 71, 150_000)
    vals = O.value_of(keys)
    t = E.BTree(max_keys=1 << 23, max_batch=1 << 18)
    t.bulk_build(dev(keys), dev(vals))
    o = O.OracleTree()
    o.bulk_build(keys, vals)
    t.retrain()
    t.set_descent(True)
    t.set_option(E.OPT_LEARNED_POLICY, policy)
    merge = E.MODE_SORTED | E.MODE_MERGE_ENGINE
    used = []
    prev = t.stats()["learned_hits"] + t.stats()["learned_fallbacks"]
    for b in range(14):
        if policy == 1 and b == 10:
            t.refit()
        rk, rv, ro = O.gen_requests("uniform", 80 + b, keys, 120_000, 50)
        ov, os_ = o.execute_merged(rk, rv, ro, engine=O.ENGINE_MERGE)
        gv, gs = run_batch(t, rk, rv, ro, merge)
        assert (gs == os_).all() and (gv == ov).all(), b
        st = t.stats()
        now = st["learned_hits"] + st["learned_fallbacks"]
        used.append(now > prev)  # this batch's lookups went through the model
        prev = now
    if policy == 0:
        assert all(used)
    elif policy == 1:
        assert used[0] and not all(used[1:10])  # dropped once stale
        assert not any(used[6:10])
        assert used[10]  # back after the refit
    else:
        assert used[0] and not all(used[1:8])
        assert any(used[8:])  # refit by itself, learned again
    gk, gv = dump(t)
    ok, ovv = o.dump()
    assert (gk == ok).all() and (gv == ovv).all()
