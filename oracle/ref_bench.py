"""Times the reference GPU program on its own benchmark shape next to this
library on the same inputs (test infrastructure; needs oracle/_ref/stm_test).

Shape of the reference's published runs (evalutaion/random_testall_v39.sh:9-28,
prof/query23_uniform_95_v39.res): build from 2^23 - 1 `P` lines, then a query
file of 95 % `R` / 5 % `P` lines, run in batches of 1,310,720.  Keys are 31-bit
(the reference is int32).  The reference reports "total gpu exec time" (device
time of its kernels, transfers excluded: v39 times the kernel only, v38 all
phases); this library is timed the same way (device time of bt_execute_batch
over resident inputs).

    python oracle/ref_bench.py --batches 10 > ref_bench.json
"""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import tempfile
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "tests", "golden"))

REF_BATCH = 1_310_720


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--batches", type=int, default=10)
    ap.add_argument("--tree", type=int, default=(1 << 23) - 1)
    ap.add_argument("--versions", default="39,38")
    a = ap.parse_args()
    import make_golden as G

    pool = G.key31(77, a.tree + a.batches * REF_BATCH)
    bk = pool[: a.tree]
    fresh = pool[a.tree:]
    bv = (bk * np.uint64(7) + np.uint64(3)) & np.uint64(0x7FFFFFFF)
    rng = np.random.default_rng(5)
    nq = a.batches * REF_BATCH
    is_get = rng.random(nq) < 0.95
    qk = np.where(rng.random(nq) < 0.5, bk[rng.integers(0, bk.size, nq)], fresh[rng.integers(0, fresh.size, nq)])
    qk = np.where(is_get, qk, fresh[rng.permutation(nq) % fresh.size])
    qo = np.where(is_get, 1, 0).astype(np.uint8)
    qv = (np.arange(nq, dtype=np.uint64) * np.uint64(13) + np.uint64(5)) & np.uint64(0x7FFFFFFF)
    out = {"tree_keys": int(bk.size), "requests": int(nq), "batch": REF_BATCH, "search_frac": 0.95}
    ref = os.path.join(HERE, "_ref", "stm_test")
    with tempfile.TemporaryDirectory() as d:
        b, q = G.write_files(d, bk, bv, qk, qv, qo)
        for v in [int(x) for x in a.versions.split(",") if x]:
            t0 = time.time()
            r = subprocess.run([ref, f"-v{v}", "-i", b, "-i", q], capture_output=True, text=True, timeout=900)
            if r.returncode != 0:
                out[f"v{v}"] = {"error": r.stderr[-500:]}
                continue
            times = [float(ln.split(":")[1]) for ln in r.stdout.splitlines() if "total gpu exec time" in ln]
            out[f"v{v}"] = {"build_s": times[0], "query_s": times[1], "query_mops": nq / times[1] / 1e6,
                            "wall_s": time.time() - t0}
    # this library on the same inputs, device timed, sorted mode (v38 meaning)
    import torch

    import eirene_b200 as E

    k = torch.from_numpy(qk.view(np.int64)).cuda()
    v = torch.from_numpy(qv.view(np.int64)).cuda()
    o = torch.from_numpy(qo).cuda()
    ov = torch.empty(REF_BATCH, dtype=torch.int64, device="cuda")
    os_ = torch.empty(REF_BATCH, dtype=torch.uint8, device="cuda")
    for mode_name, mode in [("sorted", E.MODE_SORTED), ("stm", E.MODE_STM)]:
        tt = E.BTree(max_keys=2 * bk.size + nq, max_batch=REF_BATCH)
        tt.bulk_build(torch.from_numpy(bk.view(np.int64)).cuda(), torch.from_numpy(bv.view(np.int64)).cuda())
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        for i in range(a.batches):
            s = slice(i * REF_BATCH, (i + 1) * REF_BATCH)
            tt.execute(k[s], v[s], o[s], ov, os_, mode=mode)
        e1.record()
        torch.cuda.synchronize()
        ms = e0.elapsed_time(e1)
        out[f"b200_{mode_name}"] = {"query_s": ms / 1e3, "query_mops": nq / (ms / 1e3) / 1e6}
        tt.close()
    print(json.dumps(out))


if __name__ == "__main__":
    main()
