"""Generate golden answers by running the reference program itself.

Runs oracle/_ref/stm_test (the reference built from its own sources by
oracle/build_ref.sh) on seeded 31-bit-key inputs written in the reference's
text format (`P key val` / `R key`, src/input-helper.h:161-163,
Data_Collector::readFile src/input-helper.h:257-317) and parses the answers it
prints with -t (Data_Collector::test, src/input-helper.h:327-340).  Writes
tests/golden/ref_<version>.npz: the generator parameters, the first N answers
(status, value) and a SHA-256 of all answers.  Needs a GPU (the reference is
CUDA-only); run it on the GPU box:

    python tests/golden/make_golden.py            # writes tests/golden/ref_v39.npz, ref_v38.npz

Every file holds an exact multiple of the reference's batch (1,310,720
requests, src/gpu-stm-tree-v39/bpt-gpustm.h:25-38), so v38's tail-batch path,
which reads answers it never wrote (src/gpu-stm-tree-v38/bpt-gpustm.cpp:131),
never runs.
"""
from __future__ import annotations

import argparse
import hashlib
import os
import subprocess
import sys
import tempfile
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

REF_BATCH = 1_310_720
N_KEEP = 16384


def mix64(x: np.ndarray) -> np.ndarray:
    x = x.astype(np.uint64)
    with np.errstate(over="ignore"):
        x = (x ^ (x >> np.uint64(30))) * np.uint64(0xBF58476D1CE4E5B9)
        x = (x ^ (x >> np.uint64(27))) * np.uint64(0x94D049BB133111EB)
    return x ^ (x >> np.uint64(31))


def key31(seed: int, n: int) -> np.ndarray:
    """n distinct keys in [0, 2^31 - 1) (INT_MAX is the reference's MAX_KEY)."""
    out = np.zeros(0, np.uint64)
    c = 0
    while out.size < n:
        i = np.arange(c, c + 2 * n, dtype=np.uint64)
        with np.errstate(over="ignore"):
            k = mix64(i * np.uint64(0x9E3779B97F4A7C15) + np.uint64(seed)) >> np.uint64(33)
        k = k[k < np.uint64(2**31 - 1)]
        out = np.unique(np.concatenate([out, k]))
        c += 2 * n
    rng = np.random.default_rng(seed)
    return rng.permutation(out)[:n]


def workload(version: int):
    """(build keys, build vals, query keys, query vals, query ops) for one version."""
    nb = REF_BATCH
    pool = key31(1000 + version, 2 * nb + 200_000)
    bk = pool[:nb]
    bv = (bk * np.uint64(7) + np.uint64(3)) & np.uint64(0x7FFFFFFF)
    fresh = pool[nb:]
    rng = np.random.default_rng(version)
    nq = REF_BATCH
    if version == 39:
        # distinct keys in the query batch: the v39 result is then order independent
        n_put = nq // 20
        n_hit = (nq - n_put) // 2
        qk = np.concatenate([rng.choice(bk, n_hit + n_put // 2, replace=False),
                             fresh[: nq - n_hit - n_put // 2]])
        qk = rng.permutation(qk)
        qo = np.ones(nq, np.uint8)
        put_idx = rng.choice(nq, n_put, replace=False)
        qo[put_idx] = 0
    else:
        # duplicate heavy: the v38 sort-merge meaning is exercised
        hot = np.concatenate([rng.choice(bk, 30_000, replace=False), fresh[:20_000]])
        qk = hot[rng.integers(0, hot.size, nq)]
        qo = (rng.random(nq) < 0.8).astype(np.uint8)
    qv = (np.arange(nq, dtype=np.uint64) * np.uint64(13) + np.uint64(5)) & np.uint64(0x7FFFFFFF)
    return bk, bv, qk, qv, qo


def write_files(d, bk, bv, qk, qv, qo):
    b = os.path.join(d, "build.txt")
    q = os.path.join(d, "query.txt")
    with open(b, "w") as f:
        f.write("".join(f"P {k} {v}\n" for k, v in zip(bk.tolist(), bv.tolist())))
    lines = []
    for k, v, o in zip(qk.tolist(), qv.tolist(), qo.tolist()):
        lines.append(f"P {k} {v}\n" if o == 0 else f"R {k}\n")
    with open(q, "w") as f:
        f.write("".join(lines))
    return b, q


def parse_answers(text: str, n: int):
    st = np.zeros(n, np.uint8)
    val = np.zeros(n, np.uint64)
    i = 0
    for line in text.splitlines():
        if not line.startswith("key: "):
            continue
        parts = line.split("\t")
        ans = int(parts[2].split(":")[1])
        if ans != -1:
            st[i] = 1
            val[i] = int(parts[3].split(":")[1])
        i += 1
    if i != n:
        raise RuntimeError(f"parsed {i} answers, expected {n}")
    return st, val


def digest(st, val) -> str:
    return hashlib.sha256(st.tobytes() + val.tobytes()).hexdigest()


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--ref", default=os.path.join(ROOT, "oracle", "_ref", "stm_test"))
    ap.add_argument("--out", default=HERE)
    ap.add_argument("--versions", default="39,38")
    a = ap.parse_args()
    for v in [int(x) for x in a.versions.split(",")]:
        bk, bv, qk, qv, qo = workload(v)
        with tempfile.TemporaryDirectory() as d:
            b, q = write_files(d, bk, bv, qk, qv, qo)
            t0 = time.time()
            r = subprocess.run([a.ref, f"-v{v}", "-i", b, "-t", "-i", q], capture_output=True, text=True,
                               timeout=600)
            if r.returncode != 0:
                raise RuntimeError(f"stm_test -v{v} failed rc={r.returncode}: {r.stderr[-2000:]}")
            st, val = parse_answers(r.stdout, qk.size)
            times = [ln for ln in r.stdout.splitlines() if "total gpu exec time" in ln]
        np.savez_compressed(os.path.join(a.out, f"ref_v{v}.npz"), version=v, status=st[:N_KEEP],
                            value=val[:N_KEEP], sha256=digest(st, val), n=qk.size,
                            found=int(st.sum()), ref_times=np.array(times))
        print(f"v{v}: {qk.size} answers, {int(st.sum())} found, sha256 {digest(st, val)[:16]}, "
              f"{time.time() - t0:.1f}s, {times}")


if __name__ == "__main__":
    main()
