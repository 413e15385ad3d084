"""The reference-shaped C++ plugin end to end on the GPU: the command-line
driver runs the same text files the reference program ran for the golden
fixtures (build file of `P key val` lines through batched inserts into an
empty tree, then the query file) and prints its answers in the reference's
format (src/input-helper.h:327-340); the parsed answers must hash to the
reference's own digest."""
import os
import subprocess
import sys
import tempfile

import numpy as np
import pytest

import eirene_b200 as E

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(HERE, "golden"))
import make_golden as G  # noqa: E402

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("version,flag", [(39, "-v39"), (38, "-v38"), (38, "-v40"), (38, "-v41")])
def test_cli_matches_reference_digest(gpu, version, flag):
    cli = os.path.join(os.path.dirname(E.__file__), "bt_stm_test")
    ref = np.load(os.path.join(HERE, "golden", f"ref_v{version}.npz"))
    bk, bv, qk, qv, qo = G.workload(version)
    with tempfile.TemporaryDirectory() as d:
        b, q = G.write_files(d, bk, bv, qk, qv, qo)
        r = subprocess.run([cli, flag, "-i", b, "-t", "-i", q], capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stdout[-2000:] + r.stderr[-2000:]
    st, val = G.parse_answers(r.stdout, qk.size)
    k = ref["status"].size
    assert (st[:k] == ref["status"]).all() and (val[:k] == ref["value"]).all()
    assert G.digest(st, val) == str(ref["sha256"])
    assert sum("total gpu exec time" in ln for ln in r.stdout.splitlines()) == 2


def test_cli_range_file(gpu, tmp_path):
    # -r runs "lo [hi]" queries through bt_range_batch; each printed count and
    # the first pairs must equal the keys of the loaded tree in [lo, hi]
    cli = os.path.join(os.path.dirname(E.__file__), "bt_stm_test")
    rng = np.random.default_rng(7)
    keys = np.unique(rng.integers(0, 1 << 31, 20_000, dtype=np.uint64))
    rng.shuffle(keys)
    b = tmp_path / "build.txt"
    b.write_text("".join(f"P {k} {int(k) * 3 + 1}\n" for k in keys))
    sk = np.sort(keys)
    lo = sk[rng.integers(0, sk.size, 300)]
    span = rng.integers(0, 1 << 20, 300).astype(np.uint64)
    hi = lo + span
    lines = [f"{a} {c}\n" for a, c in zip(lo, hi)] + [f"{sk[-5]}\n", "0 0\n"]
    r_file = tmp_path / "range.txt"
    r_file.write_text("".join(lines))
    r = subprocess.run([cli, "-v40", "-i", str(b), "-t", "-r", str(r_file)], capture_output=True, text=True,
                       timeout=600)
    assert r.returncode == 0, r.stdout[-2000:] + r.stderr[-2000:]
    out = [ln for ln in r.stdout.splitlines() if ln.startswith("range:") or ln.startswith("  key:")]
    queries = list(zip(lo, hi)) + [(sk[-5], np.uint64(2**64 - 1)), (np.uint64(0), np.uint64(0))]
    i = 0
    for a, c in queries:
        head = out[i].split()
        assert int(head[1]) == int(a) and int(head[2]) == int(c)
        want = sk[(sk >= a) & (sk <= c)]
        assert int(head[4]) == want.size
        i += 1
        for j in range(min(want.size, 16)):
            f = out[i].split()
            assert int(f[1]) == int(want[j])
            assert int(f[5]) == int(want[j]) * 3 + 1  # the warehouse value behind the stored offset
            i += 1
    assert i == len(out)
