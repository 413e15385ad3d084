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
