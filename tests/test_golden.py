"""Pins the oracle to the reference program's own answers.

tests/golden/ref_v39.npz and ref_v38.npz were produced by running the
reference (built from its sources by oracle/build_ref.sh) on seeded 31-bit-key
inputs; tests/golden/make_golden.py regenerates the same inputs here, the
oracle answers them, and the answers must match the reference's: the first
16384 exactly and all 1,310,720 through a SHA-256."""
import os
import sys

import numpy as np
import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(HERE, "golden"))

import make_golden as G  # noqa: E402
from oracle import oracle as O  # noqa: E402


@pytest.mark.parametrize("version", [39, 38])
def test_oracle_matches_reference_answers(version):
    path = os.path.join(HERE, "golden", f"ref_v{version}.npz")
    if not os.path.exists(path):
        pytest.skip(f"{path} missing: run tests/golden/make_golden.py on a GPU box")
    ref = np.load(path)
    bk, bv, qk, qv, qo = G.workload(version)
    t = O.OracleTree()
    t.bulk_build(bk, bv)
    if version == 39:
        ov, os_ = t.execute_serial(qk, qv, qo)
    else:
        ov, os_ = t.execute_merged(qk, qv, qo)
    k = ref["status"].size
    assert (os_[:k] == ref["status"]).all()
    assert (ov[:k] == ref["value"]).all()
    assert int(os_.sum()) == int(ref["found"])
    assert G.digest(os_.astype(np.uint8), ov.astype(np.uint64)) == str(ref["sha256"])
