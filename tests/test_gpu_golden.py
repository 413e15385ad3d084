"""The CUDA path against the reference program's own answers (fixtures made by
tests/golden/make_golden.py from the reference built from its sources):
BT_MODE_STM on the v39 workload (distinct keys), BT_MODE_SORTED on the
duplicate-heavy v38 workload."""
import os
import sys

import numpy as np
import pytest

import eirene_b200 as E
from tests.helpers import dev, run_batch

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(HERE, "golden"))
import make_golden as G  # noqa: E402

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("version,mode", [(39, E.MODE_STM), (38, E.MODE_SORTED), (39, E.MODE_SORTED)])
def test_cuda_path_matches_reference_answers(gpu, version, mode):
    ref = np.load(os.path.join(HERE, "golden", f"ref_v{version}.npz"))
    bk, bv, qk, qv, qo = G.workload(version)
    t = E.BTree(max_keys=4 * bk.size, max_batch=qk.size)
    t.bulk_build(dev(bk), dev(bv))
    gv, gs = run_batch(t, qk, qv, qo, mode)
    k = ref["status"].size
    assert (gs[:k] == ref["status"]).all()
    assert (gv[:k] == ref["value"]).all()
    assert G.digest(gs, gv) == str(ref["sha256"])
