"""CPU checks of the C ABI: the library builds for sm_100a, loads, and exports
every entry point include/eirene_b200.h declares."""
import os
import re

import eirene_b200

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def header_symbols():
    src = open(os.path.join(ROOT, "include", "eirene_b200.h")).read()
    return sorted(set(re.findall(r"^(?:int|uint64_t|const char \*)\s*\*?(bt_\w+)\(", src, re.M)))


def test_library_exports_every_declared_symbol():
    eirene_b200.build()
    L = eirene_b200.lib()
    syms = header_symbols()
    assert len(syms) >= 20
    for s in syms:
        assert hasattr(L, s), s
    assert set(syms) == set(eirene_b200.EXPORTS)


def test_status_strings():
    L = eirene_b200.lib()
    assert L.bt_status_string(0) == b"ok"
    assert L.bt_status_string(-6) == b"batch larger than max_batch"


def test_create_without_gpu_fails_cleanly():
    import torch

    if torch.cuda.is_available():
        return
    try:
        eirene_b200.BTree(max_keys=1024, max_batch=1024)
    except eirene_b200.BTError as e:
        assert e.code == -2
    else:
        raise AssertionError("bt_create succeeded without a GPU")
