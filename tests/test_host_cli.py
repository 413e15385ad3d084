"""The C++ host plugin (eirene_b200/host: GPU_BTree shape of src/tree.h:28-43)
and its command-line driver with the reference's options (src/main.cpp:57-109),
without a GPU: usage errors and the loud failure when no device is present."""
import os
import subprocess

import pytest

import eirene_b200 as E

from tests.conftest import has_gpu


@pytest.fixture(scope="module")
def cli():
    E.build()
    path = os.path.join(os.path.dirname(E.__file__), "bt_stm_test")
    assert os.access(path, os.X_OK)
    return path


def test_usage_without_version(cli):
    r = subprocess.run([cli], capture_output=True, text=True, timeout=60)
    assert r.returncode == 2 and "usage" in r.stderr


def test_unknown_version_rejected(cli):
    r = subprocess.run([cli, "-v7"], capture_output=True, text=True, timeout=60)
    assert r.returncode == 2 and "unknown version" in r.stderr


def test_range_file_before_version_rejected(cli, tmp_path):
    r = subprocess.run([cli, "-r", str(tmp_path / "x")], capture_output=True, text=True, timeout=60)
    assert r.returncode == 2 and "-v must come first" in r.stderr


@pytest.mark.skipif(has_gpu(), reason="checks the no-device path")
def test_no_device_fails_loudly(cli, tmp_path):
    f = tmp_path / "q.txt"
    f.write_text("P 5 7\nR 5\n")
    r = subprocess.run([cli, "-v39", "-i", str(f)], capture_output=True, text=True, timeout=120)
    assert r.returncode == 1 and r.stdout.startswith("Error:")
