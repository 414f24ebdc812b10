"""Error behaviour of the C++ host side (io::DataSet, tree::B200Index and the
qcp_eval driver) that needs no GPU: a bad command line prints the usage, a
missing or short data file is reported with its path, and a machine without
a CUDA device gets a message and a non-zero exit, never a crash.  The
reference exits the process on a missing file with the same message
(src/io/dataset.cpp:30-33)."""
from __future__ import annotations

import subprocess

import numpy as np
import pytest

from conftest import PKG_DIR


@pytest.fixture(scope="module")
def exe():
    path = PKG_DIR / "qcp_eval"
    if not path.exists():
        subprocess.run(["make", "-s", "-C", str(PKG_DIR)], check=True, timeout=900)
    return path


def run(exe, *args):
    return subprocess.run([str(exe), *map(str, args)], capture_output=True, text=True, timeout=120)


@pytest.fixture()
def files(tmp_path):
    data = tmp_path / "data.bin"
    query = tmp_path / "query.bin"
    np.random.default_rng(1).random((1000, 3), dtype=np.float32).tofile(data)
    np.random.default_rng(2).random((10, 6), dtype=np.float32).tofile(query)
    return data, query


def test_usage_without_arguments(exe):
    r = run(exe)
    assert r.returncode != 0
    assert "Usage" in r.stdout + r.stderr


def test_missing_data_file_is_reported(exe, files, tmp_path):
    _, query = files
    missing = tmp_path / "missing.bin"
    r = run(exe, "-d", 1000, "-q", 10, "-D", missing, "-Q", query)
    assert r.returncode == 1
    assert f"Failed to open a file({missing})" in r.stdout + r.stderr


def test_short_data_file_is_reported(exe, files):
    data, query = files
    r = run(exe, "-d", 5000, "-q", 10, "-D", data, "-Q", query)  # the file holds 1000 points
    assert r.returncode == 1
    assert f"short read from {data}" in r.stdout + r.stderr


def test_no_device_is_an_error_not_a_crash(exe, files):
    import torch
    if torch.cuda.is_available():
        pytest.skip("a CUDA device is present")
    data, query = files
    r = run(exe, "-d", 1000, "-q", 10, "-D", data, "-Q", query, "-k", 3, "-i", "b200")
    assert r.returncode == 1
    assert "no CUDA device" in r.stdout + r.stderr
