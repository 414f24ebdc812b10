"""Shared test setup.

Tests marked `gpu` need a CUDA device and call the library through its C ABI;
everything else runs on the CPU (oracle against the golden vectors, library
exports, host logic).
"""
from __future__ import annotations

import importlib.util
import pathlib
import subprocess
import sys

import numpy as np
import pytest

ROOT = pathlib.Path(__file__).resolve().parent.parent
PKG_DIR = ROOT / "query-co-processing-on-heterogeneous-architectures_b200"
GOLDEN = ROOT / "tests" / "golden"

sys.path.insert(0, str(ROOT / "oracle"))
sys.path.insert(0, str(GOLDEN))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200)")


def load_pkg():
    """Import the package directory (its name is not a Python identifier)."""
    if "qcp_b200" in sys.modules:
        return sys.modules["qcp_b200"]
    spec = importlib.util.spec_from_file_location("qcp_b200", PKG_DIR / "__init__.py",
                                                  submodule_search_locations=[str(PKG_DIR)])
    mod = importlib.util.module_from_spec(spec)
    sys.modules["qcp_b200"] = mod
    spec.loader.exec_module(mod)
    return mod


def ensure_library() -> pathlib.Path:
    lib = PKG_DIR / "libqcp_b200.so"
    if not lib.exists():
        subprocess.run(["make", "-s", "-j4", "-C", str(PKG_DIR)], check=True)
    return lib


@pytest.fixture(scope="session")
def qcp():
    ensure_library()
    return load_pkg()


@pytest.fixture(scope="session")
def workloads():
    load_pkg()
    import qcp_b200.workloads as w  # noqa: E402
    return w


@pytest.fixture(scope="session")
def oracle():
    from oracle import Oracle
    return Oracle()


@pytest.fixture(scope="session")
def cases():
    import cases as c
    return c


def golden(name: str):
    return np.load(GOLDEN / name)


def assert_same_hits(res_offsets, res_ids, ref_offsets, ref_ids, boxes=None):
    """Per-query sorted id lists equal (bit-exact)."""
    res_offsets = np.asarray(res_offsets, dtype=np.uint64)
    ref_offsets = np.asarray(ref_offsets, dtype=np.uint64)
    if not np.array_equal(res_offsets, ref_offsets):
        cr, co = np.diff(res_offsets.astype(np.int64)), np.diff(ref_offsets.astype(np.int64))
        bad = np.nonzero(cr != co)[0]
        raise AssertionError(f"{len(bad)} queries differ in hit count; first {bad[:5]}: "
                             f"got {cr[bad[:5]]} want {co[bad[:5]]}"
                             + (f" boxes {boxes[bad[:2]]}" if boxes is not None else ""))
    if not np.array_equal(np.asarray(res_ids), np.asarray(ref_ids)):
        diff = np.nonzero(np.asarray(res_ids) != np.asarray(ref_ids))[0]
        q = np.searchsorted(res_offsets, diff[0], side="right") - 1
        raise AssertionError(f"ids differ at {len(diff)} positions, first in query {q}")
