"""The C-ABI library loads and exports every entry point include/qcp.h
declares; argument validation answers without touching a GPU.  CPU only."""
from __future__ import annotations

import ctypes
import re

import pytest

from conftest import ROOT, ensure_library


def declared_symbols():
    text = (ROOT / "include" / "qcp.h").read_text()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(qcp_[a-z_]+)\s*\(", text)))


def test_header_declares_entry_points():
    syms = declared_symbols()
    for must in ["qcp_index_build", "qcp_query_batch", "qcp_query_counts", "qcp_index_free",
                 "qcp_result_release", "qcp_last_error"]:
        assert must in syms


def test_library_exports_every_declared_symbol():
    lib = ctypes.CDLL(str(ensure_library()))
    missing = [s for s in declared_symbols() if not hasattr(lib, s)]
    assert not missing, missing


def test_bad_arguments_rejected_without_device(qcp):
    lib = qcp.load_library()
    h = ctypes.c_void_p()
    # NULL objects, zero objects, dims out of range, bad fanout: all BAD_ARG
    assert lib.qcp_index_build(None, 10, 3, 0, None, ctypes.byref(h)) == 1
    buf = (ctypes.c_float * 30)()
    assert lib.qcp_index_build(buf, 0, 3, 0, None, ctypes.byref(h)) == 1
    assert lib.qcp_index_build(buf, 10, 9, 0, None, ctypes.byref(h)) == 1
    opts = qcp.BuildOpts(48, 0, 0, 0, None)
    assert lib.qcp_index_build(buf, 10, 3, 0, ctypes.byref(opts), ctypes.byref(h)) == 1
    assert b"fanout" in lib.qcp_last_error()
    opts = qcp.BuildOpts(128, 0, 40, 0, None)
    assert lib.qcp_index_build(buf, 10, 3, 0, ctypes.byref(opts), ctypes.byref(h)) == 1
    assert not h.value


def test_python_binding_fails_loudly_without_library(qcp, tmp_path):
    with pytest.raises(FileNotFoundError):
        qcp.load_library(tmp_path / "missing.so")


def test_version(qcp):
    assert qcp.load_library().qcp_version().startswith(b"qcp-b200")
