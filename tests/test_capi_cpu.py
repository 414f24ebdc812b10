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


STRUCTS = [("BuildOpts", "qcp_build_opts"), ("IndexInfo", "qcp_index_info"), ("QueryOpts", "qcp_query_opts"),
           ("QueryStats", "qcp_query_stats"), ("Result", "qcp_result"), ("TuneResult", "qcp_tune_result"),
           ("ServeOpts", "qcp_serve_opts"), ("ServeStats", "qcp_serve_stats"), ("ServeBatch", "qcp_serve_batch")]


def test_binding_struct_layouts_match_header(qcp, tmp_path):
    """Every ctypes mirror of a qcp.h struct has the C compiler's size and
    field offsets (a C program built against the header prints them)."""
    import shutil
    import subprocess
    if not shutil.which("gcc"):
        pytest.skip("gcc not found")
    lines = ["#include <stddef.h>", "#include <stdio.h>", '#include "qcp.h"', "int main(void) {"]
    for py, c in STRUCTS:
        lines.append(f'  printf("{c} sizeof %zu\\n", sizeof({c}));')
        for f in getattr(qcp, py)._fields_:
            lines.append(f'  printf("{c} {f[0]} %zu\\n", offsetof({c}, {f[0]}));')
    lines += ["  return 0;", "}"]
    src = tmp_path / "layout.c"
    src.write_text("\n".join(lines) + "\n")
    exe = tmp_path / "layout"
    subprocess.run(["gcc", "-std=c99", "-I", str(ROOT / "include"), str(src), "-o", str(exe)], check=True)
    got = {}
    for ln in subprocess.run([str(exe)], check=True, capture_output=True, text=True).stdout.splitlines():
        c, f, v = ln.split()
        got[(c, f)] = int(v)
    for py, c in STRUCTS:
        cls = getattr(qcp, py)
        assert got[(c, "sizeof")] == ctypes.sizeof(cls), c
        for f in cls._fields_:
            assert got[(c, f[0])] == getattr(cls, f[0]).offset, (c, f[0])
    assert qcp.SERVE_BATCH_DTYPE.itemsize == ctypes.sizeof(qcp.ServeBatch)


def test_newer_entry_points_reject_bad_arguments_without_device(qcp, tmp_path):
    """Plans, serving, the autotuner, the no-allocation counts and index
    files check their arguments before any device work: NULL handles and
    empty inputs are BAD_ARG with a message, a missing index file is IO."""
    lib = qcp.load_library()
    P = ctypes.c_void_p
    h = P()
    BAD_ARG, IO = 1, 7
    assert lib.qcp_plan_create(None, 16, 1000, None, ctypes.byref(h)) == BAD_ARG
    assert lib.qcp_last_error()
    assert lib.qcp_plan_run(None, None, 0, 0, None, None, None, None) == BAD_ARG
    assert lib.qcp_plan_free(None) == 0
    st = qcp.ServeStats()
    assert lib.qcp_serve_replay(None, None, None, 0, None, None, ctypes.byref(st)) == BAD_ARG
    assert lib.qcp_autotune(None, 0, 3, 0, None, 0, None, 0, None) == BAD_ARG
    assert lib.qcp_query_counts_noalloc(None, None, 4, None, None) == BAD_ARG
    buf = (ctypes.c_float * 12)()
    res = qcp.Result()
    assert lib.qcp_query_batch(None, buf, 2, None, ctypes.byref(res)) == BAD_ARG
    assert lib.qcp_query_batch(None, buf, 2, None, None) == BAD_ARG
    counts = (ctypes.c_uint64 * 2)()
    assert lib.qcp_query_counts(None, buf, 2, None, counts) == BAD_ARG
    assert lib.qcp_index_load(str(tmp_path / "none.qcpidx").encode(), None, ctypes.byref(h)) == IO
    assert not h.value


def test_build_plan_rejects_bad_arguments_without_device(qcp):
    """The captured build checks its shape and key mode before touching a
    device: n, dims, fan-out and key mode out of range are BAD_ARG."""
    lib = qcp.load_library()
    P = ctypes.c_void_p
    h = P()
    BAD_ARG = 1
    assert lib.qcp_build_plan_create(0, 3, 0, None, ctypes.byref(h)) == BAD_ARG
    assert lib.qcp_build_plan_create(1000, 9, 0, None, ctypes.byref(h)) == BAD_ARG
    bo = qcp.BuildOpts(100, 0, 0, 0, None, 0, 0)  # fan-out not a multiple of 32
    assert lib.qcp_build_plan_create(1000, 3, 0, ctypes.byref(bo), ctypes.byref(h)) == BAD_ARG
    bo = qcp.BuildOpts(128, qcp.KEY_KMEANS, 0, 0, None, 0, 0)
    assert lib.qcp_build_plan_create(1000, 3, 0, ctypes.byref(bo), ctypes.byref(h)) == BAD_ARG
    assert b"k-means" in lib.qcp_last_error()
    assert lib.qcp_build_plan_create(1000, 3, 0, None, None) == BAD_ARG
    assert not h.value
    assert lib.qcp_build_plan_run(None, None, 0, None, ctypes.byref(h)) == BAD_ARG
    assert lib.qcp_build_plan_input(None) is None
    assert lib.qcp_build_plan_free(None) == 0

