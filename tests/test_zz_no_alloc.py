"""qcp_query_counts_noalloc: the counting entry point that allocates nothing.

It exists for callers that must not call cudaMalloc while they query (their
device memory belongs to another allocator, or a serving loop cannot take
cudaMalloc's implicit synchronisation); it keeps its scratch in one fixed
array inside the library's device image.  These tests call it through the C
ABI and check it against qcp_query_counts, twice in a row, with different
batches so that nothing from the first call leaks into the second.  Needs a
GPU.  The file is named so that pytest collects it last."""
from __future__ import annotations

import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _bind(qcp):
    lib = qcp.load_library()
    fn = lib.qcp_query_counts_noalloc
    fn.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_uint32, ctypes.c_void_p, ctypes.c_void_p]
    fn.restype = ctypes.c_int
    return lib, fn


def test_noalloc_counts_match_existing_entry_point(qcp, cases, workloads):
    import torch
    lib, fn = _bind(qcp)
    objs, boxes_a, _ = cases.COUNT_CASES["g3"]()
    _, boxes_b, _ = cases.COUNT_CASES["u3"]()
    boxes_c = workloads.data_centred_cubes(objs, 3000, 1e-6, 1e-2, seed=11)
    with qcp.Index.build(objs) as ix:
        free_before_second = None
        for k, boxes in enumerate([boxes_a, boxes_b, boxes_c]):
            want = ix.counts(boxes)  # the existing entry point
            d_boxes = torch.from_numpy(np.ascontiguousarray(boxes)).cuda()
            d_counts = torch.full((len(boxes),), -1, dtype=torch.int64, device="cuda")  # must be overwritten
            torch.cuda.synchronize()
            if k == 1:
                free_before_second = torch.cuda.mem_get_info()[0]
            st = fn(ix._h, d_boxes.data_ptr(), len(boxes), d_counts.data_ptr(), None)
            assert st == 0, lib.qcp_last_error()
            torch.cuda.synchronize()
            if k == 1:
                # a call after the first allocates no device memory
                assert torch.cuda.mem_get_info()[0] == free_before_second
            got = d_counts.cpu().numpy().astype(np.uint64)
            assert np.array_equal(got, want), f"batch {k}"


def _rect8():
    rng = np.random.default_rng(8)
    lo = rng.random((20000, 8), dtype=np.float32)
    hi = (lo + rng.exponential(0.05, (20000, 8)).astype(np.float32)).astype(np.float32)
    objs = np.ascontiguousarray(np.concatenate([lo, hi], 1))
    c = rng.random((300, 8), dtype=np.float32)
    s = rng.uniform(0.3, 0.7, (300, 8)).astype(np.float32) / 2
    return objs, np.ascontiguousarray(np.concatenate([c - s, c + s], 1), dtype=np.float32), 8


@pytest.mark.parametrize("name", ["u2", "p8", "rect8"])
def test_noalloc_counts_other_shapes(qcp, cases, name):
    """2-D and 8-D points and 8-D rectangles go through the same fixed
    scratch; two calls in a row match qcp_query_counts."""
    import torch
    lib, fn = _bind(qcp)
    if name == "rect8":
        objs, boxes, _ = _rect8()
        is_rect = True
    else:
        objs, boxes, _ = cases.COUNT_CASES[name]()
        is_rect = False
    with qcp.Index.build(objs, is_rect=is_rect) as ix:
        want = ix.counts(boxes)
        d_boxes = torch.from_numpy(np.ascontiguousarray(boxes)).cuda()
        for _ in range(2):
            d_counts = torch.full((len(boxes),), -1, dtype=torch.int64, device="cuda")
            assert fn(ix._h, d_boxes.data_ptr(), len(boxes), d_counts.data_ptr(), None) == 0, lib.qcp_last_error()
            torch.cuda.synchronize()
            assert np.array_equal(d_counts.cpu().numpy().astype(np.uint64), want)


def test_noalloc_frontier_overflow_then_recovers(qcp, cases, workloads):
    """A batch whose frontier passes the scratch's 2^20 items: 1,000 boxes
    covering all of 2,000,000 points at fan-out 32 make 1,953 leaf-parent
    items each (1.95 M > 2^20).  The frontier counters are clamped to the
    scratch, so the kernels stay in bounds; the call reports the overflow,
    and the next, smaller batch is counted exactly."""
    import torch
    lib, fn = _bind(qcp)
    pts = workloads.uniform_points(2_000_000, 3, seed=17)
    every = np.tile(np.array([[-1, -1, -1, 2, 2, 2]], np.float32), (1000, 1))
    _, small, _ = cases.COUNT_CASES["u3"]()
    with qcp.Index.build(pts, fanout=32) as ix:
        d_big = torch.from_numpy(every).cuda()
        d_counts = torch.zeros(len(every), dtype=torch.int64, device="cuda")
        st = fn(ix._h, d_big.data_ptr(), len(every), d_counts.data_ptr(), None)
        assert st == 3, lib.qcp_last_error()  # QCP_ERR_OUTPUT_OVERFLOW
        assert b"split the batch" in lib.qcp_last_error()
        want = ix.counts(small)
        d_small = torch.from_numpy(np.ascontiguousarray(small)).cuda()
        d_counts = torch.full((len(small),), -1, dtype=torch.int64, device="cuda")
        assert fn(ix._h, d_small.data_ptr(), len(small), d_counts.data_ptr(), None) == 0, lib.qcp_last_error()
        torch.cuda.synchronize()
        assert np.array_equal(d_counts.cpu().numpy().astype(np.uint64), want)


def test_noalloc_rejects_what_it_cannot_take(qcp, cases):
    import torch
    lib, fn = _bind(qcp)
    objs, boxes, _ = cases.COUNT_CASES["u3"]()
    with qcp.Index.build(objs) as ix:
        d_counts = torch.zeros(300_000, dtype=torch.int64, device="cuda")
        d_boxes = torch.zeros((300_000, 6), dtype=torch.float32, device="cuda")
        assert fn(ix._h, d_boxes.data_ptr(), 300_000, d_counts.data_ptr(), None) == 1
        assert b"262144" in lib.qcp_last_error()
        host_boxes = np.ascontiguousarray(boxes)
        assert fn(ix._h, host_boxes.ctypes.data, len(boxes), d_counts.data_ptr(), None) == 1
        assert b"device" in lib.qcp_last_error()
