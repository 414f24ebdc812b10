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
