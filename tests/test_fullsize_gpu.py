"""Parity at the benchmarked sizes, through the C ABI.  Needs a GPU.

For every query of the full batches of the batched (16 M clustered 3-D
points, 10,000 cubes), bulk-load stress (64 M uniform 2-D points, 64-bit
keys, fan-outs 64/128/256, 100,000 squares) and rectangle (32 M 8-D
rectangles, 50,000 boxes) workloads:

* per-query counts of qcp_query_counts and the CSR offsets of
  qcp_query_batch equal an independent count: the reference's own CPU BVH
  traversal (BVH::TraverseInternalNodes, src/tree/bvh.cpp:256-278, compiled
  from its sources into oracle/_ref) for points, the plain one-query-per-block
  traversal for rectangles (the reference has no rectangle loader);
* every listed id is in range, every slice is strictly ascending, and every
  id passes the closed-interval predicate (src/node/node_soa.cpp:94-113)
  against its query box.  With equal counts this makes each slice the exact
  sorted hit set;
* the sorted id lists of a seeded sample of queries, the 20 largest results
  among them, equal the oracle's brute-force lists bit for bit.
"""
from __future__ import annotations

import os

import numpy as np
import pytest

from conftest import assert_same_hits, device_result, sample_ids, sample_queries, verify_all_slices

pytestmark = pytest.mark.gpu

THREADS = os.cpu_count() or 8


def _reference(dims):
    from oracle import Reference
    if not Reference.available(dims):
        pytest.skip(f"oracle/_ref/libqcpref_d{dims}.so not built")
    return Reference(dims)


def _bvh_counts(objs, boxes, dims):
    ref = _reference(dims)
    h = ref.bvh_build(objs)
    try:
        return ref.bvh_counts(h, boxes, THREADS).astype(np.uint64)
    finally:
        ref.bvh_free(h)


def _check_index(qcp, oracle, ix, objs, boxes, dims, is_rect, want_counts, nsample):
    import torch
    q = len(boxes)
    d_objs = torch.from_numpy(objs).cuda()
    d_boxes = torch.from_numpy(boxes).cuda()
    # qcp_query_counts
    got = ix.counts(d_boxes, q=q)
    assert np.array_equal(got, want_counts), f"{int((got != want_counts).sum())} counts differ"
    # qcp_query_batch, results left on the device
    res = ix.search(d_boxes, q=q, result_mem=qcp.MEM_DEVICE)
    try:
        offs, ids = device_result(res, q)
        csr = np.diff(offs.cpu().numpy()).astype(np.uint64)
        assert np.array_equal(csr, want_counts), f"{int((csr != want_counts).sum())} CSR slices differ"
        assert verify_all_slices(offs, ids, d_objs, d_boxes, dims, is_rect) == int(want_counts.sum())
        sample = sample_queries(want_counts, nsample)
        so, sids = sample_ids(offs, ids, sample)
    finally:
        res.release()
    want_o, want_i = oracle.ids(objs, dims, is_rect, boxes[sample], threads=THREADS)
    assert_same_hits(so, sids, want_o, want_i)
    return int(want_counts.sum())


def test_batched_16m_clustered_full_batch(qcp, oracle, workloads):
    """16,000,000 points from 64 Gaussians, 10,000 data-centred cubes with
    volumes log-uniform over [1e-6, 1e-2] (about 1.1e9 ids per batch)."""
    w = workloads.config2()
    want = _bvh_counts(w.objs, w.boxes, 3)
    with qcp.Index.build(w.objs, fanout=128) as ix:
        total = _check_index(qcp, oracle, ix, w.objs, w.boxes, 3, False, want, 300)
        # the plain one-query-per-block traversal counts the same
        assert np.array_equal(ix.counts(w.boxes, algo="plain"), want)
    assert total > 500_000_000


@pytest.fixture(scope="module")
def uniform2d64m(workloads):
    w = workloads.config3()
    return w, _bvh_counts(w.objs, w.boxes, 2)


@pytest.mark.parametrize("fanout", [64, 128, 256])
def test_bulk_load_64m_2d_full_batch(qcp, oracle, uniform2d64m, fanout):
    """64,000,000 uniform 2-D points with 32-bit/dim Hilbert keys, 100,000
    squares of area 1e-5.  Hit sets do not depend on the key, so the
    reference's 2-D BVH counts pin them at every fan-out."""
    w, want = uniform2d64m
    with qcp.Index.build(w.objs, fanout=fanout, key_bits=32) as ix:
        info = ix.info()
        assert info["key_bits"] == 32 and info["fanout"] == fanout
        assert info["level_nodes"] == oracle.level_sizes(w.n, fanout)
        _check_index(qcp, oracle, ix, w.objs, w.boxes, 2, False, want, 200)


def test_rectangles_32m_8d_full_batch(qcp, oracle, workloads):
    """32,000,000 8-D rectangles (sides Exp(0.002)), 50,000 boxes with sides
    U[0.05, 0.2]; intersects predicate."""
    w = workloads.config4()
    with qcp.Index.build(w.objs, is_rect=True) as ix:
        want = ix.counts(w.boxes, algo="plain")
        # the sample is checked against the oracle's brute force, so the
        # plain counts used as the yardstick are pinned there too
        total = _check_index(qcp, oracle, ix, w.objs, w.boxes, 8, True, want, 200)
    assert total > 0
