"""k-means-clustered keys (QCP_KEY_KMEANS): the device build must give
exactly the keys and the order of the oracle's restatement of the
clustering, and the hit sets must stay the oracle's.  Needs a GPU."""
from __future__ import annotations

import numpy as np
import pytest

from conftest import assert_same_hits

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("dims,is_rect,bits,K,iters", [(3, False, 21, 64, 8), (2, False, 32, 37, 5),
                                                       (8, True, 8, 16, 4)])
def test_kmeans_keys_match_restatement(qcp, oracle, workloads, dims, is_rect, bits, K, iters):
    rng = np.random.default_rng(70 + dims)
    if is_rect:
        lo = rng.random((20_000, dims), dtype=np.float32)
        hi = (lo + rng.exponential(0.01, (20_000, dims)).astype(np.float32)).astype(np.float32)
        objs = np.ascontiguousarray(np.concatenate([lo, hi], 1))
    else:
        objs = workloads.gaussian_mixture_points(30_000, dims, clusters=12, seed=71)
    want = oracle.kmeans_keys(objs, dims, is_rect, bits, K, iters)
    order = oracle.sort_perm(want)
    with qcp.Index.build(objs, is_rect=is_rect, key_mode=qcp.KEY_KMEANS, key_bits=bits,
                         kmeans_clusters=K, kmeans_iters=iters, fanout=64) as ix:
        keys, perm, _ = ix.export()
        assert np.array_equal(keys, want[order])
        assert np.array_equal(perm, order.astype(np.int32))
        c = rng.random((100, dims), dtype=np.float32)
        s = rng.uniform(0.05, 0.3, (100, dims)).astype(np.float32) / 2
        boxes = np.ascontiguousarray(np.concatenate([c - s, c + s], 1))
        res = ix.search(boxes)
        o, i = oracle.ids(objs, dims, is_rect, boxes)
        assert_same_hits(res.offsets, res.ids, o, i)


def test_kmeans_keys_are_cluster_major(qcp, workloads):
    objs = workloads.gaussian_mixture_points(50_000, 3, clusters=8, seed=72)
    with qcp.Index.build(objs, key_mode=qcp.KEY_KMEANS, kmeans_clusters=8, kmeans_iters=20) as ix:
        keys, _, _ = ix.export()
        rank = keys >> np.uint64(61)  # 3 rank bits for 8 clusters
        assert np.all(np.diff(rank.astype(np.int64)) >= 0)
        assert len(np.unique(rank)) == 8
