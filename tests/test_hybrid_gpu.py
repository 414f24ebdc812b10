"""CPU + GPU co-processing (QCP_ALGO_HYBRID): host threads walk the internal
levels down to a hand-off level, the GPU takes the rest.  Whatever the split
-- hand-off at the leaves' parents, higher up, or at the root (everything on
the GPU) -- and whatever the number of host threads, the per-query sorted ids
must equal the oracle's.  Needs a GPU."""
from __future__ import annotations

import numpy as np
import pytest

from conftest import assert_same_hits

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def clustered(workloads, oracle):
    objs = workloads.gaussian_mixture_points(1_500_000, 3, seed=61)
    boxes = workloads.data_centred_cubes(objs, 700, 1e-7, 1e-3, seed=62)
    o, i = oracle.ids(objs, 3, False, boxes)
    return objs, boxes, o, i


@pytest.mark.parametrize("fanout,handoff,threads", [(128, 1, 0), (128, 2, 4), (128, 3, 1), (64, 2, 3),
                                                    (32, 3, 8), (32, 1, 2)])
def test_hybrid_matches_oracle(qcp, clustered, fanout, handoff, threads):
    objs, boxes, o, i = clustered
    with qcp.Index.build(objs, fanout=fanout) as ix:
        assert ix.info()["levels"] >= 3
        res = ix.search(boxes, algo="hybrid", handoff_level=handoff, cpu_threads=threads)
        assert_same_hits(res.offsets, res.ids, o, i)
        counts = ix.counts(boxes, algo="hybrid")
        assert np.array_equal(counts, np.diff(o))


def test_hybrid_device_boxes_and_rectangles(qcp, oracle):
    import torch
    rng = np.random.default_rng(63)
    lo = rng.random((300_000, 8), dtype=np.float32)
    hi = (lo + rng.exponential(0.02, (300_000, 8)).astype(np.float32)).astype(np.float32)
    objs = np.ascontiguousarray(np.concatenate([lo, hi], 1))
    c = rng.random((200, 8), dtype=np.float32)
    s = rng.uniform(0.2, 0.5, (200, 8)).astype(np.float32) / 2
    boxes = np.ascontiguousarray(np.concatenate([c - s, c + s], 1))
    o, i = oracle.ids(objs, 8, True, boxes)
    with qcp.Index.build(objs, is_rect=True, fanout=64) as ix:
        d = torch.from_numpy(boxes).cuda()
        res = ix.search(d, q=len(boxes), algo="hybrid", handoff_level=1)
        assert_same_hits(res.offsets, res.ids, o, i)
