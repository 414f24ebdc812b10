"""Autotuner (qcp_autotune) and the query knobs it sets.

The knobs change how the work is laid out on the GPU, never the result: a
search with any blocks_per_sm / win_bits / leaf_prefetch must return the
oracle's ids.  The
tuner must pick from its candidate sets, record every trial, and report the
time of the trial it chose.  Needs a GPU."""
from __future__ import annotations

import numpy as np
import pytest

from conftest import assert_same_hits

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def data(workloads, oracle):
    objs = workloads.gaussian_mixture_points(2_000_000, 3, seed=31)
    boxes = workloads.data_centred_cubes(objs, 400, 1e-6, 1e-2, seed=32)
    want_offs, want_ids = oracle.ids(objs, 3, False, boxes)
    return objs, boxes, want_offs, want_ids


@pytest.mark.parametrize("bps,wb,lp,lpi", [(4, 16, 1, 32), (16, 17, 2, 16), (32, 12, 3, 8), (1, 18, 4, 16),
                                          (8, 17, 1, 8), (8, 16, 3, 32)])
def test_knobs_keep_hits_exact(qcp, data, bps, wb, lp, lpi):
    objs, boxes, want_offs, want_ids = data
    with qcp.Index.build(objs, fanout=64) as ix:
        res = ix.search(boxes, blocks_per_sm=bps, win_bits=wb, leaf_prefetch=lp, lanes_per_item=lpi)
        assert_same_hits(res.offsets, res.ids, want_offs, want_ids)
        res = ix.search(boxes, blocks_per_sm=bps, win_bits=wb, leaf_prefetch=lp, lanes_per_item=lpi, hit_cache=1)
        assert_same_hits(res.offsets, res.ids, want_offs, want_ids)
        assert np.array_equal(ix.counts(boxes, leaf_prefetch=lp, lanes_per_item=lpi), np.diff(want_offs))


@pytest.mark.parametrize("lpi", [8, 16, 32])
@pytest.mark.parametrize("fanout", [32, 96, 256])
def test_lanes_per_item_at_every_fanout(qcp, data, lpi, fanout):
    """Two or four (query, node) items per warp in the level expansion, at
    fan-outs that are and are not multiples of the group width."""
    objs, boxes, want_offs, want_ids = data
    with qcp.Index.build(objs, fanout=fanout) as ix:
        res = ix.search(boxes[:200], lanes_per_item=lpi)
        n = int(want_offs[200])
        assert_same_hits(res.offsets, res.ids, want_offs[:201], want_ids[:n])


@pytest.mark.parametrize("fanout", [32, 128, 256])
@pytest.mark.parametrize("lp", [1, 2, 4])
def test_leaf_tile_at_every_fanout(qcp, data, fanout, lp):
    """The leaf prefetch ring (bulk copies of partially covered leaves into
    shared memory) against direct loads, at fan-outs whose leaves are 128 B
    to 1 KB per coordinate run."""
    objs, boxes, want_offs, want_ids = data
    with qcp.Index.build(objs, fanout=fanout) as ix:
        res = ix.search(boxes[:150], leaf_prefetch=lp)
        n = int(want_offs[150])
        assert_same_hits(res.offsets, res.ids, want_offs[:151], want_ids[:n])


@pytest.mark.parametrize("lp", [1, 2, 3])
def test_leaf_tile_rectangles_and_2d(qcp, oracle, cases, lp):
    """Rectangles (lo and hi runs per leaf) and 2-D points through the ring."""
    rng = np.random.default_rng(81)
    lo = rng.random((40000, 8), dtype=np.float32)
    hi = (lo + rng.exponential(0.05, (40000, 8)).astype(np.float32)).astype(np.float32)
    objs = np.ascontiguousarray(np.concatenate([lo, hi], 1))
    c = rng.random((120, 8), dtype=np.float32)
    sd = rng.uniform(0.3, 0.7, (120, 8)).astype(np.float32) / 2
    boxes = np.ascontiguousarray(np.concatenate([c - sd, c + sd], 1), dtype=np.float32)
    want_offs, want_ids = oracle.ids(objs, 8, True, boxes)
    for fanout in (32, 64):
        with qcp.Index.build(objs, is_rect=True, fanout=fanout) as ix:
            res = ix.search(boxes, leaf_prefetch=lp)
            assert_same_hits(res.offsets, res.ids, want_offs, want_ids)
    objs2, boxes2, _ = cases.COUNT_CASES["u2"]()
    o2, i2 = oracle.ids(objs2, 2, False, boxes2)
    with qcp.Index.build(objs2) as ix:
        res = ix.search(boxes2, leaf_prefetch=lp)
        assert_same_hits(res.offsets, res.ids, o2, i2)


def test_autotune_choice_and_trials(qcp, data):
    objs, boxes, want_offs, want_ids = data
    r = qcp.autotune(objs, boxes, repeats=2)
    assert r["fanout"] in (64, 128, 256)
    assert r["blocks_per_sm"] in (4, 8, 16)
    assert r["win_bits"] in (16, 17, 18)
    assert r["leaf_prefetch"] in (1, 2, 3)
    assert r["lanes_per_item"] in (8, 16, 32)
    assert r["hit_cache"] in (0, 1)
    # 3 fan-outs, 2 more grids, 2 more windows, 2 more leaf tiles, 2 more lane widths, the cache off
    assert len(r["trials"]) == 12
    assert r["best_ms"] == pytest.approx(min(t["ms"] for t in r["trials"]))
    chosen = [t for t in r["trials"] if t["ms"] == r["best_ms"]][0]
    keys = ("fanout", "blocks_per_sm", "win_bits", "leaf_prefetch", "lanes_per_item", "hit_cache")
    assert tuple(chosen[k] for k in keys) == tuple(r[k] for k in keys)
    with qcp.Index.build(objs, fanout=r["fanout"]) as ix:
        res = ix.search(boxes, blocks_per_sm=r["blocks_per_sm"], win_bits=r["win_bits"],
                        leaf_prefetch=r["leaf_prefetch"], lanes_per_item=r["lanes_per_item"], hit_cache=r["hit_cache"])
        assert_same_hits(res.offsets, res.ids, want_offs, want_ids)
