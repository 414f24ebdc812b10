"""Autotuner (qcp_autotune) and the query knobs it sets.

The knobs change how the work is laid out on the GPU, never the result: a
search with any blocks_per_sm / win_bits must return the oracle's ids.  The
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


@pytest.mark.parametrize("bps,wb", [(4, 16), (16, 17), (32, 12), (1, 18)])
def test_knobs_keep_hits_exact(qcp, data, bps, wb):
    objs, boxes, want_offs, want_ids = data
    with qcp.Index.build(objs, fanout=64) as ix:
        res = ix.search(boxes, blocks_per_sm=bps, win_bits=wb)
        assert_same_hits(res.offsets, res.ids, want_offs, want_ids)


def test_autotune_choice_and_trials(qcp, data):
    objs, boxes, want_offs, want_ids = data
    r = qcp.autotune(objs, boxes, repeats=2)
    assert r["fanout"] in (64, 128, 256)
    assert r["blocks_per_sm"] in (4, 8, 16)
    assert r["win_bits"] in (16, 17, 18)
    assert len(r["trials"]) == 7  # 3 fan-outs, 2 more grids, 2 more windows
    assert r["best_ms"] == pytest.approx(min(t["ms"] for t in r["trials"]))
    chosen = [t for t in r["trials"] if t["ms"] == r["best_ms"]][0]
    assert (chosen["fanout"], chosen["blocks_per_sm"], chosen["win_bits"]) == \
        (r["fanout"], r["blocks_per_sm"], r["win_bits"])
    with qcp.Index.build(objs, fanout=r["fanout"]) as ix:
        res = ix.search(boxes, blocks_per_sm=r["blocks_per_sm"], win_bits=r["win_bits"])
        assert_same_hits(res.offsets, res.ids, want_offs, want_ids)
