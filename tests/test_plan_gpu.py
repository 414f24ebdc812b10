"""Query plans (qcp_plan_*): the batched pipeline captured once into a CUDA
graph and replayed.  Every replay must return exactly what qcp_query_batch
returns for the same boxes -- for batches smaller than the plan (padded with
empty boxes), for repeated and alternating batches, for device-resident
boxes, sorted and unsorted -- and a batch beyond the plan's capacity must be
reported, not truncated, leaving the plan usable.  Needs a GPU."""
from __future__ import annotations

import numpy as np
import pytest

from conftest import assert_same_hits

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def setup(qcp, workloads):
    objs = workloads.gaussian_mixture_points(2_000_000, 3, seed=41)
    batches = [np.ascontiguousarray(workloads.data_centred_cubes(objs, n, 1e-6, 1e-2, seed=50 + k))
               for k, n in enumerate([600, 257, 1, 600])]
    ix = qcp.Index.build(objs)
    yield qcp, ix, objs, batches
    ix.close()


def test_plan_replays_match_query_batch(setup, oracle):
    qcp, ix, objs, batches = setup
    want = [ix.search(b) for b in batches]
    with qcp.Plan(ix, 600, 60_000_000) as plan:
        for rnd in range(2):
            for k, b in enumerate(batches):
                offs, ids = plan.run(b)
                assert np.array_equal(offs, want[k].offsets), f"batch {k} round {rnd}"
                assert np.array_equal(ids, want[k].ids), f"batch {k} round {rnd}"
    o, i = oracle.ids(objs, 3, False, batches[1])
    assert_same_hits(want[1].offsets, want[1].ids, o, i)


def test_plan_device_boxes_and_unsorted(setup):
    import torch
    qcp, ix, objs, batches = setup
    b = batches[0]
    want = ix.search(b)
    with qcp.Plan(ix, 600, 60_000_000, sort=False, blocks_per_sm=4, win_bits=16) as plan:
        d = torch.from_numpy(b).cuda()
        offs, ids = plan.run(d, q=b.shape[0])
    assert np.array_equal(offs, want.offsets)
    for k in range(b.shape[0]):
        s = np.sort(ids[offs[k]:offs[k + 1]])
        assert np.array_equal(s, want.ids[want.offsets[k]:want.offsets[k + 1]]), f"query {k}"


def test_plan_overflow_is_reported_and_plan_stays_usable(setup):
    qcp, ix, objs, batches = setup
    big = batches[0]
    counts = ix.counts(big)
    small = big[counts <= 50][:20]
    assert len(small) > 0 and counts.sum() > 5000
    with qcp.Plan(ix, 600, 5000) as plan:
        with pytest.raises(qcp.QcpError) as e:
            plan.run(big)
        assert e.value.status == 3  # QCP_ERR_OUTPUT_OVERFLOW
        offs, ids = plan.run(small)
        want = ix.search(small)
        assert np.array_equal(offs, want.offsets) and np.array_equal(ids, want.ids)
    with pytest.raises(qcp.QcpError):
        qcp.Plan(ix, 600, 5000).run_device(np.zeros((601, 6), np.float32))


@pytest.mark.parametrize("wb", [16, 17])
def test_plan_sorted_at_smaller_windows(setup, wb):
    """Sorted plans at 2^16 / 2^17-id sort windows (their own window-sort
    instantiations) return what qcp_query_batch returns."""
    qcp, ix, objs, batches = setup
    b = batches[0]
    want = ix.search(b)
    with qcp.Plan(ix, 600, 60_000_000, win_bits=wb) as plan:
        offs, ids = plan.run(b)
    assert np.array_equal(offs, want.offsets) and np.array_equal(ids, want.ids)
