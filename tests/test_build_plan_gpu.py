"""The captured build (qcp_build_plan_*): one graph launch rebuilds the
plan's index from new objects.  Its keys, order and MBRs equal those of
qcp_index_build (and through the oracle's checks of that build, the
oracle's), and its hit lists equal the oracle's.  Needs a GPU."""
from __future__ import annotations

import numpy as np
import pytest

from conftest import assert_same_hits

pytestmark = pytest.mark.gpu


def _same_index(a, b, levels):
    ka, ia, _ = a.export()
    kb, ib, _ = b.export()
    assert np.array_equal(ka, kb) and np.array_equal(ia, ib)
    for l in range(levels):
        assert np.array_equal(a.export(level=l)[2], b.export(level=l)[2])


@pytest.mark.parametrize("dims,is_rect,fanout,key_mode", [(3, False, 128, 0), (2, False, 64, 0),
                                                         (3, False, 256, 1), (8, True, 32, 0)])
def test_plan_builds_equal_direct_builds(qcp, oracle, dims, is_rect, fanout, key_mode):
    rng = np.random.default_rng(dims * 10 + fanout)
    n = 50_000
    with qcp.BuildPlan(n, dims, is_rect=is_rect, fanout=fanout, key_mode=key_mode) as plan:
        for rep in range(3):  # new objects every run, same shape
            lo = rng.random((n, dims), dtype=np.float32)
            objs = (np.ascontiguousarray(np.concatenate([lo, lo + rng.exponential(0.01, (n, dims)).astype(np.float32)],
                                                        1)) if is_rect else lo)
            c = rng.random((60, dims), dtype=np.float32)
            sd = rng.uniform(0.05, 0.4, (60, 1)).astype(np.float32)
            boxes = np.ascontiguousarray(np.concatenate([c - sd, c + sd], 1), dtype=np.float32)
            ix = plan.run(objs)
            with qcp.Index.build(objs, is_rect=is_rect, fanout=fanout, key_mode=key_mode) as ref:
                _same_index(ix, ref, ref.info()["levels"])
            want_offs, want_ids = oracle.ids(objs, dims, is_rect, boxes)
            res = ix.search(boxes)
            assert_same_hits(res.offsets, res.ids, want_offs, want_ids)


def test_plan_input_buffer_and_device_objects(qcp, oracle, workloads):
    import torch
    objs = workloads.gaussian_mixture_points(300_000, 3, seed=5)
    boxes = workloads.data_centred_cubes(objs, 100, 1e-6, 1e-2, seed=6)
    want_offs, want_ids = oracle.ids(objs, 3, False, boxes)
    d = torch.from_numpy(objs).cuda()
    with qcp.BuildPlan(len(objs), 3) as plan:
        res = plan.run(d).search(boxes)  # device objects, copied in
        assert_same_hits(res.offsets, res.ids, want_offs, want_ids)
        # objects written straight into the plan's input buffer
        buf = torch.as_tensor(_View(plan.input_ptr(), objs.size), device="cuda")
        buf.copy_(d.reshape(-1))
        torch.cuda.synchronize()
        res = plan.run(None).search(boxes)
        assert_same_hits(res.offsets, res.ids, want_offs, want_ids)


class _View:
    def __init__(self, ptr, n):
        self.__cuda_array_interface__ = {"shape": (n,), "typestr": "<f4", "data": (ptr, False), "version": 3}


def test_plan_rejects_nonfinite_and_kmeans(qcp):
    objs = np.random.default_rng(1).random((5000, 3), dtype=np.float32)
    with qcp.BuildPlan(5000, 3) as plan:
        bad = objs.copy()
        bad[7, 2] = np.inf
        with pytest.raises(qcp.QcpError) as e:
            plan.run(bad)
        assert e.value.status == 1
        plan.run(objs)  # the next good run works
    with pytest.raises(qcp.QcpError):
        qcp.BuildPlan(5000, 3, key_mode=qcp.KEY_KMEANS)
