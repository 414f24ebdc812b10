"""Serving loop (qcp_serve_replay): continuous batching of an open-loop
arrival trace over one resident index.

Every served request must return exactly the ids it returns when it is
queried alone, and exactly the oracle's ids, whatever batch it shared with
other requests and whatever overlapped it on the device.  The admission cap
on result bytes must hold (a request larger than the cap runs alone).
Needs a GPU."""
from __future__ import annotations

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _mixed_trace(workloads, objs, n_req, rate, seed):
    """Arrival times and boxes of the serving mix (volumes 1e-7 / 1e-5 / 1e-3
    at 70 / 25 / 5 %, centred on data points), n_req requests."""
    t, boxes, cls = workloads.serving_stream(objs, rate=rate, duration_s=n_req / rate, seed=seed)
    return t[:n_req], np.ascontiguousarray(boxes[:n_req]), cls[:n_req]


@pytest.fixture(scope="module")
def served(qcp, workloads, oracle):
    objs = workloads.gaussian_mixture_points(300_000, 3, seed=21)
    t, boxes, cls = _mixed_trace(workloads, objs, 4000, 40_000.0, seed=5)
    want_offs, want_ids = oracle.ids(objs, 3, False, boxes)
    ix = qcp.Index.build(objs)
    yield ix, objs, t, boxes, cls, want_offs, want_ids
    ix.close()


def _check_all(got, want_offs, want_ids):
    for i, ids in enumerate(got):
        assert ids is not None, f"request {i} not delivered"
        want = want_ids[int(want_offs[i]):int(want_offs[i + 1])]
        assert np.array_equal(ids, want), f"request {i}"


def test_served_results_equal_oracle_and_alone(served):
    ix, objs, t, boxes, cls, want_offs, want_ids = served
    stats, lat, got = ix.serve(boxes, t, streams=4, max_batch=256, collect=True)
    assert stats["requests"] == len(boxes)
    assert stats["hits"] == int(want_offs[-1])
    assert stats["batches"] >= len(boxes) // 256
    _check_all(got, want_offs, want_ids)
    # the same requests queried one at a time
    rng = np.random.default_rng(3)
    for i in rng.choice(len(boxes), 40, replace=False):
        alone = ix.search(boxes[i:i + 1])
        assert np.array_equal(alone.hits(0), got[i]), f"request {i} alone vs in the mix"
    assert np.all(lat >= 0) and stats["p50_ms"] <= stats["p99_ms"] <= stats["max_ms"]
    assert stats["max_inflight"] >= 1


def test_admission_cap_on_result_bytes(served):
    ix, objs, t, boxes, cls, want_offs, want_ids = served
    counts = np.diff(want_offs).astype(np.int64)
    largest = int(counts.max()) * 4 + 16  # bytes of the largest request alone
    cap = max(4096, largest // 2)
    stats, lat, got = ix.serve(boxes, t, streams=3, max_batch=1024, output_cap_bytes=cap, collect=True)
    _check_all(got, want_offs, want_ids)
    # batches stay under the cap; the requests above it ran alone
    assert stats["max_output_bytes"] <= max(cap, largest)
    assert largest > cap


def test_serving_trace_records_every_run(served):
    ix, objs, t, boxes, cls, want_offs, want_ids = served
    stats, lat, _ = ix.serve(boxes, t, streams=3, max_batch=300, trace=100_000)
    tr = stats["trace"]
    assert len(tr) == stats["batches"]
    assert int(tr["requests"].sum()) == len(boxes)
    assert int(tr["hits"].sum()) == int(want_offs[-1])
    assert set(np.unique(tr["worker"])) <= {0, 1, 2}
    assert set(np.unique(tr["path"])) <= {0, 1, 2}
    assert np.all(tr["requests"][tr["path"] == 0] <= 256)
    for a, b in [("t_taken", "t_start"), ("t_start", "t_run"), ("t_run", "t_admitted"), ("t_admitted", "t_done")]:
        assert np.all(tr[a] <= tr[b]), (a, b)
    # a request's latency ends at its run's t_done
    assert float(lat.max()) <= (float(tr["t_done"].max()) - float(t[0])) * 1e3 + 1.0
    # a short trace keeps the first records and says how many runs there were
    stats2, _, _ = ix.serve(boxes[:500], t[:500], streams=2, trace=3)
    assert len(stats2["trace"]) == min(3, stats2["batches"])


def test_serving_rejects_bad_trace(qcp, served):
    ix, objs, t, boxes, *_ = served
    bad = t[:10].copy()
    bad[5] = bad[4] - 1e-3
    with pytest.raises(qcp.QcpError):
        ix.serve(boxes[:10], bad)


def test_concurrent_calls_on_streams_match(qcp, workloads):
    """Several host threads query one index at once, each on its own CUDA
    stream; every result equals the same batch run alone."""
    import concurrent.futures as cf
    import torch
    objs = workloads.gaussian_mixture_points(2_000_000, 3, seed=22)
    rng = np.random.default_rng(9)
    batches = [np.ascontiguousarray(workloads.data_centred_cubes(objs, 600, 1e-6, 1e-2, seed=100 + k))
               for k in range(12)]
    with qcp.Index.build(objs) as ix:
        want = [ix.search(b) for b in batches]
        streams = [torch.cuda.Stream() for _ in range(4)]

        def run(k):
            st = streams[k % 4]
            return ix.search(batches[k], stream=st.cuda_stream)

        for _ in range(3):
            order = rng.permutation(len(batches))
            with cf.ThreadPoolExecutor(4) as ex:
                got = dict(zip(order, ex.map(run, order)))
            for k in range(len(batches)):
                assert np.array_equal(got[k].offsets, want[k].offsets), f"batch {k} offsets"
                assert np.array_equal(got[k].ids, want[k].ids), f"batch {k} ids"
