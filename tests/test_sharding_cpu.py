"""Query sharding across ranks and the host-side gather, on CPU with two
gloo ranks (no GPU)."""
from __future__ import annotations

import os
import socket

import numpy as np
import pytest
import torch.distributed as dist
import torch.multiprocessing as mp

from conftest import load_pkg


def test_query_shard_covers_batch_once():
    sh = load_pkg()
    import qcp_b200.sharding as S
    for total in [0, 1, 7, 10_000, 10_001]:
        for world in [1, 2, 3, 8]:
            seen = []
            for r in range(world):
                a, b = S.query_shard(total, r, world)
                seen.extend(range(a, b))
                assert abs((b - a) - total / world) <= 1
            assert seen == list(range(total))
    del sh


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _worker(rank, world, port, q, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        load_pkg()
        import qcp_b200.sharding as S
        rng = np.random.default_rng(5)
        counts = rng.integers(0, 20, size=q)
        full_offs = np.concatenate([[0], np.cumsum(counts)]).astype(np.uint64)
        full_ids = rng.integers(0, 1000, size=int(full_offs[-1])).astype(np.int32)
        a, b = S.query_shard(q, rank, world)
        offs = full_offs[a:b + 1] - full_offs[a]
        ids = full_ids[full_offs[a]:full_offs[b]]
        g_offs, g_ids = S.gather_hit_lists(offs, ids)
        # the per-step time of a rank is reduced with MAX, as bench.py does
        import torch
        t = torch.tensor([float(rank + 1)], dtype=torch.float64)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        ok = np.array_equal(g_offs, full_offs) and np.array_equal(g_ids, full_ids) and t.item() == world
        out[rank] = 1 if ok else 0
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("world", [2])
def test_gather_over_gloo_ranks(world):
    ctx = mp.get_context("spawn")
    out = ctx.Array("i", [0] * world)
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, world, port, 101, out)) for r in range(world)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=120)
        assert p.exitcode == 0
    assert list(out) == [1] * world
