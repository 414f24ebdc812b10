"""Parity of the CUDA path with the oracle (and through it with the
reference's own counts), called through the C ABI.  Needs a GPU.

Bar: per-query sorted id lists bit-exact (integer/index output of FP32
closed-interval compares, no tolerance)."""
from __future__ import annotations

import numpy as np
import pytest

from conftest import assert_same_hits, golden

pytestmark = pytest.mark.gpu

CASES = ["u3", "g3", "small3", "ragged3", "dup3", "u2", "p8"]


@pytest.mark.parametrize("name", CASES)
@pytest.mark.parametrize("algo", ["batched", "plain"])
def test_golden_cases_exact(qcp, oracle, cases, name, algo):
    objs, boxes, dims = cases.COUNT_CASES[name]()
    ref_counts = golden(f"counts_{name}.npz")["counts"].astype(np.uint64)
    want_offs, want_ids = oracle.ids(objs, dims, False, boxes)
    assert np.array_equal(np.diff(want_offs), ref_counts)
    with qcp.Index.build(objs) as ix:
        res = ix.search(boxes, algo=algo)
        assert_same_hits(res.offsets, res.ids, want_offs, want_ids, boxes)
        assert res.total_hits == int(ref_counts.sum())
        assert np.array_equal(ix.counts(boxes, algo=algo), ref_counts)


@pytest.mark.parametrize("fanout", [32, 64, 128, 192, 256])
def test_fanouts(qcp, oracle, cases, fanout):
    objs, boxes, dims = cases.COUNT_CASES["g3"]()
    want_offs, want_ids = oracle.ids(objs, dims, False, boxes)
    with qcp.Index.build(objs, fanout=fanout) as ix:
        info = ix.info()
        assert info["level_nodes"] == oracle.level_sizes(len(objs), fanout)
        for algo in ["batched", "plain"]:
            res = ix.search(boxes, algo=algo)
            assert_same_hits(res.offsets, res.ids, want_offs, want_ids, boxes)


@pytest.mark.parametrize("n", [1, 2, 31, 32, 33, 127, 128, 129, 4095, 16384, 16385])
def test_small_and_ragged_sizes(qcp, oracle, n):
    rng = np.random.default_rng(n)
    objs = rng.random((n, 3), dtype=np.float32)
    c = rng.random((50, 3), dtype=np.float32)
    s = rng.uniform(0.05, 0.8, (50, 1)).astype(np.float32)
    boxes = np.concatenate([c - s / 2, c + s / 2], 1).astype(np.float32)
    boxes = np.concatenate([boxes, np.array([[-1, -1, -1, 2, 2, 2], [2, 2, 2, 3, 3, 3]], np.float32)])
    want_offs, want_ids = oracle.ids(objs, 3, False, boxes)
    with qcp.Index.build(objs, fanout=32) as ix:
        for algo in ["batched", "plain"]:
            res = ix.search(boxes, algo=algo)
            assert_same_hits(res.offsets, res.ids, want_offs, want_ids, boxes)


def test_empty_query_batch(qcp, cases):
    objs, _, _ = cases.COUNT_CASES["u3"]()
    with qcp.Index.build(objs) as ix:
        res = ix.search(np.zeros((0, 6), np.float32))
        assert res.total_hits == 0 and len(res.offsets) == 1


def test_config1_exact(qcp, oracle, workloads):
    """1 M uniform points, 1 000 cubes of side 0.0464 (~100 hits each)."""
    w = workloads.config1()
    want_offs, want_ids = oracle.ids(w.objs, 3, False, w.boxes, threads=16)
    with qcp.Index.build(w.objs, fanout=w.fanout) as ix:
        for algo in ["batched", "plain"]:
            res = ix.search(w.boxes, algo=algo)
            assert_same_hits(res.offsets, res.ids, want_offs, want_ids)


def test_unsorted_gives_same_sets(qcp, oracle, cases):
    objs, boxes, dims = cases.COUNT_CASES["g3"]()
    want_offs, want_ids = oracle.ids(objs, dims, False, boxes)
    with qcp.Index.build(objs) as ix:
        res = ix.search(boxes, sort=False)
        assert np.array_equal(res.offsets, want_offs)
        for i in range(len(boxes)):
            assert np.array_equal(np.sort(res.hits(i)), want_ids[want_offs[i]:want_offs[i + 1]])


class _DeviceArray:
    """A non-owning view of library-owned device memory for torch.as_tensor."""

    def __init__(self, ptr: int, n: int, typestr: str):
        self.__cuda_array_interface__ = {"shape": (n,), "typestr": typestr, "data": (int(ptr), False),
                                         "version": 3}


def test_device_buffers_in_and_out(qcp, oracle, cases):
    import torch
    objs, boxes, dims = cases.COUNT_CASES["g3"]()
    want_offs, want_ids = oracle.ids(objs, dims, False, boxes)
    d_objs = torch.from_numpy(objs).cuda()
    d_boxes = torch.from_numpy(boxes).cuda()
    with qcp.Index.build(d_objs, dims=3, n=len(objs)) as ix:
        r = ix.search(d_boxes, q=len(boxes), result_mem=qcp.MEM_DEVICE)
        try:
            offs = torch.as_tensor(_DeviceArray(r.offsets, len(boxes) + 1, "<u8"), device="cuda")
            offs = offs.cpu().numpy().astype(np.uint64)
            ids = torch.as_tensor(_DeviceArray(r.ids, r.total_hits, "<i4"), device="cuda").cpu().numpy()
        finally:
            r.release()
        assert_same_hits(offs, ids, want_offs, want_ids)


def test_ref_key_mode_matches_oracle_keys(qcp, oracle, cases):
    objs, boxes, dims = cases.COUNT_CASES["dup3"]()
    with qcp.Index.build(objs, key_mode=qcp.KEY_REF) as ix:
        keys, perm, _ = ix.export()
        want_keys = oracle.hilbert_keys(objs, 3, False, 20, 0)
        order = oracle.sort_perm(want_keys)
        assert np.array_equal(perm, order.astype(np.int32))       # stable order
        assert np.array_equal(keys, want_keys[order])
        res = ix.search(boxes)
        want_offs, want_ids = oracle.ids(objs, dims, False, boxes)
        assert_same_hits(res.offsets, res.ids, want_offs, want_ids)


@pytest.mark.parametrize("dims,bits", [(2, 32), (3, 21), (8, 8)])
def test_norm_keys_and_mbrs_match_oracle(qcp, oracle, dims, bits):
    rng = np.random.default_rng(dims)
    objs = rng.random((30000, dims), dtype=np.float32)
    with qcp.Index.build(objs, fanout=64) as ix:
        keys, perm, _ = ix.export()
        want = oracle.hilbert_keys(objs, dims, False, bits, 1)
        order = oracle.sort_perm(want)
        assert np.array_equal(perm, order.astype(np.int32))
        assert np.array_equal(keys, want[order])
        levels = oracle.node_mbrs(objs[order], dims, False, 64)
        for l, want_mbr in enumerate(levels):
            _, _, mbr = ix.export(level=l)
            assert np.array_equal(mbr, want_mbr)


def test_rectangles_8d(qcp, oracle):
    rng = np.random.default_rng(8)
    lo = rng.random((20000, 8), dtype=np.float32)
    hi = (lo + rng.exponential(0.05, (20000, 8)).astype(np.float32)).astype(np.float32)
    objs = np.ascontiguousarray(np.concatenate([lo, hi], 1))
    c = rng.random((100, 8), dtype=np.float32)
    s = rng.uniform(0.3, 0.7, (100, 8)).astype(np.float32) / 2
    boxes = np.concatenate([c - s, c + s], 1).astype(np.float32)
    want_offs, want_ids = oracle.ids(objs, 8, True, boxes)
    with qcp.Index.build(objs, is_rect=True) as ix:
        for algo in ["batched", "plain"]:
            res = ix.search(boxes, algo=algo)
            assert_same_hits(res.offsets, res.ids, want_offs, want_ids)


def test_save_load_roundtrip(qcp, cases, tmp_path):
    objs, boxes, dims = cases.COUNT_CASES["u3"]()
    with qcp.Index.build(objs) as ix:
        a = ix.search(boxes)
        ix.save(tmp_path / "ix.qcp")
    with qcp.Index.load(tmp_path / "ix.qcp") as ix2:
        b = ix2.search(boxes)
    assert np.array_equal(a.offsets, b.offsets) and np.array_equal(a.ids, b.ids)


def test_nonfinite_objects_rejected(qcp):
    objs = np.random.default_rng(0).random((1000, 3), dtype=np.float32)
    objs[10, 1] = np.nan
    with pytest.raises(qcp.QcpError) as e:
        qcp.Index.build(objs)
    assert e.value.status == 1


def test_repeated_calls_reuse_buffers(qcp, oracle, cases):
    objs, boxes, dims = cases.COUNT_CASES["g3"]()
    want_offs, want_ids = oracle.ids(objs, dims, False, boxes)
    with qcp.Index.build(objs) as ix:
        for k in range(3):
            sub = boxes[k::3]
            res = ix.search(sub)
            o, i = oracle.ids(objs, dims, False, sub)
            assert_same_hits(res.offsets, res.ids, o, i)
        res = ix.search(boxes)
        assert_same_hits(res.offsets, res.ids, want_offs, want_ids)


@pytest.mark.parametrize("n", [300_000, 2_000_000])
def test_large_result_slices(qcp, oracle, workloads, n):
    """Slices far above the shared-memory sort size: one id window (n <= 2^19)
    and many windows (n > 2^19), dense and sparse windows."""
    pts = workloads.gaussian_mixture_points(n, 3, seed=99)
    boxes = workloads.data_centred_cubes(pts, 40, 1e-5, 3e-2, seed=98)
    boxes = np.concatenate([boxes, np.array([[-1, -1, -1, 2, 2, 2]], np.float32)])  # everything
    want_offs, want_ids = oracle.ids(pts, 3, False, boxes, threads=16)
    assert np.diff(want_offs).max() > 100_000
    with qcp.Index.build(pts) as ix:
        for algo in ["batched", "plain"]:
            res = ix.search(boxes, algo=algo)
            assert_same_hits(res.offsets, res.ids, want_offs, want_ids)


def test_slice_sizes_at_every_sort_boundary(qcp, oracle):
    """Slices of exactly k ids around the sort's size classes: one warp per
    slice up to 1,024 ids, one CTA up to 8,192, id windows above.  Points
    sit on a line in random id order, so a box [x0, x1] selects an exact,
    randomly numbered run of them."""
    n = 200_000
    rng = np.random.default_rng(1024)
    order = rng.permutation(n)
    objs = np.zeros((n, 3), np.float32)
    objs[order, 0] = ((np.arange(n) + 0.5) / n).astype(np.float32)
    objs[:, 1:] = 0.5
    sizes = [1, 2, 31, 32, 33, 255, 256, 257, 1023, 1024, 1025, 4096, 8191, 8192, 8193, 20000, 131073]
    boxes = []
    for k in sizes:
        start = int(rng.integers(0, n - k))
        lo = np.float32((start + 0.25) / n)
        hi = np.float32((start + k - 0.25) / n)
        boxes.append([lo, 0.4, 0.4, hi, 0.6, 0.6])
    boxes = np.asarray(boxes * 3, np.float32)  # every size three times in one batch
    want_offs, want_ids = oracle.ids(objs, 3, False, boxes)
    assert list(np.diff(want_offs)[:len(sizes)]) == sizes
    with qcp.Index.build(objs) as ix:
        for algo in ["batched", "plain"]:
            res = ix.search(boxes, algo=algo)
            assert_same_hits(res.offsets, res.ids, want_offs, want_ids, boxes)


def test_window_sizes_at_the_one_warp_boundary(qcp, oracle):
    """Slices of more than 8,192 ids whose 2^17-id windows hold exactly 512
    and 513 ids (one warp each up to 512, the bitmap above), 1, 2, 511,
    8,000 and 9,000 ids and none: 2^19 points, so ids [w * 2^17, (w+1) * 2^17)
    form window w, and two boxes each select chosen ids of every window."""
    W = 1 << 17
    n = 4 * W
    rng = np.random.default_rng(512)
    per_box = {0: [512, 513, 8000, 1], 1: [0, 2, 9000, 511]}
    objs = np.zeros((n, 3), np.float32)
    objs[:, 0] = rng.uniform(0.6, 0.95, n)  # outside both boxes
    objs[:, 1:] = rng.uniform(0.05, 0.45, (n, 2))
    free = [rng.permutation(np.arange(w * W, (w + 1) * W)) for w in range(4)]
    used = [0, 0, 0, 0]
    for b, sizes in per_box.items():
        x0 = 0.05 if b == 0 else 0.30
        for w, k in enumerate(sizes):
            sel = free[w][used[w]:used[w] + k]
            used[w] += k
            objs[sel, 0] = rng.uniform(x0, x0 + 0.15, k)
    boxes = np.asarray([[0.0, 0.0, 0.0, 0.25, 0.5, 0.5], [0.275, 0.0, 0.0, 0.5, 0.5, 0.5]], np.float32)
    want_offs, want_ids = oracle.ids(objs, 3, False, boxes)
    for b, sizes in per_box.items():
        ids = np.asarray(want_ids[int(want_offs[b]):int(want_offs[b + 1])], np.int64)
        assert list(np.bincount(ids >> 17, minlength=4)) == sizes
    with qcp.Index.build(objs) as ix:
        for algo in ["batched", "plain"]:
            res = ix.search(boxes, algo=algo, win_bits=17)
            assert_same_hits(res.offsets, res.ids, want_offs, want_ids, boxes)


def test_hit_cache_overflow_then_full(qcp, oracle, workloads):
    """The write pass replays the count pass's leaf masks and hit bits.  The
    first call on a fresh index has room for 2^20 words of hit bits; this
    batch needs more (about 300,000 partially covered leaves), so part of its
    groups are tested again by the write pass; the second call has room for
    all.  Both must equal the oracle, sorted and unsorted."""
    pts = workloads.uniform_points(2_000_000, 3, seed=23)
    boxes = workloads.fixed_cubes(3000, 3, 0.16, seed=24)
    want_offs, want_ids = oracle.ids(pts, 3, False, boxes, threads=16)
    with qcp.Index.build(pts) as ix:
        for _ in range(2):
            res = ix.search(boxes)
            assert_same_hits(res.offsets, res.ids, want_offs, want_ids)
        res = ix.search(boxes, sort=False)
        assert np.array_equal(res.offsets, want_offs)
        for i in range(0, len(boxes), 97):
            assert np.array_equal(np.sort(res.hits(i)), want_ids[want_offs[i]:want_offs[i + 1]])
