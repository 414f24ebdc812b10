"""The CPU oracle, pinned against golden vectors produced by the reference
itself (tests/golden/make_golden.py), plus the oracle's own invariants.
CPU only."""
from __future__ import annotations

import hashlib

import numpy as np
import pytest

from conftest import golden


def _digest(*arrays) -> str:
    h = hashlib.sha256()
    for a in arrays:
        h.update(np.ascontiguousarray(a).tobytes())
    return h.hexdigest()


@pytest.mark.parametrize("dims,bits", [(3, 20), (2, 31)])
def test_hilbert_keys_match_reference(oracle, dims, bits):
    g = golden("hilbert_kat.npz")
    pts = g[f"pts_d{dims}"]
    want = g[f"keys_d{dims}_b{bits}"].astype(np.uint64)
    got = oracle.hilbert_keys(pts, dims, False, bits, 0)
    assert np.array_equal(got, want)


def test_hilbert_known_answers(oracle):
    # values printed by the reference's MappingIntoSingle for these points
    got3 = oracle.hilbert_keys(np.array([[0.5, 0.25, 0.75]], np.float32), 3, False, 20, 0)
    got2 = oracle.hilbert_keys(np.array([[0.5, 0.25]], np.float32), 2, False, 31, 0)
    assert int(got3[0]) == 1070030857132072960
    assert int(got2[0]) == 114739604736


def test_hilbert_is_a_bijection_on_small_grid(oracle):
    # every cell of an 8x8x8 grid gets a distinct key in [0, 2^9)
    g = np.stack(np.meshgrid(*[np.arange(8)] * 3, indexing="ij"), -1).reshape(-1, 3)
    pts = ((g + 0.5) / 8).astype(np.float32)
    keys = oracle.hilbert_keys(pts, 3, False, 3, 1)
    assert sorted(keys.tolist()) == list(range(512))
    # consecutive keys are neighbouring cells (Hilbert adjacency)
    order = g[np.argsort(keys)]
    steps = np.abs(np.diff(order, axis=0)).sum(1)
    assert np.all(steps == 1)


@pytest.mark.parametrize("name", ["u3", "g3", "small3", "ragged3", "dup3", "u2", "p8"])
def test_counts_match_reference_bvh(oracle, cases, name):
    objs, boxes, dims = cases.COUNT_CASES[name]()
    g = golden(f"counts_{name}.npz")
    assert str(g["digest"]) == _digest(objs, boxes), "seeded generator changed"
    got = oracle.counts(objs, dims, False, boxes)
    assert np.array_equal(got, g["counts"].astype(np.uint64))


def test_ids_sorted_and_consistent(oracle, cases):
    objs, boxes, dims = cases.COUNT_CASES["u3"]()
    offs, ids = oracle.ids(objs, dims, False, boxes)
    counts = oracle.counts(objs, dims, False, boxes)
    assert np.array_equal(np.diff(offs), counts)
    for i in range(len(boxes)):
        s = ids[offs[i]:offs[i + 1]]
        assert np.all(np.diff(s) > 0)
        if len(s):
            p = objs[s]
            b = boxes[i]
            ok = ~((b[:dims] > p) | (b[dims:] < p))
            assert np.all(ok | np.isnan(b[:dims]) | np.isnan(b[dims:]))


def test_closed_interval_edges(oracle):
    pts = np.array([[0.25, 0.25, 0.25], [0.5, 0.5, 0.5]], np.float32)
    box_on = np.array([[0.25, 0.25, 0.25, 0.25, 0.25, 0.25]], np.float32)
    box_face = np.array([[0.5, 0.0, 0.0, 0.7, 1.0, 1.0]], np.float32)
    box_inverted = np.array([[0.6, 0.6, 0.6, 0.4, 0.4, 0.4]], np.float32)
    box_nan = np.array([[np.nan, 0.0, 0.0, 0.3, 0.3, 0.3]], np.float32)
    assert oracle.counts(pts, 3, False, box_on)[0] == 1
    assert oracle.counts(pts, 3, False, box_face)[0] == 1
    assert oracle.counts(pts, 3, False, box_inverted)[0] == 0
    # a NaN bound compares false, so that dimension never excludes
    assert oracle.counts(pts, 3, False, box_nan)[0] == 1


def test_rect_predicate(oracle):
    rects = np.array([[0.1, 0.1, 0.2, 0.2], [0.5, 0.5, 0.6, 0.6]], np.float32)  # 2-D [lo, hi]
    touching = np.array([[0.2, 0.2, 0.3, 0.3]], np.float32)
    inside = np.array([[0.52, 0.52, 0.55, 0.55]], np.float32)
    assert oracle.counts(rects, 2, True, touching)[0] == 1
    assert oracle.counts(rects, 2, True, inside)[0] == 1


@pytest.mark.parametrize("n,fanout,want", [
    (1, 128, [1]), (128, 128, [1]), (129, 128, [2, 1]), (16384, 128, [128, 1]),
    (16385, 128, [129, 2, 1]), (1_000_000, 192, [5209, 28, 1]),
    (16_000_000, 192, [83334, 435, 3, 1]),
])
def test_level_sizes(oracle, n, fanout, want):
    # the 192-way sizes are the reference's for 1 M and 16 M objects
    assert oracle.level_sizes(n, fanout) == want


def test_sort_perm_stable(oracle):
    keys = np.array([5, 1, 5, 0, 1, 5], np.uint64)
    assert oracle.sort_perm(keys).tolist() == [3, 1, 4, 0, 2, 5]


def test_node_mbrs_cover_children(oracle):
    rng = np.random.default_rng(3)
    pts = rng.random((5000, 3), dtype=np.float32)
    levels = oracle.node_mbrs(pts, 3, False, 32)
    assert [len(l) for l in levels] == oracle.level_sizes(5000, 32)
    leaf = levels[0]
    for j in [0, 17, len(leaf) - 1]:
        e = pts[j * 32:(j + 1) * 32]
        assert np.array_equal(leaf[j, :3], e.min(0)) and np.array_equal(leaf[j, 3:], e.max(0))
    top = levels[-1]
    assert np.array_equal(top[0, :3], pts.min(0)) and np.array_equal(top[0, 3:], pts.max(0))
