"""Seeded inputs behind the golden vectors (shared by make_golden.py and the tests).

All coordinates are float32.  Queries are [lo.., hi..] boxes.  Besides random
boxes every 3-D case appends the edge cases the predicate must handle:
degenerate boxes equal to a data point, boxes whose faces pass exactly
through data coordinates (closed intervals), an inverted box, boxes covering
everything, boxes outside the data, infinite bounds and a NaN bound (the
reference's comparisons treat a NaN bound as overlapping).
"""
from __future__ import annotations

import numpy as np

SEED = 20240611


def _rng(k: int) -> np.random.Generator:
    return np.random.Generator(np.random.PCG64(SEED + k))


def kat_points(dims: int) -> np.ndarray:
    r = _rng(dims)
    pts = r.random((512, dims), dtype=np.float32)
    special = np.array([[0.0] * dims, [0.5] * dims, [np.nextafter(np.float32(1), np.float32(0))] * dims,
                        [0.5, 0.25, 0.75][:dims] + [0.1] * max(0, dims - 3),
                        [1e-6] * dims, [0.999999] * dims], dtype=np.float32)
    return np.ascontiguousarray(np.concatenate([special, pts]), dtype=np.float32)


def edge_boxes(objs: np.ndarray, dims: int, r: np.random.Generator) -> np.ndarray:
    inf = np.float32(np.inf)
    out = []
    for i in r.integers(0, objs.shape[0], size=6):
        p = objs[i, :dims]
        out.append(np.concatenate([p, p]))                      # degenerate box on a point
        lo = p.copy()
        hi = p + np.float32(0.05)
        out.append(np.concatenate([lo, hi]))                    # face through a data point
        out.append(np.concatenate([p - np.float32(0.05), p]))   # other face through it
    out.append(np.concatenate([np.full(dims, 0.6, np.float32), np.full(dims, 0.4, np.float32)]))  # inverted
    out.append(np.concatenate([np.full(dims, -1, np.float32), np.full(dims, 2, np.float32)]))     # all
    out.append(np.concatenate([np.full(dims, 2, np.float32), np.full(dims, 3, np.float32)]))      # outside
    out.append(np.concatenate([np.full(dims, -inf), np.full(dims, inf)]))                          # infinite
    b = np.concatenate([np.full(dims, 0.2, np.float32), np.full(dims, 0.4, np.float32)])
    b[0] = np.nan                                                                                   # NaN bound
    out.append(b)
    b2 = np.concatenate([np.full(dims, 0.3, np.float32), np.full(dims, 0.5, np.float32)])
    b2[dims] = np.nan                                                                              # NaN hi bound
    out.append(b2)
    return np.asarray(out, dtype=np.float32)


def _cubes(centres, sides):
    c = centres.astype(np.float32)
    h = (sides.astype(np.float32) * np.float32(0.5)).reshape(-1, 1)
    return np.ascontiguousarray(np.concatenate([c - h, c + h], axis=1), dtype=np.float32)


def case_u3():
    r = _rng(101)
    objs = r.random((20000, 3), dtype=np.float32)
    boxes = _cubes(r.random((300, 3), dtype=np.float32), r.uniform(0.01, 0.2, 300))
    boxes = np.concatenate([boxes, edge_boxes(objs, 3, r)])
    return objs, np.ascontiguousarray(boxes, dtype=np.float32), 3


def case_g3():
    r = _rng(102)
    centres = r.random((64, 3), dtype=np.float32)
    which = r.integers(0, 64, size=30000)
    objs = centres[which] + r.standard_normal((30000, 3), dtype=np.float32) * np.float32(0.02)
    objs = np.clip(objs, 0, np.nextafter(np.float32(1), np.float32(0))).astype(np.float32)
    idx = r.integers(0, 30000, size=300)
    vols = np.exp(r.uniform(np.log(1e-6), np.log(1e-2), 300))
    boxes = _cubes(objs[idx], vols ** (1 / 3))
    boxes = np.concatenate([boxes, edge_boxes(objs, 3, r)])
    return np.ascontiguousarray(objs), np.ascontiguousarray(boxes, dtype=np.float32), 3


def case_small3():
    """Fewer objects than one reference leaf (the reference root is a leaf)."""
    r = _rng(103)
    objs = r.random((150, 3), dtype=np.float32)
    boxes = _cubes(r.random((40, 3), dtype=np.float32), r.uniform(0.05, 0.6, 40))
    boxes = np.concatenate([boxes, edge_boxes(objs, 3, r)])
    return objs, np.ascontiguousarray(boxes, dtype=np.float32), 3


def case_ragged3():
    """192*192 + 7 objects: ragged last leaf and ragged upper levels."""
    r = _rng(104)
    objs = r.random((192 * 192 + 7, 3), dtype=np.float32)
    boxes = _cubes(r.random((200, 3), dtype=np.float32), r.uniform(0.02, 0.3, 200))
    boxes = np.concatenate([boxes, edge_boxes(objs, 3, r)])
    return objs, np.ascontiguousarray(boxes, dtype=np.float32), 3


def case_dup3():
    """Many duplicate points (equal keys) on a coarse grid."""
    r = _rng(105)
    objs = (r.integers(0, 20, size=(25000, 3)).astype(np.float32) / np.float32(20.0)).astype(np.float32)
    boxes = _cubes(r.random((150, 3), dtype=np.float32), r.uniform(0.05, 0.3, 150))
    boxes = np.concatenate([boxes, edge_boxes(objs, 3, r)])
    return objs, np.ascontiguousarray(boxes, dtype=np.float32), 3


def case_u2():
    r = _rng(106)
    objs = r.random((20000, 2), dtype=np.float32)
    boxes = _cubes(r.random((200, 2), dtype=np.float32), r.uniform(0.005, 0.1, 200))
    boxes = np.concatenate([boxes, edge_boxes(objs, 2, r)])
    return objs, np.ascontiguousarray(boxes, dtype=np.float32), 2


def case_p8():
    r = _rng(107)
    objs = r.random((5000, 8), dtype=np.float32)
    c = r.random((100, 8), dtype=np.float32)
    s = r.uniform(0.4, 0.9, size=(100, 8)).astype(np.float32) * np.float32(0.5)
    boxes = np.concatenate([c - s, c + s], axis=1).astype(np.float32)
    boxes = np.concatenate([boxes, edge_boxes(objs, 8, r)])
    return objs, np.ascontiguousarray(boxes, dtype=np.float32), 8


COUNT_CASES = {
    "u3": case_u3,
    "g3": case_g3,
    "small3": case_small3,
    "ragged3": case_ragged3,
    "dup3": case_dup3,
    "u2": case_u2,
    "p8": case_p8,
}
