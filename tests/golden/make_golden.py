"""Generate the golden vectors under tests/golden/ from the reference itself.

Run in a checkout that has the reference sources, after `make -C oracle ref`:

    python tests/golden/make_golden.py

Every vector comes from the reference compiled from its own sources
(oracle/_ref/libqcpref_d<D>.so):
  hilbert_kat.npz   HilbertMapper::MappingIntoSingle keys (3-D/20 bits and
                    2-D/31 bits, src/mapper/hilbert_mapper.cpp:15-68)
  counts_<name>.npz per-query hit counts of the reference CPU BVH traversal
                    (BVH::TraverseInternalNodes, src/tree/bvh.cpp:256-278) on
                    small seeded workloads, plus a checksum of the inputs so a
                    change in the generators is caught
Inputs are not stored; they are regenerated from the seeds in
tests/golden/cases.py.
"""
from __future__ import annotations

import hashlib
import pathlib
import sys

import numpy as np

HERE = pathlib.Path(__file__).resolve().parent
ROOT = HERE.parent.parent
sys.path.insert(0, str(ROOT / "oracle"))
sys.path.insert(0, str(HERE))

import cases  # noqa: E402
from oracle import Reference  # noqa: E402


def digest(*arrays) -> str:
    h = hashlib.sha256()
    for a in arrays:
        h.update(np.ascontiguousarray(a).tobytes())
    return h.hexdigest()


def main() -> None:
    # Hilbert known answers
    kat = {}
    for dims, bits in [(3, 20), (2, 31)]:
        ref = Reference(dims)
        pts = cases.kat_points(dims)
        kat[f"pts_d{dims}"] = pts
        kat[f"keys_d{dims}_b{bits}"] = ref.hilbert_keys(pts, bits)
    np.savez_compressed(HERE / "hilbert_kat.npz", **kat)
    print("hilbert_kat.npz", {k: v.shape for k, v in kat.items()})

    for name, make in cases.COUNT_CASES.items():
        objs, boxes, dims = make()
        ref = Reference(dims)
        h = ref.bvh_build(objs)
        counts = ref.bvh_counts(h, boxes, threads=8)
        np.savez_compressed(HERE / f"counts_{name}.npz", counts=counts.astype(np.uint32),
                            digest=np.array(digest(objs, boxes)))
        print(f"counts_{name}.npz n={objs.shape[0]} q={boxes.shape[0]} hits={int(counts.sum())}")


if __name__ == "__main__":
    main()
