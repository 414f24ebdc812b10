"""Seeded synthetic inputs for the range-search path.

The reference's experiment files (a 200 M-point synthetic set and the NOAA
set, src/evaluator/evaluator.cpp:479-505) are not part of the reference
repository, so every workload here is generated from a seed with numpy's
PCG64 bit generator (O'Neill, "PCG: A Family of Simple Fast Space-Efficient
Statistically Good Algorithms for Random Number Generation", 2014).  The same
numpy version produces the same bytes on every machine.

Layouts follow the reference's binary formats (src/io/dataset.cpp:36-39,
:82-88): objects are row-major float32, one row of D floats per point (or
2*D floats [lo.., hi..] per rectangle); queries are row-major float32 boxes
[lo0..lo(D-1), hi0..hi(D-1)].

Seeds: data 1234 (the reference generator's seed, generator/cuRAND.cpp:49),
queries 4321.
"""
from __future__ import annotations

import dataclasses

import numpy as np

DATA_SEED = 1234
QUERY_SEED = 4321
ONE_BELOW = np.nextafter(np.float32(1.0), np.float32(0.0))


@dataclasses.dataclass
class Workload:
    name: str
    dims: int
    is_rect: bool
    objs: np.ndarray      # (n, dims) or (n, 2*dims) float32, C-contiguous
    boxes: np.ndarray     # (q, 2*dims) float32, C-contiguous
    fanout: int = 128
    key_bits: int = 0     # 0 = the library default for dims

    @property
    def n(self) -> int:
        return int(self.objs.shape[0])

    @property
    def q(self) -> int:
        return int(self.boxes.shape[0])


def _cubes(centres: np.ndarray, sides: np.ndarray) -> np.ndarray:
    """Boxes lo = c - s/2, hi = c + s/2 in float32, not clipped."""
    c = centres.astype(np.float32)
    h = (sides.astype(np.float32) * np.float32(0.5)).reshape(-1, 1) if sides.ndim == 1 \
        else sides.astype(np.float32) * np.float32(0.5)
    lo = (c - h).astype(np.float32)
    hi = (c + h).astype(np.float32)
    return np.ascontiguousarray(np.concatenate([lo, hi], axis=1), dtype=np.float32)


def uniform_points(n: int, dims: int, seed: int = DATA_SEED) -> np.ndarray:
    rng = np.random.Generator(np.random.PCG64(seed))
    return np.ascontiguousarray(rng.random((n, dims), dtype=np.float32))


def gaussian_mixture_points(n: int, dims: int = 3, clusters: int = 64, sigma: float = 0.02,
                            seed: int = DATA_SEED) -> np.ndarray:
    """n points from `clusters` isotropic Gaussians with centres U[0,1)^dims,
    each coordinate clamped to [0, nextafterf(1, 0)]."""
    rng = np.random.Generator(np.random.PCG64(seed))
    centres = rng.random((clusters, dims), dtype=np.float32)
    which = rng.integers(0, clusters, size=n)
    pts = rng.standard_normal((n, dims), dtype=np.float32)
    pts *= np.float32(sigma)
    pts += centres[which]
    np.clip(pts, np.float32(0.0), ONE_BELOW, out=pts)
    return np.ascontiguousarray(pts, dtype=np.float32)


def fixed_cubes(q: int, dims: int, side: float, seed: int = QUERY_SEED) -> np.ndarray:
    rng = np.random.Generator(np.random.PCG64(seed))
    centres = rng.random((q, dims), dtype=np.float32)
    return _cubes(centres, np.full(q, side, dtype=np.float32))


def data_centred_cubes(objs: np.ndarray, q: int, vol_lo: float, vol_hi: float,
                       seed: int = QUERY_SEED) -> np.ndarray:
    """Cubes centred on random data points with volume log-uniform in
    [vol_lo, vol_hi]; side = volume^(1/dims)."""
    dims = objs.shape[1]
    rng = np.random.Generator(np.random.PCG64(seed))
    idx = rng.integers(0, objs.shape[0], size=q)
    logv = rng.uniform(np.log(vol_lo), np.log(vol_hi), size=q)
    sides = np.exp(logv / dims).astype(np.float32)
    return _cubes(objs[idx], sides)


def config1(scale: float = 1.0) -> Workload:
    """1,000,000 uniform 3-D points, 1,000 cubes of side 0.0464 (~100 hits)."""
    n = max(1, int(1_000_000 * scale))
    q = max(1, int(1000 * min(1.0, scale * 10)))
    return Workload("uniform3d_1M_q1k", 3, False, uniform_points(n, 3),
                    fixed_cubes(q, 3, 0.0464), fanout=128)


def config2(scale: float = 1.0, q: int | None = None) -> Workload:
    """16,000,000 points from 64 Gaussians (sigma 0.02); 10,000 data-centred
    cubes with volume log-uniform over [1e-6, 1e-2]."""
    n = max(1, int(16_000_000 * scale))
    pts = gaussian_mixture_points(n, 3)
    nq = q if q is not None else 10_000
    return Workload("gauss64_3d_16M_q10k", 3, False, pts,
                    data_centred_cubes(pts, nq, 1e-6, 1e-2), fanout=128)


def config3(scale: float = 1.0, fanout: int = 128) -> Workload:
    """64,000,000 uniform 2-D points, 100,000 squares of area 1e-5."""
    n = max(1, int(64_000_000 * scale))
    q = max(1, int(100_000 * min(1.0, scale * 10)))
    return Workload("uniform2d_64M_q100k", 2, False, uniform_points(n, 2),
                    fixed_cubes(q, 2, float(np.sqrt(1e-5))), fanout=fanout, key_bits=32)


def config4(scale: float = 1.0) -> Workload:
    """32,000,000 8-D rectangles: lo U[0,1)^8, sides Exp(mean 0.002);
    50,000 boxes with centre U[0,1)^8 and sides U[0.05, 0.2]."""
    n = max(1, int(32_000_000 * scale))
    rng = np.random.Generator(np.random.PCG64(DATA_SEED))
    lo = rng.random((n, 8), dtype=np.float32)
    side = rng.exponential(0.002, size=(n, 8)).astype(np.float32)
    objs = np.ascontiguousarray(np.concatenate([lo, (lo + side).astype(np.float32)], axis=1))
    q = max(1, int(50_000 * min(1.0, scale * 10)))
    return Workload("rect8d_32M_q50k", 8, True, objs, rect8d_boxes(q), fanout=128)


def rect8d_boxes(q: int, seed: int = QUERY_SEED) -> np.ndarray:
    """q 8-D boxes: centre U[0,1)^8, side per dimension U[0.05, 0.2]."""
    qr = np.random.Generator(np.random.PCG64(seed))
    centres = qr.random((q, 8), dtype=np.float32)
    sides = qr.uniform(0.05, 0.2, size=(q, 8)).astype(np.float32)
    return _cubes(centres, sides)


def serving_stream(objs: np.ndarray, rate: float = 200_000.0, duration_s: float = 10.0,
                   seed: int = QUERY_SEED):
    """Open-loop Poisson arrivals: returns (arrival_times_s, boxes, volume_class).
    Cube volumes 1e-7 / 1e-5 / 1e-3 with probabilities 0.70 / 0.25 / 0.05,
    centred on random data points."""
    dims = objs.shape[1]
    rng = np.random.Generator(np.random.PCG64(seed + 5))
    nreq = int(rate * duration_s)
    gaps = rng.exponential(1.0 / rate, size=nreq)
    t = np.cumsum(gaps)
    cls = rng.choice(3, size=nreq, p=[0.70, 0.25, 0.05])
    vols = np.array([1e-7, 1e-5, 1e-3])[cls]
    idx = rng.integers(0, objs.shape[0], size=nreq)
    sides = (vols ** (1.0 / dims)).astype(np.float32)
    return t, _cubes(objs[idx], sides), cls
