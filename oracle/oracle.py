"""ctypes wrappers of the CPU oracle and of the reference harness.

TEST INFRASTRUCTURE ONLY: used by tests/, __graft_entry__.smoke() and the
CPU-baseline / reference arm of bench.py as the checker and the timed
reference, never by the product path.

  Oracle      oracle/_build/libqcp_oracle.so, the C restatement (qcp_oracle.c)
  Reference   oracle/_ref/libqcpref_d<D>.so, the reference compiled from its
              own sources plus ref_harness.cu (built by oracle/Makefile from
              the reference checkout; the built files travel with the repo
              snapshot, the sources are not needed at run time)
"""
from __future__ import annotations

import ctypes
import pathlib
import subprocess

import numpy as np

HERE = pathlib.Path(__file__).resolve().parent
ORACLE_SO = HERE / "_build" / "libqcp_oracle.so"
P, U32, U64 = ctypes.c_void_p, ctypes.c_uint32, ctypes.c_uint64


def _p(a: np.ndarray) -> ctypes.c_void_p:
    return ctypes.c_void_p(a.ctypes.data)


def build_oracle() -> None:
    subprocess.run(["make", "-s", "-C", str(HERE), "oracle"], check=True)


class Oracle:
    def __init__(self):
        if not ORACLE_SO.exists():
            build_oracle()
        lib = ctypes.CDLL(str(ORACLE_SO))
        lib.oracle_hilbert_keys.argtypes = [P, U64, U32, U32, U32, U32, P]
        lib.oracle_range_counts.argtypes = [P, U64, U32, U32, P, U32, U32, P]
        lib.oracle_range_ids.argtypes = [P, U64, U32, U32, P, U32, U32, P, P, U64]
        lib.oracle_range_ids.restype = U64
        lib.oracle_sort_perm.argtypes = [P, U64, P]
        lib.oracle_level_sizes.argtypes = [U64, U32, P, U32]
        lib.oracle_level_sizes.restype = U32
        lib.oracle_node_mbrs.argtypes = [P, U64, U32, U32, U32, P]
        lib.oracle_hilbert_coords.argtypes = [U32, U32, P]
        lib.oracle_hilbert_coords.restype = U64
        self.lib = lib

    @staticmethod
    def _objs(objs):
        return np.ascontiguousarray(objs, dtype=np.float32)

    def hilbert_keys(self, objs, dims, is_rect, bits, mode):
        o = self._objs(objs)
        out = np.zeros(o.shape[0], np.uint64)
        self.lib.oracle_hilbert_keys(_p(o), o.shape[0], dims, int(is_rect), bits, mode, _p(out))
        return out

    def counts(self, objs, dims, is_rect, boxes, threads=8):
        o, b = self._objs(objs), self._objs(boxes)
        out = np.zeros(b.shape[0], np.uint64)
        self.lib.oracle_range_counts(_p(o), o.shape[0], dims, int(is_rect), _p(b), b.shape[0], threads, _p(out))
        return out

    def ids(self, objs, dims, is_rect, boxes, threads=8):
        """(offsets[q+1], sorted ids) by brute force."""
        o, b = self._objs(objs), self._objs(boxes)
        q = b.shape[0]
        offs = np.zeros(q + 1, np.uint64)
        total = self.lib.oracle_range_ids(_p(o), o.shape[0], dims, int(is_rect), _p(b), q, threads,
                                          _p(offs), None, 0)
        ids = np.zeros(max(int(total), 1), np.int32)
        self.lib.oracle_range_ids(_p(o), o.shape[0], dims, int(is_rect), _p(b), q, threads, _p(offs),
                                  _p(ids), int(total))
        return offs, ids[:int(total)]

    def sort_perm(self, keys):
        k = np.ascontiguousarray(keys, dtype=np.uint64)
        out = np.zeros(k.shape[0], np.uint32)
        self.lib.oracle_sort_perm(_p(k), k.shape[0], _p(out))
        return out

    def kmeans_keys(self, objs, dims, is_rect, bits, clusters, iters):
        """Restatement of the library's k-means-clustered keys (QCP_KEY_KMEANS),
        in numpy + the C key above: representative point (the object, or the
        FP32 centre 0.5*(lo+hi) of a rectangle); centres start at the objects
        floor(k*n/K); assignment = FP32 squared distance accumulated dimension
        by dimension, first minimum; update = mean through 64-bit fixed point
        relative to the bounding box (32 fractional bits); stop when at most
        1e-5 of the objects changed or after `iters` assignments; clusters
        ranked by the normalised key of their centre (ties by index); key =
        rank in the top ceil(log2 K) bits, the object's own normalised key
        below.  The reference's clustering step this follows is
        KmeansMapper::ClusteringBranches (src/mapper/kmeans_mapper.cpp:204-259)
        with cuda_kmeans (:15-199)."""
        o = self._objs(objs)
        n = o.shape[0]
        rep = (np.float32(0.5) * (o[:, :dims] + o[:, dims:2 * dims])).astype(np.float32) if is_rect else o[:, :dims]
        K = max(1, min(int(clusters), n))
        lo = rep.min(0).astype(np.float64)
        hi = rep.max(0).astype(np.float64)
        with np.errstate(divide="ignore", invalid="ignore"):
            scale = np.where((hi > lo) & np.isfinite(hi - lo), 4294967296.0 / (hi - lo), 0.0)
        cen = rep[(np.arange(K, dtype=np.uint64) * np.uint64(n)) // np.uint64(K)].copy()
        member = np.full(n, -1, np.int64)
        f = (rep.astype(np.float64) - lo) * scale
        f[~(f > 0)] = 0.0
        f = np.minimum(f, 4294967296.0).astype(np.uint64)
        for _ in range(int(iters)):
            dist = np.zeros((n, K), np.float32)
            for d in range(dims):
                t = rep[:, d, None] - cen[None, :, d]
                dist = dist + t * t
            arg = dist.argmin(1)
            changes = int((arg != member).sum())
            member = arg
            cnt = np.bincount(arg, minlength=K).astype(np.uint64)
            for d in range(dims):
                sums = np.zeros(K, np.uint64)
                np.add.at(sums, arg, f[:, d])
                upd = (cnt > 0) & (scale[d] > 0)
                cen[upd, d] = (lo[d] + (sums[upd].astype(np.float64) / cnt[upd].astype(np.float64)) / scale[d]
                               ).astype(np.float32)
            if changes / n <= 1e-5:
                break
        ckey = self.hilbert_keys(cen, dims, False, bits, 1)
        order = np.lexsort((np.arange(K), ckey))
        rank = np.empty(K, np.uint64)
        rank[order] = np.arange(K, dtype=np.uint64)
        rbits = 1
        while rbits < 32 and (1 << rbits) < K:
            rbits += 1
        own = self.hilbert_keys(o, dims, is_rect, bits, 1)
        own_bits = dims * bits
        shift = own_bits - (64 - rbits) if own_bits > 64 - rbits else 0
        return (rank[member] << np.uint64(64 - rbits)) | (own >> np.uint64(shift))

    def level_sizes(self, n, fanout):
        out = np.zeros(64, np.uint64)
        L = self.lib.oracle_level_sizes(n, fanout, _p(out), 64)
        return [int(x) for x in out[:L]]

    def node_mbrs(self, sorted_objs, dims, is_rect, fanout):
        o = self._objs(sorted_objs)
        sizes = self.level_sizes(o.shape[0], fanout)
        out = np.zeros((sum(sizes), 2 * dims), np.float32)
        self.lib.oracle_node_mbrs(_p(o), o.shape[0], dims, int(is_rect), fanout, _p(out))
        levels, at = [], 0
        for s in sizes:
            levels.append(out[at:at + s])
            at += s
        return levels


class Reference:
    """The reference implementation (compiled for `dims` dimensions)."""

    def __init__(self, dims: int = 3):
        path = HERE / "_ref" / f"libqcpref_d{dims}.so"
        if not path.exists():
            raise FileNotFoundError(f"{path} not built (make -C oracle ref, needs the reference sources)")
        lib = ctypes.CDLL(str(path))
        lib.ref_dims.restype = U32
        lib.ref_hilbert_keys.argtypes = [U32, P, U64, P]
        lib.ref_bvh_build.argtypes = [P, U64]
        lib.ref_bvh_build.restype = P
        lib.ref_bvh_counts.argtypes = [P, P, U32, U32, P]
        lib.ref_bvh_search_seconds.argtypes = [P, P, U32, U32]
        lib.ref_bvh_search_seconds.restype = ctypes.c_double
        lib.ref_bvh_free.argtypes = [P]
        lib.ref_mphr_build.argtypes = [P, U64]
        lib.ref_mphr_build.restype = P
        lib.ref_mphr_counts.argtypes = [P, P, U32, P, P]
        lib.ref_mphr_free.argtypes = [P]
        self.lib = lib
        self.dims = int(lib.ref_dims())

    @staticmethod
    def available(dims: int = 3) -> bool:
        return (HERE / "_ref" / f"libqcpref_d{dims}.so").exists()

    def hilbert_keys(self, pts, bits):
        p = np.ascontiguousarray(pts, dtype=np.float32)
        out = np.zeros(p.shape[0], np.int64)
        self.lib.ref_hilbert_keys(bits, _p(p), p.shape[0], _p(out))
        return out

    def bvh_build(self, pts):
        p = np.ascontiguousarray(pts, dtype=np.float32)
        h = self.lib.ref_bvh_build(_p(p), p.shape[0])
        if not h:
            raise RuntimeError("reference BVH build failed")
        return h

    def bvh_counts(self, h, boxes, threads=8):
        b = np.ascontiguousarray(boxes, dtype=np.float32)
        out = np.zeros(b.shape[0], np.uint32)
        self.lib.ref_bvh_counts(h, _p(b), b.shape[0], threads, _p(out))
        return out

    def bvh_search_seconds(self, h, boxes, threads):
        b = np.ascontiguousarray(boxes, dtype=np.float32)
        return float(self.lib.ref_bvh_search_seconds(h, _p(b), b.shape[0], threads))

    def bvh_free(self, h):
        self.lib.ref_bvh_free(h)

    def mphr_build(self, pts):
        p = np.ascontiguousarray(pts, dtype=np.float32)
        h = self.lib.ref_mphr_build(_p(p), p.shape[0])
        if not h:
            raise RuntimeError("reference MPHR build failed")
        return h

    def mphr_counts(self, h, boxes):
        b = np.ascontiguousarray(boxes, dtype=np.float32)
        out = np.zeros(b.shape[0], np.uint32)
        ms = ctypes.c_float(0.0)
        rc = self.lib.ref_mphr_counts(h, _p(b), b.shape[0], _p(out), ctypes.byref(ms))
        if rc != 0:
            raise RuntimeError(f"reference MPHR search failed ({rc})")
        return out, float(ms.value)
