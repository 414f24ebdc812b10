"""B200 range-search library: Python binding of the C ABI in include/qcp.h.

The compute path is the CUDA library libqcp_b200.so next to this file
(built by the Makefile here, or by __graft_entry__.build()).  This module
only marshals arguments; there is no CPU fallback, and loading fails loudly
when the library is missing.

Index mirrors the reference's tree interface (src/tree/tree.h:15-155):
``Index.build`` stands for Tree::Build, ``Index.search`` for Tree::Search
(returning per-query id lists instead of a logged total), ``save``/``load``
for DumpToFile/DumpFromFile.
"""
from __future__ import annotations

import ctypes
import os
import pathlib

import numpy as np

PKG_DIR = pathlib.Path(__file__).resolve().parent
LIB_PATH = PKG_DIR / "libqcp_b200.so"

QCP_OK = 0
STATUS_NAMES = {
    0: "QCP_OK", 1: "QCP_ERR_BAD_ARG", 2: "QCP_ERR_OOM", 3: "QCP_ERR_OUTPUT_OVERFLOW",
    4: "QCP_ERR_TIMEOUT", 5: "QCP_ERR_CUDA", 6: "QCP_ERR_NO_DEVICE", 7: "QCP_ERR_IO",
}
MEM_HOST, MEM_DEVICE = 0, 1
KEY_NORM, KEY_REF, KEY_KMEANS = 0, 1, 2
ALGO_BATCHED, ALGO_PLAIN, ALGO_HYBRID = 0, 1, 2


class QcpError(RuntimeError):
    def __init__(self, status: int, message: str):
        super().__init__(f"{STATUS_NAMES.get(status, status)}: {message}")
        self.status = status
        self.message = message


class BuildOpts(ctypes.Structure):
    _fields_ = [("fanout", ctypes.c_uint32), ("key_mode", ctypes.c_uint32),
                ("key_bits", ctypes.c_uint32), ("input_mem", ctypes.c_uint32),
                ("stream", ctypes.c_void_p), ("kmeans_clusters", ctypes.c_uint32),
                ("kmeans_iters", ctypes.c_uint32)]


class IndexInfo(ctypes.Structure):
    _fields_ = [("n", ctypes.c_uint64), ("dims", ctypes.c_uint32), ("is_rect", ctypes.c_uint32),
                ("fanout", ctypes.c_uint32), ("levels", ctypes.c_uint32),
                ("level_nodes", ctypes.c_uint64 * 16), ("device_bytes", ctypes.c_uint64),
                ("key_mode", ctypes.c_uint32), ("key_bits", ctypes.c_uint32)]


class QueryOpts(ctypes.Structure):
    _fields_ = [("algo", ctypes.c_uint32), ("boxes_mem", ctypes.c_uint32),
                ("result_mem", ctypes.c_uint32), ("unsorted", ctypes.c_uint32),
                ("stream", ctypes.c_void_p), ("flags", ctypes.c_uint32),
                ("blocks_per_sm", ctypes.c_uint32), ("win_bits", ctypes.c_uint32),
                ("cpu_threads", ctypes.c_uint32), ("handoff_level", ctypes.c_uint32),
                ("leaf_prefetch", ctypes.c_uint32), ("lanes_per_item", ctypes.c_uint32),
                ("hit_cache", ctypes.c_uint32)]


QUERY_TIMING = 1


class QueryStats(ctypes.Structure):
    _fields_ = [("algo", ctypes.c_uint32), ("num_queries", ctypes.c_uint32),
                ("frontier_items", ctypes.c_uint64 * 16), ("leaf_items", ctypes.c_uint64),
                ("leaves_covered", ctypes.c_uint64), ("leaves_partial", ctypes.c_uint64),
                ("objects_covered", ctypes.c_uint64), ("hits", ctypes.c_uint64),
                ("sort_small_jobs", ctypes.c_uint32), ("sort_msd_jobs", ctypes.c_uint32),
                ("ms_expand", ctypes.c_float), ("ms_count", ctypes.c_float),
                ("ms_scan", ctypes.c_float), ("ms_write", ctypes.c_float),
                ("ms_sort", ctypes.c_float), ("ms_total", ctypes.c_float),
                ("ms_sort_small", ctypes.c_float), ("ms_sort_partition", ctypes.c_float),
                ("ms_sort_windows", ctypes.c_float), ("sort_window_ids", ctypes.c_uint64),
                ("ms_sort_windows_bitmap", ctypes.c_float), ("sort_window_bitmap_ids", ctypes.c_uint64)]


DELIVER_FN = ctypes.CFUNCTYPE(None, ctypes.c_void_p, ctypes.c_uint32, ctypes.POINTER(ctypes.c_int32),
                              ctypes.c_uint64)


class ServeOpts(ctypes.Structure):
    _fields_ = [("streams", ctypes.c_uint32), ("max_batch", ctypes.c_uint32),
                ("output_cap_bytes", ctypes.c_uint64), ("deliver", DELIVER_FN),
                ("user", ctypes.c_void_p), ("trace", ctypes.c_void_p), ("trace_cap", ctypes.c_uint64)]


class ServeBatch(ctypes.Structure):
    """qcp_serve_batch: one run of a serving replay (times in seconds)."""
    _fields_ = [("worker", ctypes.c_uint32), ("requests", ctypes.c_uint32), ("path", ctypes.c_uint32),
                ("split", ctypes.c_uint32), ("hits", ctypes.c_uint64), ("t_taken", ctypes.c_double),
                ("t_start", ctypes.c_double), ("t_run", ctypes.c_double), ("t_admitted", ctypes.c_double),
                ("t_done", ctypes.c_double)]


# numpy view of an array of qcp_serve_batch records
SERVE_BATCH_DTYPE = np.dtype([(n, {ctypes.c_uint32: "<u4", ctypes.c_uint64: "<u8", ctypes.c_double: "<f8"}[t])
                              for n, t in ServeBatch._fields_])


class ServeStats(ctypes.Structure):
    _fields_ = [("requests", ctypes.c_uint64), ("hits", ctypes.c_uint64), ("batches", ctypes.c_uint64),
                ("mean_batch", ctypes.c_double), ("seconds", ctypes.c_double), ("qps", ctypes.c_double),
                ("p50_ms", ctypes.c_double), ("p99_ms", ctypes.c_double), ("max_ms", ctypes.c_double),
                ("mean_ms", ctypes.c_double), ("max_inflight", ctypes.c_uint32),
                ("reserved_", ctypes.c_uint32), ("max_output_bytes", ctypes.c_uint64)]


TUNE_MAX_TRIALS = 16


class TuneResult(ctypes.Structure):
    _fields_ = [("fanout", ctypes.c_uint32), ("blocks_per_sm", ctypes.c_uint32),
                ("win_bits", ctypes.c_uint32), ("trials", ctypes.c_uint32),
                ("best_ms", ctypes.c_float), ("build_ms", ctypes.c_float),
                ("trial_fanout", ctypes.c_uint32 * TUNE_MAX_TRIALS),
                ("trial_blocks_per_sm", ctypes.c_uint32 * TUNE_MAX_TRIALS),
                ("trial_win_bits", ctypes.c_uint32 * TUNE_MAX_TRIALS),
                ("trial_ms", ctypes.c_float * TUNE_MAX_TRIALS),
                ("leaf_prefetch", ctypes.c_uint32),
                ("trial_leaf_prefetch", ctypes.c_uint32 * TUNE_MAX_TRIALS),
                ("lanes_per_item", ctypes.c_uint32),
                ("trial_lanes_per_item", ctypes.c_uint32 * TUNE_MAX_TRIALS),
                ("hit_cache", ctypes.c_uint32),
                ("trial_hit_cache", ctypes.c_uint32 * TUNE_MAX_TRIALS)]


class Result(ctypes.Structure):
    _fields_ = [("num_queries", ctypes.c_uint32), ("mem", ctypes.c_uint32),
                ("total_hits", ctypes.c_uint64), ("offsets", ctypes.c_void_p),
                ("ids", ctypes.c_void_p), ("owner_", ctypes.c_void_p)]


_lib = None


def load_library(path: os.PathLike | str | None = None) -> ctypes.CDLL:
    """Load libqcp_b200.so (raises if it has not been built)."""
    global _lib
    if _lib is not None and path is None:
        return _lib
    p = pathlib.Path(path) if path else LIB_PATH
    if not p.exists():
        raise FileNotFoundError(
            f"{p} not found: build it with `make -C {PKG_DIR}` or __graft_entry__.build()")
    lib = ctypes.CDLL(str(p))
    P, U32, U64 = ctypes.c_void_p, ctypes.c_uint32, ctypes.c_uint64
    sig = {
        "qcp_index_build": ([P, U64, U32, U32, ctypes.POINTER(BuildOpts), ctypes.POINTER(P)], ctypes.c_int),
        "qcp_index_free": ([P], ctypes.c_int),
        "qcp_index_get_info": ([P, ctypes.POINTER(IndexInfo)], ctypes.c_int),
        "qcp_query_batch": ([P, P, U32, ctypes.POINTER(QueryOpts), ctypes.POINTER(Result)], ctypes.c_int),
        "qcp_query_counts": ([P, P, U32, ctypes.POINTER(QueryOpts), P], ctypes.c_int),
        "qcp_result_release": ([ctypes.POINTER(Result)], ctypes.c_int),
        "qcp_index_save": ([P, ctypes.c_char_p], ctypes.c_int),
        "qcp_index_load": ([ctypes.c_char_p, P, ctypes.POINTER(P)], ctypes.c_int),
        "qcp_index_export": ([P, P, P, U32, P], ctypes.c_int),
        "qcp_last_error": ([], ctypes.c_char_p),
        "qcp_launch_count": ([ctypes.c_int], U64),
        "qcp_version": ([], ctypes.c_char_p),
        "qcp_query_stats_last": ([ctypes.POINTER(QueryStats)], ctypes.c_int),
        "qcp_serve_replay": ([P, P, P, U32, ctypes.POINTER(ServeOpts), P, ctypes.POINTER(ServeStats)],
                             ctypes.c_int),
        "qcp_autotune": ([P, U64, U32, U32, P, U32, ctypes.POINTER(BuildOpts), U32, ctypes.POINTER(TuneResult)],
                         ctypes.c_int),
        "qcp_plan_create": ([P, U32, U64, ctypes.POINTER(QueryOpts), ctypes.POINTER(P)], ctypes.c_int),
        "qcp_plan_run": ([P, P, U32, U32, P, ctypes.POINTER(U64), ctypes.POINTER(P), ctypes.POINTER(P)],
                         ctypes.c_int),
        "qcp_plan_free": ([P], ctypes.c_int),
        "qcp_build_plan_create": ([U64, U32, U32, ctypes.POINTER(BuildOpts), ctypes.POINTER(P)], ctypes.c_int),
        "qcp_build_plan_input": ([P], P),
        "qcp_build_plan_run": ([P, P, U32, P, ctypes.POINTER(P)], ctypes.c_int),
        "qcp_build_plan_free": ([P], ctypes.c_int),
    }
    for name, (args, res) in sig.items():
        fn = getattr(lib, name)
        fn.argtypes = args
        fn.restype = res
    if path is None:
        _lib = lib
    return lib


def _check(status: int) -> None:
    if status != QCP_OK:
        msg = _lib.qcp_last_error().decode(errors="replace") if _lib else ""
        raise QcpError(status, msg)


def _ptr(a: np.ndarray) -> ctypes.c_void_p:
    return ctypes.c_void_p(a.ctypes.data)


def _device_ptr(t) -> int:
    """Device address of a CUDA tensor (torch) or an int."""
    if isinstance(t, int):
        return t
    return int(t.data_ptr())


class SearchResult:
    """CSR hit lists: ids of query i are ids[offsets[i]:offsets[i+1]]."""

    def __init__(self, offsets, ids, total_hits: int, mem: int, raw: Result | None = None):
        self.offsets = offsets
        self.ids = ids
        self.total_hits = total_hits
        self.mem = mem
        self._raw = raw

    def __len__(self) -> int:
        return len(self.offsets) - 1 if self.mem == MEM_HOST else int(self._raw.num_queries)

    def hits(self, i: int) -> np.ndarray:
        return self.ids[self.offsets[i]:self.offsets[i + 1]]

    def counts(self) -> np.ndarray:
        return np.diff(self.offsets)

    def release(self) -> None:
        if self._raw is not None and self._raw.owner_:
            load_library().qcp_result_release(ctypes.byref(self._raw))
        self._raw = None


class Index:
    """A device-resident bulk-loaded R-tree (one GPU)."""

    def __init__(self, handle: ctypes.c_void_p, dims: int, is_rect: bool, owned: bool = True):
        self._h = handle
        self.dims = dims
        self.is_rect = is_rect
        self._owned = owned  # False: a BuildPlan's index, freed with the plan

    # -- construction ---------------------------------------------------------
    @classmethod
    def build(cls, objs, dims: int | None = None, is_rect: bool = False, fanout: int = 128,
              key_mode: int = KEY_NORM, key_bits: int = 0, n: int | None = None,
              stream: int = 0, kmeans_clusters: int = 0, kmeans_iters: int = 0) -> "Index":
        """Build from a host numpy array (n x D points or n x 2D rects) or a
        CUDA tensor / device pointer (then pass n and dims)."""
        lib = load_library()
        opts = BuildOpts(fanout, key_mode, key_bits, MEM_HOST, ctypes.c_void_p(stream or None), kmeans_clusters,
                         kmeans_iters)
        if isinstance(objs, np.ndarray):
            a = np.ascontiguousarray(objs, dtype=np.float32)
            n = a.shape[0]
            width = a.shape[1]
            d = width // 2 if is_rect else width
            if dims is not None and dims != d:
                raise ValueError("dims does not match the array width")
            ptr = _ptr(a)
            keep = a
        else:
            if n is None or dims is None:
                raise ValueError("device input needs n and dims")
            d = dims
            opts.input_mem = MEM_DEVICE
            ptr = ctypes.c_void_p(_device_ptr(objs))
            keep = objs
        h = ctypes.c_void_p()
        _check(lib.qcp_index_build(ptr, n, d, 1 if is_rect else 0, ctypes.byref(opts), ctypes.byref(h)))
        del keep
        return cls(h, d, is_rect)

    @classmethod
    def load(cls, path: str) -> "Index":
        lib = load_library()
        h = ctypes.c_void_p()
        _check(lib.qcp_index_load(str(path).encode(), None, ctypes.byref(h)))
        idx = cls(h, 0, False)
        info = idx.info()
        idx.dims, idx.is_rect = info["dims"], bool(info["is_rect"])
        return idx

    def save(self, path: str) -> None:
        _check(load_library().qcp_index_save(self._h, str(path).encode()))

    def close(self) -> None:
        if self._h and self._owned:
            load_library().qcp_index_free(self._h)
        self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    # -- inspection -----------------------------------------------------------
    def info(self) -> dict:
        inf = IndexInfo()
        _check(load_library().qcp_index_get_info(self._h, ctypes.byref(inf)))
        return {"n": inf.n, "dims": inf.dims, "is_rect": inf.is_rect, "fanout": inf.fanout,
                "levels": inf.levels, "level_nodes": [inf.level_nodes[i] for i in range(inf.levels)],
                "device_bytes": inf.device_bytes, "key_mode": inf.key_mode, "key_bits": inf.key_bits}

    def export(self, level: int | None = None):
        """(sorted keys, sorted-position -> input id, MBRs of `level`)."""
        inf = self.info()
        n = inf["n"]
        keys = np.zeros(n, np.uint64)
        ids = np.zeros(n, np.int32)
        mbr = None
        mptr = None
        lv = 0
        if level is not None:
            lv = level
            mbr = np.zeros((inf["level_nodes"][level], 2 * inf["dims"]), np.float32)
            mptr = _ptr(mbr)
        _check(load_library().qcp_index_export(self._h, _ptr(keys), _ptr(ids), lv, mptr))
        return keys, ids, mbr

    # -- queries --------------------------------------------------------------
    def _opts(self, algo, boxes_mem, result_mem, sort, stream, timing=False, blocks_per_sm=0, win_bits=0,
              cpu_threads=0, handoff_level=0, leaf_prefetch=0, lanes_per_item=0, hit_cache=0):
        a = {"batched": ALGO_BATCHED, "plain": ALGO_PLAIN, "hybrid": ALGO_HYBRID}.get(algo, algo)
        return QueryOpts(a, boxes_mem, result_mem, 0 if sort else 1, ctypes.c_void_p(stream or None),
                         QUERY_TIMING if timing else 0, blocks_per_sm, win_bits, cpu_threads, handoff_level,
                         leaf_prefetch, lanes_per_item, hit_cache)

    def search(self, boxes, algo="batched", sort: bool = True, result_mem: int = MEM_HOST,
               q: int | None = None, stream: int = 0, timing: bool = False,
               copy: bool = True, blocks_per_sm: int = 0, win_bits: int = 0, cpu_threads: int = 0,
               handoff_level: int = 0, leaf_prefetch: int = 0, lanes_per_item: int = 0,
               hit_cache: int = 0) -> SearchResult:
        """Run a batch of box queries.  Host numpy boxes (q x 2D) or a CUDA
        tensor/pointer (then pass q).  Host results are copied into numpy
        arrays (copy=False: numpy views of the library's pinned result arena,
        valid until release()); device results stay library-owned until
        release()."""
        lib = load_library()
        if isinstance(boxes, np.ndarray):
            b = np.ascontiguousarray(boxes, dtype=np.float32).reshape(-1, 2 * self.dims)
            nq, ptr, bmem = b.shape[0], _ptr(b), MEM_HOST
        else:
            if q is None:
                raise ValueError("device boxes need q")
            b, nq, ptr, bmem = boxes, q, ctypes.c_void_p(_device_ptr(boxes)), MEM_DEVICE
        opts = self._opts(algo, bmem, result_mem, sort, stream, timing, blocks_per_sm, win_bits, cpu_threads,
                          handoff_level, leaf_prefetch, lanes_per_item, hit_cache)
        r = Result()
        _check(lib.qcp_query_batch(self._h, ptr, nq, ctypes.byref(opts), ctypes.byref(r)))
        if result_mem == MEM_HOST and not copy:
            offs = np.ctypeslib.as_array(ctypes.cast(r.offsets, ctypes.POINTER(ctypes.c_uint64)),
                                         shape=(nq + 1,))
            ids = (np.ctypeslib.as_array(ctypes.cast(r.ids, ctypes.POINTER(ctypes.c_int32)),
                                         shape=(int(r.total_hits),)) if r.total_hits
                   else np.zeros(0, np.int32))
            return SearchResult(offs, ids, int(r.total_hits), MEM_HOST, raw=r)
        if result_mem == MEM_HOST:
            total = int(r.total_hits)
            try:
                offs = np.ctypeslib.as_array(ctypes.cast(r.offsets, ctypes.POINTER(ctypes.c_uint64)),
                                             shape=(nq + 1,)).copy()
                if total:
                    ids = np.ctypeslib.as_array(ctypes.cast(r.ids, ctypes.POINTER(ctypes.c_int32)),
                                                shape=(total,)).copy()
                else:
                    ids = np.zeros(0, np.int32)
            finally:
                lib.qcp_result_release(ctypes.byref(r))
            return SearchResult(offs, ids, total, MEM_HOST)
        return SearchResult(r.offsets, r.ids, int(r.total_hits), MEM_DEVICE, raw=r)

    def counts(self, boxes, algo="batched", q: int | None = None, stream: int = 0,
               leaf_prefetch: int = 0, lanes_per_item: int = 0) -> np.ndarray:
        lib = load_library()
        if isinstance(boxes, np.ndarray):
            b = np.ascontiguousarray(boxes, dtype=np.float32).reshape(-1, 2 * self.dims)
            nq, ptr, bmem = b.shape[0], _ptr(b), MEM_HOST
        else:
            b, nq, ptr, bmem = boxes, q, ctypes.c_void_p(_device_ptr(boxes)), MEM_DEVICE
        out = np.zeros(nq, np.uint64)
        opts = self._opts(algo, bmem, MEM_HOST, True, stream, leaf_prefetch=leaf_prefetch,
                          lanes_per_item=lanes_per_item)
        _check(lib.qcp_query_counts(self._h, ptr, nq, ctypes.byref(opts), _ptr(out)))
        return out


    def serve(self, boxes, arrival_s, streams: int = 4, max_batch: int = 16384,
              output_cap_bytes: int = 2 << 30, collect: bool = False, trace: int = 0):
        """Replay an open-loop arrival trace through the library's continuous
        batching loop (qcp_serve_replay).  boxes: (q, 2*dims) float32 host
        array; arrival_s: non-decreasing arrival times in seconds.  Returns
        (stats dict, per-request latency in ms, per-request id arrays or
        None when collect is False).  With trace > 0, stats["trace"] holds
        the first `trace` runs as a SERVE_BATCH_DTYPE array."""
        lib = load_library()
        b = np.ascontiguousarray(boxes, dtype=np.float32).reshape(-1, 2 * self.dims)
        t = np.ascontiguousarray(arrival_s, dtype=np.float64)
        if t.shape[0] != b.shape[0]:
            raise ValueError("one arrival time per box")
        lat = np.zeros(b.shape[0], np.float32)
        got = [None] * b.shape[0] if collect else None
        opts = ServeOpts()
        opts.streams, opts.max_batch, opts.output_cap_bytes = streams, max_batch, output_cap_bytes
        tr = np.zeros(int(trace), SERVE_BATCH_DTYPE) if trace > 0 else None
        if tr is not None:
            opts.trace, opts.trace_cap = tr.ctypes.data, tr.shape[0]
        if collect:
            import threading
            lock = threading.Lock()

            def _deliver(_user, req, ids, n):
                a = np.ctypeslib.as_array(ids, shape=(int(n),)).copy() if n else np.zeros(0, np.int32)
                with lock:
                    got[req] = a
            cb = DELIVER_FN(_deliver)
            opts.deliver = cb
        st = ServeStats()
        _check(lib.qcp_serve_replay(self._h, _ptr(b), _ptr(t), b.shape[0], ctypes.byref(opts), _ptr(lat),
                                    ctypes.byref(st)))
        stats = {k: getattr(st, k) for k, _ in ServeStats._fields_ if k != "reserved_"}
        if tr is not None:
            stats["trace"] = tr[:min(int(st.batches), tr.shape[0])]
        return stats, lat, got


class _DeviceArray:
    """A device buffer described by __cuda_array_interface__ (read-only view)."""

    def __init__(self, ptr: int, n: int, typestr: str):
        self.__cuda_array_interface__ = {"shape": (n,), "typestr": typestr, "data": (ptr, False),
                                         "version": 3}


class Plan:
    """A captured query pipeline for batches of at most max_queries boxes and
    max_hits ids (qcp_plan_create).  run() returns host copies of the
    offsets and ids; run_device() the plan's device pointers."""

    def __init__(self, index: "Index", max_queries: int, max_hits: int, sort: bool = True,
                 blocks_per_sm: int = 0, win_bits: int = 0, leaf_prefetch: int = 0, lanes_per_item: int = 0):
        self.index = index
        self._h = ctypes.c_void_p()
        opts = index._opts("batched", MEM_HOST, MEM_DEVICE, sort, 0, False, blocks_per_sm, win_bits,
                           leaf_prefetch=leaf_prefetch, lanes_per_item=lanes_per_item)
        _check(load_library().qcp_plan_create(index._h, max_queries, max_hits, ctypes.byref(opts),
                                              ctypes.byref(self._h)))

    def run_device(self, boxes, q: int | None = None, stream: int = 0):
        lib = load_library()
        if isinstance(boxes, np.ndarray):
            b = np.ascontiguousarray(boxes, dtype=np.float32).reshape(-1, 2 * self.index.dims)
            nq, ptr, mem = b.shape[0], _ptr(b), MEM_HOST
        else:
            nq, ptr, mem = q, ctypes.c_void_p(_device_ptr(boxes)), MEM_DEVICE
        total = ctypes.c_uint64()
        offs, ids = ctypes.c_void_p(), ctypes.c_void_p()
        _check(lib.qcp_plan_run(self._h, ptr, nq, mem, ctypes.c_void_p(stream or None), ctypes.byref(total),
                                ctypes.byref(offs), ctypes.byref(ids)))
        return nq, int(total.value), offs.value, ids.value

    def run(self, boxes, q: int | None = None, stream: int = 0):
        import torch
        nq, total, offs, ids = self.run_device(boxes, q, stream)
        o = torch.as_tensor(_DeviceArray(offs, nq + 1, "<u8"), device="cuda").cpu().numpy().copy()
        i = (torch.as_tensor(_DeviceArray(ids, total, "<i4"), device="cuda").cpu().numpy().copy()
             if total else np.zeros(0, np.int32))
        return o, i

    def close(self):
        if self._h:
            load_library().qcp_plan_free(self._h)
            self._h = ctypes.c_void_p()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()


class BuildPlan:
    """A captured device build for n objects of one shape
    (qcp_build_plan_create): run() rebuilds the plan's index from new
    objects by one graph launch and returns it (valid until the next run
    or close; do not close it yourself)."""

    def __init__(self, n: int, dims: int, is_rect: bool = False, fanout: int = 128, key_mode: int = KEY_NORM,
                 key_bits: int = 0):
        self.n, self.dims, self.is_rect = n, dims, is_rect
        self._h = ctypes.c_void_p()
        opts = BuildOpts(fanout, key_mode, key_bits, MEM_HOST, None, 0, 0)
        _check(load_library().qcp_build_plan_create(n, dims, 1 if is_rect else 0, ctypes.byref(opts),
                                                    ctypes.byref(self._h)))

    def input_ptr(self) -> int:
        """Device address of the plan's input buffer (n rows of D or 2D floats)."""
        return int(load_library().qcp_build_plan_input(self._h) or 0)

    def run(self, objs=None, stream: int = 0) -> Index:
        """objs: a host numpy array, a CUDA tensor / device pointer, or None
        when the objects are already in input_ptr()."""
        lib = load_library()
        h = ctypes.c_void_p()
        if objs is None:
            ptr, mem = None, MEM_DEVICE
        elif isinstance(objs, np.ndarray):
            a = np.ascontiguousarray(objs, dtype=np.float32)
            if a.shape[0] != self.n:
                raise ValueError("the plan was created for a different object count")
            ptr, mem = _ptr(a), MEM_HOST
        else:
            ptr, mem = ctypes.c_void_p(_device_ptr(objs)), MEM_DEVICE
        _check(lib.qcp_build_plan_run(self._h, ptr, mem, ctypes.c_void_p(stream or None), ctypes.byref(h)))
        return Index(h, self.dims, self.is_rect, owned=False)

    def close(self) -> None:
        if self._h:
            load_library().qcp_build_plan_free(self._h)
            self._h = ctypes.c_void_p()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()


def autotune(objs, boxes, is_rect: bool = False, dims: int | None = None, key_mode: int = 0,
             repeats: int = 3) -> dict:
    """Pick the fan-out and the query knobs (blocks_per_sm, win_bits) for a
    data set and a sample of its queries by timed trials (qcp_autotune).
    Returns the choice, its batch time and every trial."""
    o = np.ascontiguousarray(objs, dtype=np.float32)
    d = dims or (o.shape[1] // 2 if is_rect else o.shape[1])
    b = np.ascontiguousarray(boxes, dtype=np.float32).reshape(-1, 2 * d)
    bo = BuildOpts()
    bo.key_mode = key_mode
    r = TuneResult()
    _check(load_library().qcp_autotune(_ptr(o), o.shape[0], d, int(is_rect), _ptr(b), b.shape[0],
                                       ctypes.byref(bo), repeats, ctypes.byref(r)))
    n = r.trials
    return {"fanout": r.fanout, "blocks_per_sm": r.blocks_per_sm, "win_bits": r.win_bits,
            "leaf_prefetch": r.leaf_prefetch, "lanes_per_item": r.lanes_per_item, "hit_cache": r.hit_cache,
            "best_ms": r.best_ms, "build_ms": r.build_ms,
            "trials": [{"fanout": r.trial_fanout[i], "blocks_per_sm": r.trial_blocks_per_sm[i],
                        "win_bits": r.trial_win_bits[i], "leaf_prefetch": r.trial_leaf_prefetch[i],
                        "lanes_per_item": r.trial_lanes_per_item[i], "hit_cache": r.trial_hit_cache[i],
                        "ms": r.trial_ms[i]} for i in range(n)]}


def last_stats() -> dict:
    """Work counters and (with timing=True) phase times of the last query
    call on this thread."""
    st = QueryStats()
    _check(load_library().qcp_query_stats_last(ctypes.byref(st)))
    d = {k: getattr(st, k) for k, _ in QueryStats._fields_ if k != "frontier_items"}
    d["frontier_items"] = list(st.frontier_items)
    return d


def launch_count(reset: bool = False) -> int:
    """Kernels this library launched on the calling thread."""
    return int(load_library().qcp_launch_count(1 if reset else 0))
