"""Shared test setup.

Tests marked `gpu` need a CUDA device and call the library through its C ABI;
everything else runs on the CPU (oracle against the golden vectors, library
exports, host logic).
"""
from __future__ import annotations

import importlib.util
import pathlib
import subprocess
import sys

import numpy as np
import pytest

ROOT = pathlib.Path(__file__).resolve().parent.parent
PKG_DIR = ROOT / "query-co-processing-on-heterogeneous-architectures_b200"
GOLDEN = ROOT / "tests" / "golden"

sys.path.insert(0, str(ROOT / "oracle"))
sys.path.insert(0, str(GOLDEN))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200)")


def load_pkg():
    """Import the package directory (its name is not a Python identifier)."""
    if "qcp_b200" in sys.modules:
        return sys.modules["qcp_b200"]
    spec = importlib.util.spec_from_file_location("qcp_b200", PKG_DIR / "__init__.py",
                                                  submodule_search_locations=[str(PKG_DIR)])
    mod = importlib.util.module_from_spec(spec)
    sys.modules["qcp_b200"] = mod
    spec.loader.exec_module(mod)
    return mod


def ensure_library() -> pathlib.Path:
    lib = PKG_DIR / "libqcp_b200.so"
    if not lib.exists():
        subprocess.run(["make", "-s", "-j4", "-C", str(PKG_DIR)], check=True)
    return lib


@pytest.fixture(scope="session")
def qcp():
    ensure_library()
    return load_pkg()


@pytest.fixture(scope="session")
def workloads():
    load_pkg()
    import qcp_b200.workloads as w  # noqa: E402
    return w


@pytest.fixture(scope="session")
def oracle():
    from oracle import Oracle
    return Oracle()


@pytest.fixture(scope="session")
def cases():
    import cases as c
    return c


def golden(name: str):
    return np.load(GOLDEN / name)


class DeviceArray:
    """A non-owning view of library-owned device memory for torch.as_tensor."""

    def __init__(self, ptr: int, n: int, typestr: str):
        self.__cuda_array_interface__ = {"shape": (n,), "typestr": typestr, "data": (int(ptr), False),
                                         "version": 3}


def device_result(res, q: int):
    """(offsets int64, ids int32) torch tensors viewing a MEM_DEVICE result."""
    import torch
    offs = torch.as_tensor(DeviceArray(res.offsets, q + 1, "<u8"), device="cuda").to(torch.int64)
    if res.total_hits:
        ids = torch.as_tensor(DeviceArray(res.ids, res.total_hits, "<i4"), device="cuda")
    else:
        ids = torch.zeros(0, dtype=torch.int32, device="cuda")
    return offs, ids


def verify_all_slices(offs, ids, d_objs, d_boxes, dims: int, is_rect: bool, chunk: int = 1 << 24):
    """Size-independent checks of every query's id list of a device result:
    ids in [0, n), strictly ascending inside each slice (so distinct), and
    every id passes the closed-interval predicate !(q.lo > e.hi || q.hi < e.lo)
    against its own query box.  With per-query counts equal to an
    independent count this proves each slice IS the sorted hit set.
    Returns the number of ids checked."""
    import torch
    n = d_objs.shape[0]
    total = ids.shape[0]
    ends = offs[1:].contiguous()
    for a in range(0, total, chunk):
        b = min(total, a + chunk)
        a0 = max(0, a - 1)  # one id of overlap: ascending across chunk edges
        seg = ids[a0:b].to(torch.int64)
        if int(seg.min()) < 0 or int(seg.max()) >= n:
            raise AssertionError(f"ids out of range in [{a0}, {b})")
        pos = torch.arange(a0, b, device=ids.device, dtype=torch.int64)
        qi = torch.searchsorted(ends, pos, right=True)
        same = qi[1:] == qi[:-1]
        if bool(((seg[1:] <= seg[:-1]) & same).any()):
            k = int(torch.nonzero((seg[1:] <= seg[:-1]) & same)[0, 0]) + a0
            raise AssertionError(f"slice not strictly ascending at position {k} (query {int(qi[k - a0])})")
        box = d_boxes[qi]
        e = d_objs[seg]
        lo_e = e[:, :dims]
        hi_e = e[:, dims:2 * dims] if is_rect else lo_e
        bad = ((box[:, :dims] > hi_e) | (box[:, dims:] < lo_e)).any(1)
        if bool(bad.any()):
            k = int(torch.nonzero(bad)[0, 0])
            raise AssertionError(f"id {int(seg[k])} listed for query {int(qi[k])} fails the predicate")
    return total


def sample_queries(counts: np.ndarray, k: int, largest: int = 20, seed: int = 5) -> np.ndarray:
    """The `largest` queries with the most hits plus seeded random ones, k in all."""
    q = len(counts)
    top = np.argsort(counts, kind="stable")[::-1][:largest]
    rest = np.setdiff1d(np.arange(q), top)
    rng = np.random.Generator(np.random.PCG64(seed))
    pick = rng.choice(rest, size=min(len(rest), max(0, k - len(top))), replace=False)
    return np.sort(np.concatenate([top, pick]))


def sample_ids(offs, ids, sample: np.ndarray):
    """(offsets, concatenated ids) of the sampled queries' slices, on the host."""
    import torch
    o = offs.cpu().numpy()
    parts = [ids[int(o[i]):int(o[i + 1])] for i in sample]
    cat = torch.cat(parts).cpu().numpy() if parts else np.zeros(0, np.int32)
    so = np.zeros(len(sample) + 1, np.uint64)
    so[1:] = np.cumsum([int(o[i + 1] - o[i]) for i in sample])
    return so, cat


def assert_same_hits(res_offsets, res_ids, ref_offsets, ref_ids, boxes=None):
    """Per-query sorted id lists equal (bit-exact)."""
    res_offsets = np.asarray(res_offsets, dtype=np.uint64)
    ref_offsets = np.asarray(ref_offsets, dtype=np.uint64)
    if not np.array_equal(res_offsets, ref_offsets):
        cr, co = np.diff(res_offsets.astype(np.int64)), np.diff(ref_offsets.astype(np.int64))
        bad = np.nonzero(cr != co)[0]
        raise AssertionError(f"{len(bad)} queries differ in hit count; first {bad[:5]}: "
                             f"got {cr[bad[:5]]} want {co[bad[:5]]}"
                             + (f" boxes {boxes[bad[:2]]}" if boxes is not None else ""))
    if not np.array_equal(np.asarray(res_ids), np.asarray(ref_ids)):
        diff = np.nonzero(np.asarray(res_ids) != np.asarray(ref_ids))[0]
        q = np.searchsorted(res_offsets, diff[0], side="right") - 1
        raise AssertionError(f"ids differ at {len(diff)} positions, first in query {q}")
