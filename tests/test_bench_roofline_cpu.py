"""The bench's roofline accounting (bench.py), on CPU: the algorithmic bytes
of every kernel and the choice and timing of the dominant one, from a
hand-made stats record."""
from __future__ import annotations

import importlib.util

import pytest

from conftest import ROOT


@pytest.fixture(scope="module")
def bench():
    spec = importlib.util.spec_from_file_location("qcp_bench", ROOT / "bench.py")
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


STATS = {"leaf_items": 1000, "leaves_partial": 300, "hits": 10_000_000, "sort_window_ids": 9_000_000,
         "sort_window_bitmap_ids": 8_000_000}


def test_algorithmic_bytes_with_and_without_the_hit_cache(bench):
    F, D = 128, 3
    mbr = 1000 * F * 2 * D * 4
    coords = 300 * F * D * 4
    cache = 1000 * (F // 32) * 12 + 300 * 1 * 16
    ab = bench.algorithmic_bytes(STATS, D, F, False, True)
    assert ab["count"] == mbr + coords + cache
    assert ab["write"] == cache + 8 * 10_000_000
    ab0 = bench.algorithmic_bytes(STATS, D, F, False, False)
    assert ab0["count"] == mbr + coords
    assert ab0["write"] == mbr + coords + 8 * 10_000_000
    # the window phase: the bitmap kernel's ids and the one-warp sort's
    assert ab["sort_windows"] == 8 * 8_000_000
    assert ab["sort_windows_warp"] == 8 * 1_000_000
    assert ab["sort_small"] == 8 * 1_000_000
    # rectangles carry lo and hi coordinates
    assert bench.algorithmic_bytes(STATS, D, F, True, False)["count"] == mbr + 2 * coords


def test_roofline_times_the_bitmap_kernel_alone(bench):
    # two steps; the window phase 8 ms of which the bitmap kernel 6 ms
    phase = {"count": 1.0, "write": 2.0, "sort_small": 0.5, "sort_windows": 8.0, "sort_windows_bitmap": 6.0}
    r = bench.roofline_of(STATS, phase, 2, 3, 128, False, 6500.0, "measured")
    assert r["kernel"] == "k_win_sort"
    assert r["launch_ms"] == pytest.approx(3.0)
    assert r["algorithmic_bytes_per_launch"] == 8 * 8_000_000
    # achieved is reported to 0.1 GB/s, frac to 4 decimals
    assert r["achieved"] == pytest.approx(8 * 8_000_000 / 3e-3 / 1e9, abs=0.05)
    assert r["frac"] == pytest.approx(r["achieved"] / 6500.0, abs=1e-4)
    assert r["traffic"] == int(bench.K_WIN_SORT_DRAM_BYTES_PER_ID * 8_000_000)
    # the one-warp sort gets the rest of the window phase
    assert r["kernels_achieved_gbs"]["k_win_sort_warp"] == pytest.approx(8 * 1_000_000 / 1e-3 / 1e9, abs=0.05)
    # the caller's phase record is left as it was
    assert phase["sort_windows"] == 8.0


def test_roofline_without_a_bitmap_split(bench):
    # a record without the bitmap event (no window phase): the write pass dominates
    st = dict(STATS, sort_window_ids=0, sort_window_bitmap_ids=0)
    phase = {"count": 1.0, "write": 2.0, "sort_small": 0.5, "sort_windows": 0.0, "sort_windows_bitmap": 0.0}
    r = bench.roofline_of(st, phase, 1, 3, 128, False, 6500.0, "measured")
    assert r["kernel"] == "k_leafscan<write>"
    assert r["traffic"] is None
    assert "k_win_sort_warp" not in r["kernels_achieved_gbs"]
