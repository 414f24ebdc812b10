#!/usr/bin/env python
"""Range-search throughput benchmark.

Workload (default): 16,000,000 3-D float32 points from 64 Gaussians
(sigma 0.02, seed 1234) indexed on the device at fan-out 128; each step is
one batch of 10,000 data-centred cube queries with volumes log-uniform over
[1e-6, 1e-2] (seed 4321), answered with every query's sorted hit ids.

  value   queries/s, index and query boxes resident in HBM, results left in
          HBM (one step = qcp_query_batch over the batch)
  e2e     queries/s through the same public call with host buffers: pinned
          host boxes in, hit lists out to pinned host memory (both copies
          inside the timed region)
  plain   queries/s of the one-query-per-block traversal on the same batch

With torchrun (N ranks) every rank holds the whole index and answers its own
10,000 queries (weak scaling, no collective on the data path); times are the
max over ranks.  `--impl reference` times the reference's CPU BVH traversal
(src/tree/bvh.cpp:165-278, compiled from its sources into oracle/_ref) on
this host's cores instead.
"""
from __future__ import annotations

import argparse
import importlib.util
import json
import os
import pathlib
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = pathlib.Path(__file__).resolve().parent
PKG_DIR = ROOT / "query-co-processing-on-heterogeneous-architectures_b200"
METRIC = "range queries/sec & p99 ms, batched/served vs plain GPU traversal; HBM GB/s"
FALLBACK_HBM_GBS = 6650.0


def import_pkg():
    if "qcp_b200" in sys.modules:
        return sys.modules["qcp_b200"]
    spec = importlib.util.spec_from_file_location("qcp_b200", PKG_DIR / "__init__.py",
                                                  submodule_search_locations=[str(PKG_DIR)])
    mod = importlib.util.module_from_spec(spec)
    sys.modules["qcp_b200"] = mod
    spec.loader.exec_module(mod)
    return mod


def peaks():
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        d = json.loads(p.read_text())
        return float(d["hbm_gbs"]), "measured"
    return FALLBACK_HBM_GBS, "fallback"


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu: int):
        self.gpu = gpu
        self.proc = None
        self.out = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.gpu), f"--query-gpu={self.FIELDS}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=self.out, stderr=subprocess.DEVNULL)
        except OSError:
            self.proc = None
        time.sleep(0.3)
        return self

    def __exit__(self, *exc):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        self.out.flush()
        rows = []
        with open(self.out.name) as f:
            for line in f:
                parts = [x.strip() for x in line.split(",")]
                if len(parts) >= 9:
                    rows.append(parts)
        os.unlink(self.out.name)
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        sm = [float(r[1]) for r in rows if r[1].replace(".", "").isdigit()]
        smax = [float(r[2]) for r in rows if r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[k] for r in rows for k in range(4) if r[5 + k].lower() == "active"})
        return {"sm_mhz": float(np.median(sm)) if sm else None,
                "sm_max_mhz": max(smax) if smax else None, "reasons": reasons,
                "samples": len(rows)}


def dist_setup(n_gpus):
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return rank, world, local


def algorithmic_bytes(st: dict, dims: int, fanout: int, is_rect: bool = False, hit_cache: bool = True) -> dict:
    """Bytes each kernel must move at minimum for the work it did, per launch
    (one launch of each per step):
    k_leafscan<count>  leaf-MBR reads of every (query, leaf-parent) item +
                       coordinates of partially covered leaves (+ with the hit
                       cache, its records written: 12 B per item and 32-leaf
                       group, 16 B per partial leaf and 128-object chunk)
    k_leafscan<write>  with the hit cache: those records read back + 4 B id
                       read and 4 B id write per hit; without it the count
                       pass's MBR and coordinate reads again + 8 B per hit
    k_sort_small       4 B read + 4 B write per id of the slices <= 8192 ids
    k_win_sort         4 B read + 4 B write per id of the windows of more than
                       512 ids (the larger slices' windows)
    k_win_sort_warp    the same for their windows of at most 512 ids
    """
    mbr = st["leaf_items"] * fanout * 2 * dims * 4
    coords = st["leaves_partial"] * fanout * (2 if is_rect else 1) * dims * 4
    cache = (st["leaf_items"] * ((fanout + 31) // 32) * 12
             + st["leaves_partial"] * ((fanout + 127) // 128) * 16) if hit_cache else 0
    hits = st["hits"]
    win = st["sort_window_ids"]
    winb = st.get("sort_window_bitmap_ids", win)
    return {"count": mbr + coords + cache, "write": (cache if hit_cache else mbr + coords) + 8 * hits,
            "sort_small": 8 * (hits - win), "sort_windows": 8 * winb, "sort_windows_warp": 8 * (win - winb)}


# DRAM bytes (read + write) per id of k_win_sort measured by ncu on the
# 16M-point Gaussian workload at 2,000 queries (its windows of more than 512
# ids), applied to the ids of the timed launch: traffic grows with the ids
# processed.
K_WIN_SORT_DRAM_BYTES_PER_ID = (803071488 + 750159104) / 199061408  # 7.80 B per id

KERNEL_NAMES = {"count": "k_leafscan<count>", "write": "k_leafscan<write>",
                "sort_small": "k_sort_small", "sort_windows": "k_win_sort", "sort_windows_warp": "k_win_sort_warp"}


def roofline_of(stats, phase, steps, dims, fanout, is_rect, hbm, peak_kind, hit_cache=True):
    """HBM roofline of the step's dominant kernel: algorithmic bytes of one
    launch / that launch's CUDA-event time (the library's phase events on
    the launching stream), against the measured copy bandwidth."""
    ab = algorithmic_bytes(stats, dims, fanout, is_rect, hit_cache)
    # the window phase is two kernels: the bitmap sort (timed between its own
    # events) and the one-warp sort of the small windows (the rest)
    phase = dict(phase)
    if phase.get("sort_windows_bitmap", 0.0) > 0:
        phase["sort_windows_warp"] = max(0.0, phase["sort_windows"] - phase["sort_windows_bitmap"])
        phase["sort_windows"] = phase["sort_windows_bitmap"]
    else:
        phase["sort_windows_warp"] = 0.0
    dominant = max(KERNEL_NAMES, key=lambda k: phase[k])
    per_launch_ms = phase[dominant] / steps
    achieved = ab[dominant] / (per_launch_ms / 1e3) / 1e9 if per_launch_ms > 0 else 0.0
    traffic = None
    if dominant == "sort_windows" and K_WIN_SORT_DRAM_BYTES_PER_ID:
        traffic = int(K_WIN_SORT_DRAM_BYTES_PER_ID * stats.get("sort_window_bitmap_ids", stats["sort_window_ids"]))
    kernels_gbs = {KERNEL_NAMES[k]: round(ab[k] / (phase[k] / steps / 1e3) / 1e9, 1)
                   for k in KERNEL_NAMES if phase[k] > 0}
    return {"bound": "hbm", "kernel": KERNEL_NAMES[dominant],
            "achieved": round(achieved, 1), "peak": hbm, "unit": "GB/s",
            "frac": round(achieved / hbm, 4), "traffic": traffic,
            "peak_kind": peak_kind, "launch_ms": round(per_launch_ms, 4),
            "algorithmic_bytes_per_launch": int(ab[dominant]),
            "kernels_achieved_gbs": kernels_gbs}


class _DeviceArray:
    def __init__(self, ptr: int, n: int, typestr: str):
        self.__cuda_array_interface__ = {"shape": (n,), "typestr": typestr, "data": (int(ptr), False),
                                         "version": 3}


def verify_result(res, q, d_objs, d_boxes, dims, is_rect, chunk=1 << 24):
    """Checks of every query's id list of a device-resident result, outside
    any timed region: ids in [0, n), strictly ascending inside each slice,
    and every id passes the closed-interval predicate !(q.lo > e.hi || q.hi <
    e.lo) against its own box.  Returns (per-query counts, ids checked,
    failure text or None).  With the counts equal to an independent count
    (the reference's BVH traversal) every slice is the exact sorted hit set."""
    import torch
    offs = torch.as_tensor(_DeviceArray(res.offsets, q + 1, "<u8"), device=d_boxes.device).to(torch.int64)
    total = int(res.total_hits)
    counts = np.diff(offs.cpu().numpy()).astype(np.uint64)
    if not total:
        return counts, 0, None
    ids = torch.as_tensor(_DeviceArray(res.ids, total, "<i4"), device=d_boxes.device)
    n = d_objs.shape[0]
    ends = offs[1:].contiguous()
    for a in range(0, total, chunk):
        b = min(total, a + chunk)
        a0 = max(0, a - 1)
        seg = ids[a0:b].to(torch.int64)
        if int(seg.min()) < 0 or int(seg.max()) >= n:
            return counts, a0, f"id out of range in [{a0}, {b})"
        pos = torch.arange(a0, b, device=ids.device, dtype=torch.int64)
        qi = torch.searchsorted(ends, pos, right=True)
        bad_order = (seg[1:] <= seg[:-1]) & (qi[1:] == qi[:-1])
        if bool(bad_order.any()):
            return counts, a0, f"slice not ascending at position {int(torch.nonzero(bad_order)[0, 0]) + a0}"
        box = d_boxes[qi]
        e = d_objs[seg]
        lo_e = e[:, :dims]
        hi_e = e[:, dims:2 * dims] if is_rect else lo_e
        bad = ((box[:, :dims] > hi_e) | (box[:, dims:] < lo_e)).any(1)
        if bool(bad.any()):
            k = int(torch.nonzero(bad)[0, 0])
            return counts, a0, f"id {int(seg[k])} listed for query {int(qi[k])} fails the predicate"
    return counts, total, None


def load_workload(W, name, queries, world):
    """(workload, query boxes of all ranks) for a workload name."""
    if name == "uniform1m":
        w = W.config1()
        return w, W.fixed_cubes((queries or 1000) * world, 3, 0.0464)
    if name == "uniform2d64m":
        w = W.config3()
        q = (queries or 100_000) * world
        return w, W.fixed_cubes(q, 2, float(np.sqrt(1e-5)))
    if name == "rect8d32m":
        w = W.config4()
        return w, W.rect8d_boxes((queries or 50_000) * world)
    w = W.config2(q=(queries or 10_000) * world)
    return w, w.boxes


def tune_sample(W, name, w, n=2000):
    """A query sample of the workload's distribution, with its own seed: at
    least n queries and a fifth of the workload's batch, so that a trial's
    time is the batch's work rather than the per-call overhead."""
    n = max(n, len(w.boxes) // 5) if w.boxes is not None else n
    seed = W.QUERY_SEED + 77
    if name == "uniform1m":
        return W.fixed_cubes(n, 3, 0.0464, seed=seed)
    if name == "uniform2d64m":
        return W.fixed_cubes(n, 2, float(np.sqrt(1e-5)), seed=seed)
    if name == "rect8d32m":
        return W.rect8d_boxes(n, seed=seed)
    return W.data_centred_cubes(w.objs, n, 1e-6, 1e-2, seed=seed)


def run_ours(args, rank, world, local):
    import torch
    import torch.distributed as dist
    qcp = import_pkg()
    import qcp_b200.workloads as W

    torch.cuda.set_device(local)
    if world > 1:
        import datetime
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    dev = torch.device("cuda", local)

    # ---- workload (identical on every rank) --------------------------------
    w, boxes_all = load_workload(W, args.workload, args.queries, world)
    import qcp_b200.sharding as S
    a, b = S.query_shard(len(boxes_all), rank, world)
    boxes = np.ascontiguousarray(boxes_all[a:b])
    Q = boxes.shape[0]

    d_objs = torch.from_numpy(w.objs).to(dev)  # kept for the parity check
    d_boxes = torch.from_numpy(boxes).to(dev)
    stream = torch.cuda.current_stream(dev)
    sp = stream.cuda_stream
    torch.cuda.synchronize()

    # ---- autotune on a separate query sample of the same distribution -------
    knobs = {"fanout": args.fanout, "blocks_per_sm": args.blocks_per_sm, "win_bits": args.win_bits,
             "leaf_prefetch": args.leaf_prefetch, "lanes_per_item": args.lanes_per_item, "hit_cache": args.hit_cache}
    tune = None
    if args.algo == "batched" and not args.no_tune:
        sample = tune_sample(W, args.workload, w)
        tune = qcp.autotune(w.objs, sample, is_rect=w.is_rect, dims=w.dims, repeats=3)
        knobs = {k: tune[k] for k in ("fanout", "blocks_per_sm", "win_bits", "leaf_prefetch", "lanes_per_item",
                                      "hit_cache")}
    args.fanout = knobs["fanout"]

    t0 = time.perf_counter()
    ix = qcp.Index.build(d_objs, dims=w.dims, n=w.n, is_rect=w.is_rect, fanout=args.fanout, stream=sp)
    build_ms = (time.perf_counter() - t0) * 1e3
    hbm, peak_kind = peaks()
    build_plan = time_build_plan(qcp, w, args.fanout, d_objs, sp, hbm, peak_kind)
    info = ix.info()

    def barrier():
        if world > 1:
            dist.barrier()

    def max_over_ranks(v: float) -> float:
        if world == 1:
            return v
        t = torch.tensor([v], dtype=torch.float64, device=dev)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        return float(t.item())

    def step_device(algo, timing):
        r = ix.search(d_boxes, q=Q, algo=algo, result_mem=qcp.MEM_DEVICE, stream=sp, timing=timing,
                      blocks_per_sm=knobs["blocks_per_sm"], win_bits=knobs["win_bits"],
                    leaf_prefetch=knobs["leaf_prefetch"], lanes_per_item=knobs["lanes_per_item"],
                    hit_cache=knobs["hit_cache"])
        hits = r.total_hits
        r.release()
        return hits

    # ---- value: device-resident -------------------------------------------
    for _ in range(args.warmup):
        step_device(args.algo, True)
    barrier()
    torch.cuda.synchronize()
    qcp.launch_count(reset=True)
    phase = {"expand": 0.0, "count": 0.0, "scan": 0.0, "write": 0.0, "sort": 0.0, "total": 0.0,
             "sort_small": 0.0, "sort_partition": 0.0, "sort_windows": 0.0, "sort_windows_bitmap": 0.0}
    step_ms = []
    stats = None
    ev0 = torch.cuda.Event(enable_timing=True)
    ev1 = torch.cuda.Event(enable_timing=True)
    with ClockSampler(local) as clocks:
        ev0.record(stream)
        for _ in range(args.steps):
            e_a = torch.cuda.Event(enable_timing=True)
            e_b = torch.cuda.Event(enable_timing=True)
            e_a.record(stream)
            hits = step_device(args.algo, True)
            e_b.record(stream)
            stats = qcp.last_stats()
            for k in phase:
                phase[k] += stats[f"ms_{k}"]
            e_b.synchronize()
            step_ms.append(e_a.elapsed_time(e_b))
        ev1.record(stream)
        torch.cuda.synchronize()
    launches = qcp.launch_count()
    barrier()
    elapsed_ms = max_over_ranks(ev0.elapsed_time(ev1))
    clk = clocks.summary()
    value = world * Q * args.steps / (elapsed_ms / 1e3)

    # ---- roofline of the dominant kernel ------------------------------------
    # every candidate is ONE kernel launched once per step, timed by the
    # library's CUDA events on the launching stream
    hbm, peak_kind = peaks()
    roof = roofline_of(stats, phase, args.steps, w.dims, args.fanout, w.is_rect, hbm, peak_kind,
                       hit_cache=knobs["hit_cache"] != 1)

    # ---- parity of the timed batch (after the timed region) -----------------
    res = ix.search(d_boxes, q=Q, algo=args.algo, result_mem=qcp.MEM_DEVICE, stream=sp,
                    blocks_per_sm=knobs["blocks_per_sm"], win_bits=knobs["win_bits"],
                    leaf_prefetch=knobs["leaf_prefetch"], lanes_per_item=knobs["lanes_per_item"],
                    hit_cache=knobs["hit_cache"])
    got_counts, nchecked, fail = verify_result(res, Q, d_objs, d_boxes, w.dims, w.is_rect)
    res.release()
    parity = {"ids_checked": int(nchecked), "slices_ascending_and_in_box": fail is None}
    if fail:
        parity["failure"] = fail

    # ---- plain one-query-per-block traversal, same batch -------------------
    plain = None
    forms = None
    if args.plain_steps > 0 and args.algo != "plain":
        def qps_of(fn):
            fn()
            torch.cuda.synchronize()
            e_a = torch.cuda.Event(enable_timing=True)
            e_b = torch.cuda.Event(enable_timing=True)
            e_a.record(stream)
            for _ in range(args.plain_steps):
                fn()
            e_b.record(stream)
            e_b.synchronize()
            return world * Q * args.plain_steps / (max_over_ranks(e_a.elapsed_time(e_b)) / 1e3)

        def step_unsorted(algo):
            r = ix.search(d_boxes, q=Q, algo=algo, sort=False, result_mem=qcp.MEM_DEVICE, stream=sp,
                          blocks_per_sm=knobs["blocks_per_sm"], win_bits=knobs["win_bits"],
                    leaf_prefetch=knobs["leaf_prefetch"], lanes_per_item=knobs["lanes_per_item"],
                    hit_cache=knobs["hit_cache"])
            r.release()

        plain = qps_of(lambda: step_device("plain", False))
        # the same comparison at the output forms short of sorted ids: hit
        # sets in traversal order, and per-query counts (the form the
        # reference's plain kernel returns)
        forms = {}
        for form, fb, fp in [
                ("unsorted_hit_sets", lambda: step_unsorted(args.algo), lambda: step_unsorted("plain")),
                ("counts", lambda: ix.counts(d_boxes, q=Q, algo=args.algo, stream=sp),
                 lambda: ix.counts(d_boxes, q=Q, algo="plain", stream=sp))]:
            b_, p_ = qps_of(fb), qps_of(fp)
            forms[form] = {"batched": round(b_, 1), "plain": round(p_, 1), "speedup": round(b_ / p_, 2)}

    # ---- e2e: host buffers through the public call -------------------------
    h_boxes = torch.from_numpy(boxes).pin_memory()
    h_np = h_boxes.numpy()
    h2d = boxes.nbytes
    d2h = 0

    def step_host(st):
        r = ix.search(h_np, algo=args.algo, result_mem=qcp.MEM_HOST, stream=st.cuda_stream, copy=False,
                      blocks_per_sm=knobs["blocks_per_sm"], win_bits=knobs["win_bits"],
                    leaf_prefetch=knobs["leaf_prefetch"], lanes_per_item=knobs["lanes_per_item"],
                    hit_cache=knobs["hit_cache"])
        nb = (Q + 1) * 8 + r.total_hits * 4
        r.release()
        return nb

    # Steps run as concurrent calls on `e2e_streams` streams from as many host
    # threads (the library serves concurrent calls from separate workspaces),
    # so one step's device->host copy overlaps the next step's compute.  The
    # device clock spans all streams: every stream starts after e_a on the
    # first one, and e_b is recorded after the first one has waited for the
    # others' last work.
    import concurrent.futures as cf
    e2e_st = [torch.cuda.Stream(dev) for _ in range(max(1, args.e2e_streams))]
    pool = cf.ThreadPoolExecutor(len(e2e_st))
    # warm-up runs the calls concurrently too, all starting together (a
    # barrier), so that every concurrent call has its own workspace and
    # pinned result buffer sized before timing
    import threading
    start_together = threading.Barrier(len(e2e_st))

    def warm(st_):
        start_together.wait()
        return step_host(st_)
    for _ in range(max(2, args.warmup)):
        list(pool.map(warm, e2e_st))
    barrier()
    torch.cuda.synchronize()
    e_a = torch.cuda.Event(enable_timing=True)
    e_b = torch.cuda.Event(enable_timing=True)
    e_a.record(e2e_st[0])
    for st_ in e2e_st[1:]:
        st_.wait_event(e_a)

    def run_share(i):
        nb = 0
        for _ in range(i, args.e2e_steps, len(e2e_st)):
            nb = step_host(e2e_st[i])
        return nb
    d2h = max(pool.map(run_share, range(len(e2e_st))))
    pool.shutdown()
    for st_ in e2e_st[1:]:
        ev = torch.cuda.Event()
        ev.record(st_)
        e2e_st[0].wait_event(ev)
    e_b.record(e2e_st[0])
    e_b.synchronize()
    e2e_ms = max_over_ranks(e_a.elapsed_time(e_b))
    e2e_value = world * Q * args.e2e_steps / (e2e_ms / 1e3)

    # ---- serving: open-loop Poisson arrivals through continuous batching ----
    serving = None
    if args.serve_seconds > 0 and world == 1 and args.workload == "gauss16m":
        t_arr, s_boxes, s_cls = W.serving_stream(w.objs, rate=args.serve_rate, duration_s=args.serve_seconds)
        # warm-up: a burst at t = 0 sizes every stream's workspace for full
        # batches, then a short open-loop run
        nburst = min(len(s_boxes), 4 * 16384 * args.serve_streams)
        ix.serve(s_boxes[:nburst], np.zeros(nburst), streams=args.serve_streams, max_batch=16384)
        ix.serve(s_boxes[:20000], t_arr[:20000] - t_arr[0], streams=args.serve_streams)
        st, lat, _ = ix.serve(s_boxes, t_arr, streams=args.serve_streams, max_batch=16384,
                              output_cap_bytes=2 << 30)
        serving = {"workload": "config-2 index; Poisson %.0f req/s for %.1f s; cube volumes 1e-7/1e-5/1e-3 "
                               "at 70/25/5%%" % (args.serve_rate, args.serve_seconds),
                   "requests": int(st["requests"]), "sustained_qps": round(st["qps"], 1),
                   "p50_ms": round(st["p50_ms"], 3), "p99_ms": round(st["p99_ms"], 3),
                   "max_ms": round(st["max_ms"], 3), "mean_batch": round(st["mean_batch"], 1),
                   "batches": int(st["batches"]), "max_inflight": int(st["max_inflight"]),
                   "hits_per_request": round(st["hits"] / max(1, st["requests"]), 1),
                   "output_cap_bytes": 2 << 30, "max_output_bytes": int(st["max_output_bytes"]),
                   "streams": args.serve_streams,
                   "requests_over_10ms": int((lat > 10.0).sum()),
                   "worst_arrival_s": round(float(t_arr[int(np.argmax(lat))]), 4)}

    # ---- captured query plans (CUDA graph replay) vs qcp_query_batch ---------
    plan_out = None
    if args.plan_batches > 0 and world == 1 and args.workload == "gauss16m" and args.algo == "batched":
        plan_out = {}
        # (a) the timed batch itself through one plan
        with qcp.Plan(ix, Q, int(stats["hits"] * 1.05) + 1024, blocks_per_sm=knobs["blocks_per_sm"],
                      win_bits=knobs["win_bits"], leaf_prefetch=knobs["leaf_prefetch"],
                      lanes_per_item=knobs["lanes_per_item"]) as plan:
            plan.run_device(d_boxes, q=Q, stream=sp)
            torch.cuda.synchronize()
            e_a = torch.cuda.Event(enable_timing=True)
            e_b = torch.cuda.Event(enable_timing=True)
            e_a.record(stream)
            for _ in range(args.steps):
                plan.run_device(d_boxes, q=Q, stream=sp)
            e_b.record(stream)
            e_b.synchronize()
            pm = e_a.elapsed_time(e_b) / args.steps
        plan_out["batch"] = {"queries": Q, "ms_per_batch": round(pm, 4), "queries_per_s": round(Q / (pm / 1e3), 1),
                             "direct_ms_per_batch": round(elapsed_ms / args.steps, 4)}
        # (b) serving-sized batches: host wall time per call, both ways
        for nb in (64, 1024):
            need = nb * (args.plan_batches + 3)
            _, s_boxes, _ = W.serving_stream(w.objs, rate=args.serve_rate, duration_s=1.05 * need / args.serve_rate)
            d_sb = torch.from_numpy(np.ascontiguousarray(s_boxes[:nb * args.plan_batches])).to(dev)
            with qcp.Plan(ix, nb, 64_000_000) as plan:
                def direct(k):
                    r = ix.search(d_sb[k * nb:(k + 1) * nb], q=nb, result_mem=qcp.MEM_DEVICE, stream=sp)
                    r.release()

                def planned(k):
                    plan.run_device(d_sb[k * nb:(k + 1) * nb], q=nb, stream=sp)
                res = {}
                for name, fn in (("direct", direct), ("plan", planned)):
                    for k in range(3):
                        fn(k)
                    lat = []
                    for k in range(args.plan_batches):
                        t0 = time.perf_counter()
                        fn(k)
                        lat.append((time.perf_counter() - t0) * 1e3)
                    res[name + "_p50_ms"] = round(float(np.percentile(lat, 50)), 4)
                    res[name + "_p99_ms"] = round(float(np.percentile(lat, 99)), 4)
            plan_out[f"serving_batches_of_{nb}"] = res

    # ---- CPU + GPU co-processing (host walks the internal levels) ----------
    hybrid = None
    if args.algo == "batched" and world == 1:
        hybrid = {"cpu_threads": os.cpu_count()}
        levels = info["levels"]
        for h in sorted({1, max(1, levels - 2)}):
            ix.search(h_np, algo="hybrid", result_mem=qcp.MEM_DEVICE, stream=sp, handoff_level=h).release()
            torch.cuda.synchronize()
            e_a = torch.cuda.Event(enable_timing=True)
            e_b = torch.cuda.Event(enable_timing=True)
            e_a.record(stream)
            for _ in range(args.steps):
                ix.search(h_np, algo="hybrid", result_mem=qcp.MEM_DEVICE, stream=sp, handoff_level=h,
                          blocks_per_sm=knobs["blocks_per_sm"], win_bits=knobs["win_bits"],
                    leaf_prefetch=knobs["leaf_prefetch"], lanes_per_item=knobs["lanes_per_item"],
                    hit_cache=knobs["hit_cache"]).release()
            e_b.record(stream)
            e_b.synchronize()
            hm = e_a.elapsed_time(e_b) / args.steps
            hybrid[f"handoff_level_{h}"] = {"queries_per_s": round(Q / (hm / 1e3), 1), "ms_per_batch": round(hm, 3)}

    # ---- the reference's own GPU traversal (MPHR), same data and queries ---
    ref_gpu = None
    if args.ref_gpu and world == 1 and not w.is_rect and w.dims == 3:
        ref = _reference_lib(3)
        if ref is None:
            ref_gpu = {"unavailable": "oracle/_ref not built"}
        else:
            t0 = time.perf_counter()
            h = ref.mphr_build(w.objs)
            build_s = time.perf_counter() - t0
            _, ms = ref.mphr_counts(h, boxes)
            ref_gpu = {"kind": "reference MPHR kernel global_RestartScanning_and_ParentCheck "
                               "(src/tree/mphr.cpp:303-438) built for sm_100a; batches of 128 queries, a host "
                               "copy after each, as MPHR::Search (mphr.cpp:231-258); counts only",
                       "value": round(Q / (ms / 1e3), 1), "unit": "queries/s", "ms_per_batch": round(ms, 3),
                       "host_build_s": round(build_s, 2),
                       "counts": "not compared: the kernel sums t_hit[0..255] but zeroes only [0..191] "
                                 "(mphr.cpp:325-328), so its counts carry leftover shared memory"}
            ref_qps = Q / (ms / 1e3)
            # batched against the reference's plain kernel: sorted ids (the
            # full contract) and counts (the form that kernel returns)
            ref_gpu["speedup_batched_sorted_ids"] = round(value / ref_qps, 1)
            if forms:
                ref_gpu["speedup_batched_counts"] = round(forms["counts"]["batched"] / ref_qps, 1)

    # ---- CPU baseline (rank 0, N = 1 only) ----------------------------------
    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        if w.is_rect:
            cpu = {"value": None, "unit": "queries/s", "cores": 0, "kind": "reference",
                   "sample": "unavailable: the reference's data path loads points only"}
        else:
            cpu, bvh_counts = cpu_baseline(w.objs, boxes, args.cpu_seconds, w.dims)
            if bvh_counts is not None:
                parity["counts_vs_reference_bvh"] = compare_counts(got_counts, bvh_counts)
    if w.is_rect and args.plain_steps > 0:
        # the reference has no rectangle loader: the plain traversal counts
        parity["counts_vs_plain"] = compare_counts(got_counts, ix.counts(d_boxes, q=Q, algo="plain", stream=sp))
    if world > 1:
        bad = torch.tensor([0 if parity_ok(parity) else 1], device=dev)
        dist.all_reduce(bad, op=dist.ReduceOp.MAX)
        parity["all_ranks_ok"] = int(bad.item()) == 0

    ix.close()
    del d_objs
    torch.cuda.empty_cache()
    others = None
    if world == 1 and args.other_configs and args.workload == "gauss16m" and args.algo == "batched":
        others = {}
        for name in ("uniform2d64m", "rect8d32m"):
            others[name] = measure_other(args, qcp, W, name, dev, sp, hbm, peak_kind)

    if world > 1:
        dist.barrier()
        dist.destroy_process_group()
    if rank != 0:
        return
    lat = np.array(step_ms)
    out = {
        "metric": METRIC,
        "value": round(value, 1),
        "unit": "queries/s",
        "n_gpus": world,
        "steps": args.steps,
        "warmup": args.warmup,
        "ms_per_step": round(elapsed_ms / args.steps, 4),
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "f32",
        "data": "synthetic (seeded numpy PCG64; no public dataset)",
        "config": {
            "workload": f"{w.name}: {w.n} {w.dims}-D {'rectangles' if w.is_rect else 'points'}, "
                        f"{Q} queries per GPU per step",
            "fanout": args.fanout, "blocks_per_sm": knobs["blocks_per_sm"] or 8,
            "win_bits": knobs["win_bits"] or 17,
            "leaf_prefetch": knobs["leaf_prefetch"] or 2,
            "lanes_per_item": knobs["lanes_per_item"] or 32,
            "hit_cache": "off" if knobs["hit_cache"] == 1 else "on",
            "tuned": None if tune is None else {"sample_queries": int(len(sample)), "best_ms": round(tune["best_ms"], 3),
                                                "trial_fields": ["fanout", "blocks_per_sm", "win_bits",
                                                                 "leaf_prefetch", "lanes_per_item", "hit_cache", "ms"],
                                                "trials": [[t["fanout"], t["blocks_per_sm"], t["win_bits"],
                                                            t["leaf_prefetch"], t["lanes_per_item"], t["hit_cache"],
                                                            round(t["ms"], 3)] for t in tune["trials"]]},
            "algo": args.algo, "queries_per_step_per_gpu": Q,
            "n_objects": w.n, "key": f"hilbert {info['key_bits']} bits/dim",
            "levels": info["levels"], "index_bytes": info["device_bytes"],
            "l2": "inputs larger than L2 (index %.0f MB, %.0f MB of ids written per step)"
                  % (info["device_bytes"] / 1e6, stats["hits"] * 4 / 1e6),
            "parallelism": f"replicated index, queries sharded over {world} GPU(s)",
        },
        "batch_latency_ms": {"p50": round(float(np.percentile(lat, 50)), 3),
                             "p99": round(float(np.percentile(lat, 99)), 3)},
        "hits_per_step": int(stats["hits"]),
        "build_ms": round(build_ms, 2),
        "build_plan": build_plan,
        "phase_ms_per_step": {k: round(v / args.steps, 4) for k, v in phase.items()},
        "work_per_step": {k: stats[k] for k in ["leaf_items", "leaves_covered", "leaves_partial",
                                                 "objects_covered", "sort_small_jobs", "sort_msd_jobs",
                                                 "sort_window_ids", "sort_window_bitmap_ids"]},
        "roofline": roof,
        "parity": parity,
        "plain": {"value": round(plain, 1) if plain else None, "unit": "queries/s",
                  "speedup_batched_vs_plain": round(value / plain, 2) if plain else None,
                  "by_output_form": forms},
        "e2e": {"value": round(e2e_value, 1), "unit": "queries/s", "h2d_bytes_per_step": int(h2d),
                "d2h_bytes_per_step": int(d2h), "steps": args.e2e_steps, "concurrent_calls": len(e2e_st)},
        "gpu_launches": int(launches),
        "clocks": clk,
    }
    if serving is not None:
        out["serving"] = serving
    if plan_out is not None:
        out["plan"] = plan_out
    if ref_gpu is not None:
        out["reference_gpu"] = ref_gpu
    if hybrid is not None:
        out["hybrid"] = hybrid
    if cpu is not None:
        out["cpu_baseline"] = cpu
    if others is not None:
        out["other_configs"] = others
    print(json.dumps(out), flush=True)
    ok = parity_ok(parity) and all(parity_ok(o.get("parity", {})) for o in (others or {}).values())
    if not ok:
        print("bench: PARITY FAILED (see the parity keys of the line above)", file=sys.stderr, flush=True)
        sys.exit(3)


def time_build_plan(qcp, w, fanout, d_objs, sp, hbm, peak_kind, runs=5):
    """Device time of the captured build (qcp_build_plan_run, one graph
    launch, objects already in the plan's input buffer) and its HBM
    roofline with the algorithmic bytes of the build: keys N*(4D + 12) (read
    the coordinates, write key and id), sort 4*N*12*2 (four passes of 16-bit
    digits over key + id, read and write), packing N*(4D' + 4) read plus
    the written index (coordinates, ids, every MBR level); D' = D or 2D."""
    import torch
    stream = torch.cuda.current_stream(d_objs.device)
    with qcp.BuildPlan(w.n, w.dims, is_rect=w.is_rect, fanout=fanout, key_bits=w.key_bits) as plan:
        ix = plan.run(d_objs, stream=sp)  # objects into the plan's input buffer
        info = ix.info()
        for _ in range(2):
            plan.run(None, stream=sp)
        torch.cuda.synchronize()
        ms = []
        for _ in range(runs):
            e_a, e_b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e_a.record(stream)
            plan.run(None, stream=sp)
            e_b.record(stream)
            e_b.synchronize()
            ms.append(e_a.elapsed_time(e_b))
    n, d = w.n, w.dims
    nc = 2 * d if w.is_rect else d
    F = fanout
    npad = -(-n // F) * F
    mbr_bytes = sum(-(-k // F) * F * 2 * d * 4 for k in info["level_nodes"])
    algo = n * (4 * d + 12) + 4 * n * 12 * 2 + n * (4 * nc + 4) + npad * (4 * nc + 4) + mbr_bytes
    best = float(np.median(ms))
    gbs = algo / (best / 1e3) / 1e9
    return {"ms": round(best, 3), "runs_ms": [round(x, 3) for x in ms],
            "what": "qcp_build_plan_run: keys, radix sort, packing, MBR levels replayed as one CUDA graph, "
                    "objects resident on the device",
            "roofline": {"bound": "hbm", "achieved": round(gbs, 1), "peak": hbm, "unit": "GB/s",
                         "frac": round(gbs / hbm, 4), "peak_kind": peak_kind,
                         "algorithmic_bytes": int(algo)}}


def measure_other(args, qcp, W, name, dev, sp, hbm, peak_kind):
    """A compact line for another workload on the same GPU: tuned knobs,
    device-resident queries/s, the plain traversal, host-buffer e2e, the
    build, the dominant kernel's roofline and the parity of the batch."""
    import torch
    w, boxes = load_workload(W, name, None, 1)
    Q = len(boxes)
    stream = torch.cuda.current_stream(dev)
    d_objs = torch.from_numpy(w.objs).to(dev)
    d_boxes = torch.from_numpy(boxes).to(dev)
    knobs = {"fanout": 128, "blocks_per_sm": 0, "win_bits": 0, "leaf_prefetch": 0, "lanes_per_item": 0,
             "hit_cache": 0}
    tune = None
    if not args.no_tune:
        tune = qcp.autotune(w.objs, tune_sample(W, name, w), is_rect=w.is_rect, dims=w.dims, repeats=3)
        knobs = {k: tune[k] for k in ("fanout", "blocks_per_sm", "win_bits", "leaf_prefetch", "lanes_per_item",
                                      "hit_cache")}
    build = dict(fanout=knobs["fanout"], dims=w.dims, n=w.n, is_rect=w.is_rect, key_bits=w.key_bits, stream=sp)
    qcp.Index.build(d_objs, **build).close()  # warm-up build
    torch.cuda.synchronize()
    build_ms = []
    for _ in range(3):
        t0 = time.perf_counter()
        ixb = qcp.Index.build(d_objs, **build)
        build_ms.append((time.perf_counter() - t0) * 1e3)
        ixb.close()
    build_plan = time_build_plan(qcp, w, knobs["fanout"], d_objs, sp, hbm, peak_kind)
    ix = qcp.Index.build(d_objs, **build)
    info = ix.info()
    kq = dict(blocks_per_sm=knobs["blocks_per_sm"], win_bits=knobs["win_bits"],
                    leaf_prefetch=knobs["leaf_prefetch"], lanes_per_item=knobs["lanes_per_item"],
                    hit_cache=knobs["hit_cache"])

    def step(algo, timing=False):
        r = ix.search(d_boxes, q=Q, algo=algo, result_mem=qcp.MEM_DEVICE, stream=sp, timing=timing, **kq)
        r.release()

    def timed(algo, steps, timing=False):
        for _ in range(args.warmup):
            step(algo, timing)
        torch.cuda.synchronize()
        e_a, e_b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        phase = {"expand": 0.0, "count": 0.0, "scan": 0.0, "write": 0.0, "sort": 0.0, "total": 0.0,
                 "sort_small": 0.0, "sort_partition": 0.0, "sort_windows": 0.0, "sort_windows_bitmap": 0.0}
        e_a.record(stream)
        st = None
        for _ in range(steps):
            step(algo, timing)
            if timing:
                st = qcp.last_stats()
                for k in phase:
                    phase[k] += st[f"ms_{k}"]
        e_b.record(stream)
        e_b.synchronize()
        return e_a.elapsed_time(e_b), phase, st

    with ClockSampler(dev.index or 0) as clocks:
        ms, phase, stats = timed("batched", args.steps, timing=True)
    clk = clocks.summary()
    value = Q * args.steps / (ms / 1e3)
    roof = roofline_of(stats, phase, args.steps, w.dims, knobs["fanout"], w.is_rect, hbm, peak_kind,
                       hit_cache=knobs["hit_cache"] != 1)
    plain = None
    if args.plain_steps > 0:
        pms, _, _ = timed("plain", args.plain_steps)
        plain = Q * args.plain_steps / (pms / 1e3)
    # e2e through the public call with pinned host boxes and host hit lists
    h_np = torch.from_numpy(boxes).pin_memory().numpy()
    for _ in range(2):
        ix.search(h_np, result_mem=qcp.MEM_HOST, stream=sp, copy=False, **kq).release()
    torch.cuda.synchronize()
    e_a, e_b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e_a.record(stream)
    d2h = 0
    for _ in range(args.e2e_steps):
        r = ix.search(h_np, result_mem=qcp.MEM_HOST, stream=sp, copy=False, **kq)
        d2h = (Q + 1) * 8 + r.total_hits * 4
        r.release()
    e_b.record(stream)
    e_b.synchronize()
    e2e = Q * args.e2e_steps / (e_a.elapsed_time(e_b) / 1e3)
    # parity of the batch
    res = ix.search(d_boxes, q=Q, result_mem=qcp.MEM_DEVICE, stream=sp, **kq)
    got, nchecked, fail = verify_result(res, Q, d_objs, d_boxes, w.dims, w.is_rect)
    res.release()
    parity = {"ids_checked": int(nchecked), "slices_ascending_and_in_box": fail is None}
    if fail:
        parity["failure"] = fail
    if w.is_rect:
        parity["counts_vs_plain"] = compare_counts(got, ix.counts(d_boxes, q=Q, algo="plain", stream=sp))
        cpu = None
    else:
        cpu, want = cpu_baseline(w.objs, boxes, 0.0 if args.no_cpu_baseline else args.cpu_seconds / 3, w.dims)
        if want is not None:
            parity["counts_vs_reference_bvh"] = compare_counts(got, want)
    ix.close()
    del d_objs, d_boxes
    torch.cuda.empty_cache()
    out = {"workload": f"{w.name}: {w.n} {w.dims}-D {'rectangles' if w.is_rect else 'points'}, {Q} queries per step",
           "value": round(value, 1), "unit": "queries/s", "ms_per_step": round(ms / args.steps, 4),
           "steps": args.steps, "warmup": args.warmup, "hits_per_step": int(stats["hits"]),
           "knobs": knobs, "key": f"hilbert {info['key_bits']} bits/dim", "levels": info["levels"],
           "tuned": None if tune is None else [[t["fanout"], t["blocks_per_sm"], t["win_bits"], t["leaf_prefetch"],
                                                t["lanes_per_item"], t["hit_cache"], round(t["ms"], 3)]
                                               for t in tune["trials"]],
           "phase_ms_per_step": {k: round(v / args.steps, 4) for k, v in phase.items()},
           "roofline": roof,
           "plain": {"value": round(plain, 1) if plain else None,
                     "speedup_batched_vs_plain": round(value / plain, 2) if plain else None},
           "e2e": {"value": round(e2e, 1), "unit": "queries/s", "h2d_bytes_per_step": int(boxes.nbytes),
                   "d2h_bytes_per_step": int(d2h)},
           "build_ms": {"min": round(min(build_ms), 2), "runs": [round(x, 2) for x in build_ms],
                        "what": "qcp_index_build from device-resident objects, host wall clock, allocation included"},
           "build_plan": build_plan,
           "parity": parity, "clocks": clk}
    if cpu is not None:
        out["cpu_baseline"] = cpu
    return out


def compare_counts(got, want):
    got = np.asarray(got, dtype=np.uint64)
    want = np.asarray(want, dtype=np.uint64)
    bad = np.nonzero(got != want)[0]
    return {"queries": int(len(want)), "equal": bool(len(bad) == 0 and len(got) == len(want)),
            "mismatches": int(len(bad)), "first_mismatch": int(bad[0]) if len(bad) else None}


def parity_ok(p: dict) -> bool:
    if p.get("slices_ascending_and_in_box") is False or p.get("all_ranks_ok") is False:
        return False
    return all(v.get("equal", True) for k, v in p.items() if k.startswith("counts_vs"))


def _reference_lib(dims: int = 3):
    sys.path.insert(0, str(ROOT / "oracle"))
    from oracle import Reference  # test infrastructure: the timed reference
    if not Reference.available(dims):
        return None
    return Reference(dims)


def cpu_baseline(objs, boxes, seconds, dims=3, counts=True):
    """The reference's CPU BVH traversal on this host's cores over a bounded
    sample of the batch (as many queries as fit in about `seconds`), and
    (counts=True) the reference BVH's per-query counts of the whole batch
    (BVH::TraverseInternalNodes, src/tree/bvh.cpp:256-278) for the parity
    check.  Returns (baseline dict, counts or None)."""
    ref = _reference_lib(dims)
    if ref is None:
        return ({"value": None, "unit": "queries/s", "cores": 0, "kind": "reference",
                 "sample": "unavailable: oracle/_ref not built"}, None)
    threads = os.cpu_count() or 1
    h = ref.bvh_build(objs)
    want = None
    try:
        n = min(len(boxes), 256)
        t = ref.bvh_search_seconds(h, boxes[:n], threads)
        while seconds > 0 and t < seconds / 4 and n < len(boxes):
            n = min(len(boxes), int(n * max(2.0, seconds / max(t, 1e-3) / 2)))
            t = ref.bvh_search_seconds(h, boxes[:n], threads)
        if counts:
            want = ref.bvh_counts(h, boxes, threads)
    finally:
        ref.bvh_free(h)
    return ({"value": round(n / t, 1), "unit": "queries/s", "cores": threads, "kind": "reference",
             "sample": f"first {n} of the {len(boxes)} queries of one step, {t:.2f} s, "
                       f"BVH::Search with {threads} threads"}, want)


def run_reference(args, rank, world):
    if rank != 0:
        return
    import qcp_b200.workloads as W  # noqa: F401  (package import below)
    w, _ = load_workload(W, args.workload, args.queries, 1)
    if w.is_rect:
        print(json.dumps({"impl": "reference",
                          "unavailable": "the reference's data path loads points only; this workload is rectangles"}))
        return
    ref = _reference_lib(w.dims)
    if ref is None:
        print(json.dumps({"impl": "reference", "unavailable": "oracle/_ref/libqcpref_d3.so not built"}))
        return
    threads = os.cpu_count() or 1
    h = ref.bvh_build(w.objs)
    boxes = w.boxes
    # size one step to about args.cpu_seconds of CPU work
    n = min(len(boxes), 256)
    t = ref.bvh_search_seconds(h, boxes[:n], threads)
    while t < args.cpu_seconds / 4 and n < len(boxes):
        n = min(len(boxes), int(n * max(2.0, args.cpu_seconds / max(t, 1e-3) / 2)))
        t = ref.bvh_search_seconds(h, boxes[:n], threads)
    sample = boxes[:n]
    for _ in range(args.warmup):
        ref.bvh_search_seconds(h, sample, threads)
    times = [ref.bvh_search_seconds(h, sample, threads) for _ in range(args.steps)]
    ref.bvh_free(h)
    total = sum(times)
    value = n * len(times) / total
    print(json.dumps({
        "impl": "reference",
        "metric": METRIC, "value": round(value, 1), "unit": "queries/s", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(total / len(times) * 1e3, 3),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic (seeded numpy PCG64; no public dataset)",
        "config": {"workload": f"{w.name}: {w.n} {w.dims}-D points; each step the first {n} queries of the batch",
                   "fanout": "reference BVH, <=128 per node"},
        "cpu_baseline": {"value": round(value, 1), "unit": "queries/s", "cores": threads,
                         "kind": "reference",
                         "sample": f"{n} queries per step, BVH::Search with {threads} threads"},
        "e2e": {"value": round(value, 1), "unit": "queries/s", "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0},
    }), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--algo", default="batched", choices=["batched", "plain"])
    ap.add_argument("--workload", default="gauss16m",
                    choices=["gauss16m", "uniform1m", "uniform2d64m", "rect8d32m"],
                    help="gauss16m: 16M clustered 3-D points; uniform1m: 1M uniform 3-D points; "
                         "uniform2d64m: 64M uniform 2-D points (64-bit keys); rect8d32m: 32M 8-D rectangles")
    ap.add_argument("--queries", type=int, default=None,
                    help="queries per GPU per step (default: the workload's own count; 10,000 for gauss16m)")
    ap.add_argument("--fanout", type=int, default=128)
    ap.add_argument("--blocks-per-sm", type=int, default=0, help="traversal blocks per SM with --no-tune (0: default)")
    ap.add_argument("--win-bits", type=int, default=0, help="sort window bits with --no-tune (0: default)")
    ap.add_argument("--hit-cache", type=int, default=0, help="with --no-tune: 0 = hit cache on, 1 = off")
    ap.add_argument("--lanes-per-item", type=int, default=0,
                    help="lanes per (query, node) item of the level expansion with --no-tune (0: 32)")
    ap.add_argument("--leaf-prefetch", type=int, default=0,
                    help="leaf prefetch buffers per warp with --no-tune (0: default 2, 1: none)")
    ap.add_argument("--plain-steps", type=int, default=2)
    ap.add_argument("--e2e-steps", type=int, default=4)
    ap.add_argument("--e2e-streams", type=int, default=2,
                    help="concurrent host calls (each on its own stream) of the e2e measurement")
    ap.add_argument("--cpu-seconds", type=float, default=15.0)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-tune", action="store_true", help="skip the autotuner (use --fanout and defaults)")
    ap.add_argument("--no-ref-gpu", dest="ref_gpu", action="store_false",
                    help="skip timing the reference's MPHR GPU kernel")
    ap.add_argument("--plan-batches", type=int, default=200,
                    help="serving-sized batches timed through qcp_query_batch and a captured plan (0 = skip)")
    ap.add_argument("--serve-seconds", type=float, default=10.0,
                    help="length of the serving replay at N=1 (0 = skip)")
    ap.add_argument("--serve-rate", type=float, default=200_000.0, help="serving arrivals per second")
    ap.add_argument("--serve-streams", type=int, default=4, help="serving batches in flight")
    ap.add_argument("--no-other-configs", dest="other_configs", action="store_false",
                    help="skip the compact lines of the 64M 2-D and 32M 8-D rectangle workloads")
    args = ap.parse_args()
    if args.warmup < 3:
        ap.error("--warmup must be >= 3")
    rank, world, local = dist_setup(args.gpus)
    import_pkg()
    if args.impl == "reference":
        run_reference(args, rank, world)
    else:
        run_ours(args, rank, world, local)


if __name__ == "__main__":
    main()
