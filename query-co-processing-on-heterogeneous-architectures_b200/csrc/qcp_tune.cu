// Autotuner (qcp_autotune): picks the build fan-out and the query knobs of the
// batched pipeline for one data set and a sample of its queries by timing
// trials on the current device.
//
// The reference fixes its node size at compile time (NODE_SIZE,
// src/common/config.h) and has no tuner.  Here the fan-out is a build option
// and two query knobs are exposed through qcp_query_opts:
//   blocks_per_sm  grid of the traversal kernels (k_expand, k_leafscan) in
//                  256-thread blocks per SM; their work is fetched from a
//                  device counter, so the grid sets only how many items are
//                  in flight per SM;
//   win_bits       id window of the per-query sort (2^win_bits ids per
//                  bitmap), which trades partition fan-out against the
//                  density of the window bitmaps;
//   leaf_prefetch  the leaf tile of the traversal's leaf passes: how many
//                  partially covered leaves each warp keeps in flight in its
//                  shared-memory ring (bulk copies), or none, which trades
//                  latency hiding against CTAs per SM;
//   lanes_per_item queries per warp of the level expansion: 32, 16 or 8
//                  lanes per (query, node) item;
//   hit_cache      the count pass's leaf masks and hit bits replayed by the
//                  write pass, or both passes testing (a leaner count pass).
// Search: coordinate descent -- fan-out first (every candidate built and
// queried with default knobs), then blocks_per_sm, then win_bits, then
// leaf_prefetch, then lanes_per_item, then hit_cache, each at the best values
// found so far.  A trial is the median of `repeats` timed
// batches after one untimed batch, timed with CUDA events on the call's
// stream, sorted output left on the device.
#include <algorithm>
#include <chrono>
#include <vector>

#include "qcp_internal.cuh"

namespace {

struct Trial {
  qcp_status st = QCP_OK;
  float ms = 0.f;
};

Trial time_batch(qcp_index* ix, const float* d_boxes, uint32_t q, cudaStream_t s, uint32_t bps, uint32_t wb,
                 uint32_t lp, uint32_t lpi, uint32_t hcache, uint32_t repeats, cudaEvent_t e0, cudaEvent_t e1) {
  Trial tr;
  qcp_query_opts o;
  memset(&o, 0, sizeof(o));
  o.boxes_mem = QCP_MEM_DEVICE;
  o.result_mem = QCP_MEM_DEVICE;
  o.stream = s;
  o.blocks_per_sm = bps;
  o.win_bits = wb;
  o.leaf_prefetch = lp;
  o.lanes_per_item = lpi;
  o.hit_cache = hcache;
  std::vector<float> ms;
  for (uint32_t r = 0; r <= repeats; ++r) {
    qcp_result res;
    memset(&res, 0, sizeof(res));
    cudaEventRecord(e0, s);
    tr.st = qcp_query_batch(ix, d_boxes, q, &o, &res);
    cudaEventRecord(e1, s);
    if (tr.st != QCP_OK) return tr;
    cudaEventSynchronize(e1);
    float v = 0.f;
    cudaEventElapsedTime(&v, e0, e1);
    qcp_result_release(&res);
    if (r > 0) ms.push_back(v);  // the first batch is untimed
  }
  std::sort(ms.begin(), ms.end());
  tr.ms = ms[ms.size() / 2];
  return tr;
}

}  // namespace

extern "C" qcp_status qcp_autotune(const float* objs, uint64_t n, uint32_t dims, uint32_t is_rect,
                                   const float* boxes, uint32_t q, const qcp_build_opts* base, uint32_t repeats,
                                   qcp_tune_result* out) {
  qcp::clear_error();
  if (!objs || !boxes || !out || n == 0 || q == 0 || dims == 0 || dims > (uint32_t)qcp::kMaxDims) {
    qcp::set_error("qcp_autotune: objects, a non-empty query sample and an output struct are required");
    return QCP_ERR_BAD_ARG;
  }
  if (repeats == 0) repeats = 3;
  memset(out, 0, sizeof(*out));
  qcp_build_opts bo;
  memset(&bo, 0, sizeof(bo));
  if (base) bo = *base;
  bo.input_mem = QCP_MEM_HOST;
  cudaStream_t s = (cudaStream_t)bo.stream;
  void* d_boxes = nullptr;
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  const size_t box_bytes = sizeof(float) * 2 * dims * (size_t)q;
  QCP_CUDA(cudaMalloc(&d_boxes, box_bytes));
  qcp_status st = QCP_OK;
  qcp_index* best_ix = nullptr;
  do {
    if (cudaMemcpy(d_boxes, boxes, box_bytes, cudaMemcpyHostToDevice) != cudaSuccess ||
        cudaEventCreate(&e0) != cudaSuccess || cudaEventCreate(&e1) != cudaSuccess) {
      st = qcp::cuda_status(cudaGetLastError(), "qcp_autotune setup");
      break;
    }
    uint32_t best_lpi = 32, best_hc = 0;
    auto record = [&](uint32_t f, uint32_t b, uint32_t w, uint32_t lp, float ms) {
      if (out->trials < QCP_TUNE_MAX_TRIALS) {
        out->trial_lanes_per_item[out->trials] = best_lpi;
        out->trial_hit_cache[out->trials] = best_hc;
        out->trial_fanout[out->trials] = f;
        out->trial_blocks_per_sm[out->trials] = b;
        out->trial_win_bits[out->trials] = w;
        out->trial_leaf_prefetch[out->trials] = lp;
        out->trial_ms[out->trials] = ms;
        ++out->trials;
      }
    };
    // 1. fan-out, default knobs
    const uint32_t fanouts[] = {64, 128, 256};
    uint32_t best_f = 0, best_b = 8, best_w = qcp::kDefaultWinBits, best_lp = qcp::kDefaultLeafRing;
    float best = 0.f, best_build = 0.f;
    for (uint32_t f : fanouts) {
      bo.fanout = f;
      qcp_index* ix = nullptr;
      const auto t0 = std::chrono::steady_clock::now();
      st = qcp_index_build(objs, n, dims, is_rect, &bo, &ix);
      const float build_ms =
          std::chrono::duration<float, std::milli>(std::chrono::steady_clock::now() - t0).count();
      if (st != QCP_OK) break;
      const Trial tr = time_batch(ix, (const float*)d_boxes, q, s, best_b, best_w, best_lp, best_lpi, best_hc, repeats, e0, e1);
      if (tr.st != QCP_OK) {
        st = tr.st;
        qcp_index_free(ix);
        break;
      }
      record(f, best_b, best_w, best_lp, tr.ms);
      if (!best_ix || tr.ms < best) {
        if (best_ix) qcp_index_free(best_ix);
        best_ix = ix;
        best = tr.ms;
        best_f = f;
        best_build = build_ms;
      } else {
        qcp_index_free(ix);
      }
    }
    if (st != QCP_OK) break;
    // 2. blocks per SM, then 3. sort window bits, at the best so far
    for (uint32_t b : {4u, 16u}) {
      const Trial tr = time_batch(best_ix, (const float*)d_boxes, q, s, b, best_w, best_lp, best_lpi, best_hc, repeats, e0, e1);
      if ((st = tr.st) != QCP_OK) break;
      record(best_f, b, best_w, best_lp, tr.ms);
      if (tr.ms < best) {
        best = tr.ms;
        best_b = b;
      }
    }
    if (st != QCP_OK) break;
    const uint32_t first_w = best_w;
    for (uint32_t w : {16u, 17u, 18u}) {
      if (w == first_w) continue;
      const Trial tr = time_batch(best_ix, (const float*)d_boxes, q, s, best_b, w, best_lp, best_lpi, best_hc, repeats, e0, e1);
      if ((st = tr.st) != QCP_OK) break;
      record(best_f, best_b, w, best_lp, tr.ms);
      if (tr.ms < best) {
        best = tr.ms;
        best_w = w;
      }
    }
    if (st != QCP_OK) break;
    // 4. leaf tile: no ring (1), or 3 buffers per warp instead of 2
    for (uint32_t lp : {1u, 3u}) {
      const Trial tr = time_batch(best_ix, (const float*)d_boxes, q, s, best_b, best_w, lp, best_lpi, best_hc, repeats, e0, e1);
      if ((st = tr.st) != QCP_OK) break;
      record(best_f, best_b, best_w, lp, tr.ms);
      if (tr.ms < best) {
        best = tr.ms;
        best_lp = lp;
      }
    }
    if (st != QCP_OK) break;
    // 5. queries per warp of the level expansion
    for (uint32_t lpi : {16u, 8u}) {
      const Trial tr = time_batch(best_ix, (const float*)d_boxes, q, s, best_b, best_w, best_lp, lpi, best_hc, repeats, e0, e1);
      if ((st = tr.st) != QCP_OK) break;
      const uint32_t keep = best_lpi;
      best_lpi = lpi;
      record(best_f, best_b, best_w, best_lp, tr.ms);
      best_lpi = keep;
      if (tr.ms < best) {
        best = tr.ms;
        best_lpi = lpi;
      }
    }
    if (st != QCP_OK) break;
    // 6. the hit cache off
    {
      const Trial tr = time_batch(best_ix, (const float*)d_boxes, q, s, best_b, best_w, best_lp, best_lpi, 1u, repeats,
                                  e0, e1);
      if ((st = tr.st) != QCP_OK) break;
      best_hc = 1;
      record(best_f, best_b, best_w, best_lp, tr.ms);
      best_hc = 0;
      if (tr.ms < best) {
        best = tr.ms;
        best_hc = 1;
      }
    }
    out->hit_cache = best_hc;
    out->lanes_per_item = best_lpi;
    out->fanout = best_f;
    out->leaf_prefetch = best_lp;
    out->blocks_per_sm = best_b;
    out->win_bits = best_w;
    out->best_ms = best;
    out->build_ms = best_build;
  } while (false);
  if (best_ix) qcp_index_free(best_ix);
  if (e0) cudaEventDestroy(e0);
  if (e1) cudaEventDestroy(e1);
  cudaFree(d_boxes);
  return st;
}
