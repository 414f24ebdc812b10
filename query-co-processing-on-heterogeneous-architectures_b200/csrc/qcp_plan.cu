// Query plans: the batched pipeline for a fixed batch size, captured once
// into a CUDA graph and replayed (qcp_plan_create / qcp_plan_run).
//
// qcp_query_batch decides buffer sizes and launch shapes on the host between
// its phases (one readback after counting, one after classifying the slices,
// one for the tile count).  A plan fixes them up front instead -- at most
// max_queries boxes, at most max_hits ids -- so the whole pipeline (frontier
// expansion, count, scan, write, per-query sort) runs from device-resident
// counts with fixed grids (run_batched_device) and is captured into one
// graph.  A run copies the boxes in, pads the batch with empty boxes (no
// object overlaps lo = +inf, hi = -inf), launches the graph, and reads back
// one counter block and the hit total.  Overflows of the item frontier or of
// max_hits are flagged on the device and returned as
// QCP_ERR_OUTPUT_OVERFLOW; nothing is written out of bounds.
//
// The reference launches one kernel per 128 queries with a host
// synchronisation between launches (MPHR::Search, src/tree/mphr.cpp:231-258).
#include <cmath>
#include <vector>

#include "qcp_internal.cuh"

struct qcp_plan {
  qcp_index* ix = nullptr;
  qcp::Workspace* ws = nullptr;
  uint32_t max_q = 0;
  uint64_t max_hits = 0;
  bool sort = true;
  void* tables = nullptr;
  float* empty = nullptr;  // max_q empty boxes
  cudaStream_t capture = nullptr;
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
};

namespace {

void plan_destroy(qcp_plan* p) {
  if (!p) return;
  if (p->exec) cudaGraphExecDestroy(p->exec);
  if (p->graph) cudaGraphDestroy(p->graph);
  if (p->capture) cudaStreamDestroy(p->capture);
  cudaFree(p->tables);
  cudaFree(p->empty);
  if (p->ws) qcp::ws_destroy(p->ws, p->ix);
  delete p;
}

}  // namespace

extern "C" qcp_status qcp_plan_create(qcp_index* ix, uint32_t max_queries, uint64_t max_hits,
                                      const qcp_query_opts* opts, qcp_plan** out) {
  using namespace qcp;
  clear_error();
  if (!ix || !out || max_queries == 0 || max_hits == 0) {
    set_error("qcp_plan_create: index, a batch size and a hit capacity are required");
    return QCP_ERR_BAD_ARG;
  }
  if (opts && opts->algo != QCP_ALGO_BATCHED) {
    set_error("qcp_plan_create: plans run the batched traversal only");
    return QCP_ERR_BAD_ARG;
  }
  if (max_hits >= (1ull << 40)) {
    set_error("qcp_plan_create: max_hits is out of range");
    return QCP_ERR_BAD_ARG;
  }
  *out = nullptr;
  qcp_plan* p = new (std::nothrow) qcp_plan();
  if (!p) return QCP_ERR_OOM;
  p->ix = ix;
  p->max_q = max_queries;
  p->max_hits = max_hits;
  p->sort = !(opts && opts->unsorted);
  p->ws = new (std::nothrow) Workspace();
  if (!p->ws) {
    delete p;
    return QCP_ERR_OOM;
  }
  Workspace* ws = p->ws;
  ws->blocks_per_sm = (opts && opts->blocks_per_sm) ? (opts->blocks_per_sm > 32 ? 32u : opts->blocks_per_sm) : 8u;
  ws->win_bits = (opts && opts->win_bits) ? (opts->win_bits < 12 ? 12u : opts->win_bits) : kDefaultWinBits;
  ws->leaf_ring = leaf_ring_of(opts ? opts->leaf_prefetch : 0u);
  ws->lanes_per_item = lanes_per_item_of(opts ? opts->lanes_per_item : 0u);
  qcp_status st = QCP_OK;
  do {
    const size_t row = 2 * (size_t)ix->dims;
    if ((st = ws_reserve_queries(ix, ws, max_queries)) != QCP_OK) break;
    // (query, node) items per frontier: 64 per query plus one per 1024 hits
    if ((st = ws_reserve_items(ix, ws, (size_t)max_queries * 64 + (size_t)(max_hits >> 10) + (1u << 16))) != QCP_OK)
      break;
    if ((st = ws_reserve_out(ix, ws, (size_t)max_hits)) != QCP_OK) break;
    if ((st = ws_reserve_sort(ix, ws, (size_t)max_queries + 256, (size_t)(max_hits / kSortTile) + max_queries + 1)) !=
        QCP_OK)
      break;
    if (p->sort) {  // the write pass gathers the sort's per-window counts
      uint32_t wbits = 0, G = 0;
      sort_window_shape(ix, ws, &wbits, &G);
      if (G <= kHistMaxG) {
        if ((st = ws_reserve_qwhist(ws, (size_t)max_queries * G)) != QCP_OK) break;
        ws->hist_G = G;
        ws->hist_bits = wbits;
      }
    }
    // scan scratch owned by the workspace: no stream-ordered temporaries in the graph
    ws->scan_tmp_cap = scan_scratch_bytes((uint64_t)max_queries + 1);
    if (cudaMalloc(&ws->scan_tmp, ws->scan_tmp_cap) != cudaSuccess ||
        cudaMalloc(&p->tables, sort_tables_bytes(ix, ws, max_queries)) != cudaSuccess ||
        cudaMalloc(&p->empty, sizeof(float) * row * max_queries) != cudaSuccess) {
      st = cuda_status(cudaGetLastError(), "qcp_plan_create");
      break;
    }
    std::vector<float> e(row * max_queries);
    for (size_t i = 0; i < e.size(); ++i) e[i] = (i % row) < ix->dims ? INFINITY : -INFINITY;
    if (cudaMemcpy(p->empty, e.data(), sizeof(float) * e.size(), cudaMemcpyHostToDevice) != cudaSuccess ||
        cudaStreamCreateWithFlags(&p->capture, cudaStreamNonBlocking) != cudaSuccess ||
        cudaMemcpyAsync(ws->boxes, p->empty, sizeof(float) * e.size(), cudaMemcpyDeviceToDevice, p->capture) !=
            cudaSuccess) {
      st = cuda_status(cudaGetLastError(), "qcp_plan_create");
      break;
    }
    // one plain run first: kernel attributes are set up outside the capture
    if ((st = run_batched_device(ix, ws, max_queries, max_hits, p->sort, p->tables, p->capture)) != QCP_OK) break;
    if (cudaStreamSynchronize(p->capture) != cudaSuccess) {
      st = cuda_status(cudaGetLastError(), "qcp_plan_create warm-up");
      break;
    }
    if (cudaStreamBeginCapture(p->capture, cudaStreamCaptureModeThreadLocal) != cudaSuccess) {
      st = cuda_status(cudaGetLastError(), "qcp_plan_create capture");
      break;
    }
    const qcp_status cs = run_batched_device(ix, ws, max_queries, max_hits, p->sort, p->tables, p->capture);
    const cudaError_t ce = cudaStreamEndCapture(p->capture, &p->graph);
    if (cs != QCP_OK) {
      st = cs;
      break;
    }
    if (ce != cudaSuccess) {
      st = cuda_status(cudaGetLastError(), "qcp_plan_create graph");
      break;
    }
    // the pipeline must not allocate inside the graph: the physical memory of
    // a graph memory node is mapped at whichever launch first needs more of
    // it than the graphs already running hold, which stalled replays of
    // concurrent plans for hundreds of milliseconds
    {
      size_t nn = 0;
      std::vector<cudaGraphNode_t> nodes;
      if (cudaGraphGetNodes(p->graph, nullptr, &nn) == cudaSuccess) {
        nodes.resize(nn);
        if (nn && cudaGraphGetNodes(p->graph, nodes.data(), &nn) != cudaSuccess) nn = 0;
      }
      bool mem_node = false;
      for (size_t k = 0; k < nn; ++k) {
        cudaGraphNodeType ty;
        if (cudaGraphNodeGetType(nodes[k], &ty) == cudaSuccess &&
            (ty == cudaGraphNodeTypeMemAlloc || ty == cudaGraphNodeTypeMemFree))
          mem_node = true;
      }
      if (mem_node) {
        set_error("qcp_plan_create: the captured pipeline holds a memory allocation node");
        st = QCP_ERR_CUDA;
        break;
      }
    }
    if (cudaGraphInstantiate(&p->exec, p->graph, 0) != cudaSuccess) {
      st = cuda_status(cudaGetLastError(), "qcp_plan_create graph");
      break;
    }
    // one replay of the empty batch (ws->boxes still holds it): the graph's
    // first launch uploads it, which would otherwise land on the first real
    // batch
    if (cudaGraphLaunch(p->exec, p->capture) != cudaSuccess || cudaStreamSynchronize(p->capture) != cudaSuccess) {
      st = cuda_status(cudaGetLastError(), "qcp_plan_create first replay");
      break;
    }
  } while (false);
  if (st != QCP_OK) {
    cudaStreamSynchronize(p->capture);
    plan_destroy(p);
    return st;
  }
  *out = p;
  return QCP_OK;
}

extern "C" qcp_status qcp_plan_run(qcp_plan* p, const float* boxes, uint32_t q, uint32_t boxes_mem, void* stream,
                                   uint64_t* total_hits, const uint64_t** d_offsets, const int32_t** d_ids) {
  using namespace qcp;
  clear_error();
  if (!p || (q && !boxes) || q > p->max_q) {
    set_error("qcp_plan_run: plan and boxes are required, at most the plan's batch size");
    return QCP_ERR_BAD_ARG;
  }
  Workspace* ws = p->ws;
  cudaStream_t s = (cudaStream_t)stream;
  const size_t row = 2 * (size_t)p->ix->dims;
  if (q) {
    QCP_CUDA(cudaMemcpyAsync(ws->boxes, boxes, sizeof(float) * row * q,
                             boxes_mem == QCP_MEM_DEVICE ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice, s));
  }
  if (q < p->max_q)
    QCP_CUDA(cudaMemcpyAsync(ws->boxes + row * q, p->empty + row * q, sizeof(float) * row * (p->max_q - q),
                             cudaMemcpyDeviceToDevice, s));
  QCP_CUDA(cudaGraphLaunch(p->exec, s));
  note_launch();
  QCP_CUDA(cudaMemcpyAsync(ws->h_ctr, ws->ctr, sizeof(uint32_t) * kCtrCount, cudaMemcpyDeviceToHost, s));
  QCP_CUDA(cudaMemcpyAsync(ws->h_total, ws->offsets + q, sizeof(uint64_t), cudaMemcpyDeviceToHost, s));
  QCP_CUDA(cudaStreamSynchronize(s));
  if (ws->h_ctr[kCtrTimeout]) {
    set_error("qcp_plan_run: a bounded wait for a leaf's bulk copy ran out");
    return QCP_ERR_TIMEOUT;
  }
  const uint32_t flags = ws->h_ctr[kCtrOverflow];
  if (flags & 1u) {
    set_error("qcp_plan_run: the batch's traversal frontier exceeded the plan's item capacity");
    return QCP_ERR_OUTPUT_OVERFLOW;
  }
  if (flags & 2u) {
    set_error("qcp_plan_run: the batch has more hits than the plan's max_hits");
    return QCP_ERR_OUTPUT_OVERFLOW;
  }
  if (total_hits) *total_hits = *ws->h_total;
  if (d_offsets) *d_offsets = ws->offsets;
  if (d_ids) *d_ids = ws->out_ids;
  return QCP_OK;
}

extern "C" qcp_status qcp_plan_free(qcp_plan* p) {
  qcp::clear_error();
  if (!p) return QCP_OK;
  cudaDeviceSynchronize();
  plan_destroy(p);
  return QCP_OK;
}
