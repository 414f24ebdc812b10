// Serving loop: continuous batching of an open-loop arrival trace over one
// resident index (qcp_serve_replay).
//
// The reference has no serving loop: its Evaluator runs fixed query files
// through Tree::Search (src/evaluator/evaluator.cpp:171-280).  This loop
// keeps the index resident and lets requests join the GPU as capacity frees:
//
//   feeder    the calling thread moves every request whose arrival time has
//             passed into the pending queue (open loop: arrivals never wait
//             for completions);
//   workers   `streams` host threads, each with its own CUDA stream.  A
//             free worker takes every pending request (up to max_batch),
//             counts their hits (qcp_query_counts) and admits the longest
//             prefix whose result bytes fit the output cap next to the
//             results other workers hold (at least one request, so an
//             oversized request still runs alone); the rest go back to the
//             front of the queue.  The admitted batch runs through
//             qcp_query_batch (sorted ids, copied to pinned host memory),
//             its requests complete together, results are handed to the
//             deliver callback and the batch's bytes are released.
//
// Batches on different workers overlap on the device: the library gives
// every concurrent call its own workspace and stream.  Latency of a request
// = time its results are on the host - its arrival time.
#include <algorithm>
#include <atomic>
#include <chrono>
#include <condition_variable>
#include <deque>
#include <thread>

#include "qcp_internal.cuh"

namespace {

using Clock = std::chrono::steady_clock;

struct ServeState {
  qcp_index* ix = nullptr;
  const float* boxes = nullptr;
  uint32_t dims2 = 0;  // floats per box
  const double* arrival = nullptr;
  Clock::time_point t0;
  qcp_serve_opts o{};
  float* latency_ms = nullptr;

  std::mutex mu;
  std::condition_variable cv;
  std::deque<uint32_t> pending;
  bool fed = false;         // every request has arrived
  qcp_status error = QCP_OK;
  std::string error_msg;
  std::atomic<bool> failed{false};

  std::mutex mem_mu;
  std::condition_variable mem_cv;
  uint64_t held = 0;        // result bytes admitted and not yet released

  // statistics (under mu)
  uint64_t done = 0, hits = 0, batches = 0, batch_sum = 0;
  uint32_t inflight = 0, max_inflight = 0;
  uint64_t max_held = 0;
  Clock::time_point last_done;
};

double since(const ServeState& st, Clock::time_point t) {
  return std::chrono::duration<double>(t - st.t0).count();
}

void fail(ServeState& st, qcp_status s) {
  {
    std::lock_guard<std::mutex> g(st.mu);
    if (st.error == QCP_OK) {
      st.error = s;
      st.error_msg = qcp_last_error();
    }
    st.failed = true;
    st.cv.notify_all();
  }
  std::lock_guard<std::mutex> g(st.mem_mu);
  st.mem_cv.notify_all();
}

void worker(ServeState* sp) {
  ServeState& st = *sp;
  cudaStream_t stream = nullptr;
  if (cudaStreamCreateWithFlags(&stream, cudaStreamNonBlocking) != cudaSuccess) {
    fail(st, qcp::cuda_status(cudaGetLastError(), "serve stream"));
    return;
  }
  const uint32_t cap = st.o.max_batch;
  std::vector<uint32_t> batch;
  std::vector<float> boxes((size_t)cap * st.dims2);
  std::vector<uint64_t> counts(cap);
  for (;;) {
    batch.clear();
    {
      std::unique_lock<std::mutex> lk(st.mu);
      st.cv.wait(lk, [&] { return !st.pending.empty() || st.fed || st.error != QCP_OK; });
      if (st.error != QCP_OK) break;
      if (st.pending.empty()) {
        if (st.fed) break;
        continue;
      }
      while (!st.pending.empty() && batch.size() < cap) {
        batch.push_back(st.pending.front());
        st.pending.pop_front();
      }
    }
    uint32_t nb = (uint32_t)batch.size();
    for (uint32_t k = 0; k < nb; ++k)
      std::copy(st.boxes + (size_t)batch[k] * st.dims2, st.boxes + (size_t)(batch[k] + 1) * st.dims2,
                boxes.begin() + (size_t)k * st.dims2);
    qcp_query_opts qo;
    memset(&qo, 0, sizeof(qo));
    qo.stream = stream;
    qcp_status s = qcp_query_counts(st.ix, boxes.data(), nb, &qo, counts.data());
    if (s != QCP_OK) {
      fail(st, s);
      break;
    }
    // admission by result bytes: the longest prefix that fits the cap
    uint64_t bytes = 8;
    uint32_t take = 0;
    while (take < nb) {
      const uint64_t add = counts[take] * 4 + 8;
      if (take > 0 && bytes + add > st.o.output_cap_bytes) break;
      bytes += add;
      ++take;
    }
    if (take < nb) {
      std::lock_guard<std::mutex> g(st.mu);
      for (uint32_t k = nb; k-- > take;) st.pending.push_front(batch[k]);
      st.cv.notify_all();
      nb = take;
    }
    {
      std::unique_lock<std::mutex> lk(st.mem_mu);
      st.mem_cv.wait(lk, [&] {
        return st.failed.load() || st.held == 0 || st.held + bytes <= st.o.output_cap_bytes;
      });
      if (st.failed.load()) break;
      st.held += bytes;
      std::lock_guard<std::mutex> g(st.mu);
      st.max_held = std::max(st.max_held, st.held);
      ++st.inflight;
      st.max_inflight = std::max(st.max_inflight, st.inflight);
    }
    qcp_result res;
    memset(&res, 0, sizeof(res));
    s = qcp_query_batch(st.ix, boxes.data(), nb, &qo, &res);
    const Clock::time_point now = Clock::now();
    if (s != QCP_OK) {
      {
        std::lock_guard<std::mutex> g(st.mem_mu);
        st.held -= bytes;
      }
      fail(st, s);
      break;
    }
    const double t_done = since(st, now);
    const uint64_t* offs = reinterpret_cast<const uint64_t*>(res.offsets);
    const int32_t* ids = reinterpret_cast<const int32_t*>(res.ids);
    for (uint32_t k = 0; k < nb; ++k) {
      const uint32_t r = batch[k];
      if (st.latency_ms) st.latency_ms[r] = (float)((t_done - st.arrival[r]) * 1e3);
      if (st.o.deliver) st.o.deliver(st.o.user, r, ids + offs[k], offs[k + 1] - offs[k]);
    }
    const uint64_t total = res.total_hits;
    qcp_result_release(&res);
    {
      std::lock_guard<std::mutex> g(st.mem_mu);
      st.held -= bytes;
    }
    st.mem_cv.notify_all();
    {
      std::lock_guard<std::mutex> g(st.mu);
      --st.inflight;
      st.done += nb;
      st.hits += total;
      ++st.batches;
      st.batch_sum += nb;
      st.last_done = now;
    }
  }
  cudaStreamDestroy(stream);
}

}  // namespace

extern "C" qcp_status qcp_serve_replay(qcp_index* ix, const float* boxes, const double* arrival_s, uint32_t q,
                                       const qcp_serve_opts* opts, float* latency_ms, qcp_serve_stats* stats) {
  qcp::clear_error();
  if (!ix || (!boxes && q) || (!arrival_s && q)) {
    qcp::set_error("qcp_serve_replay: index, boxes and arrival times are required");
    return QCP_ERR_BAD_ARG;
  }
  for (uint32_t i = 1; i < q; ++i) {
    if (!(arrival_s[i] >= arrival_s[i - 1])) {
      qcp::set_error("qcp_serve_replay: arrival times must be non-decreasing");
      return QCP_ERR_BAD_ARG;
    }
  }
  ServeState st;
  st.ix = ix;
  st.boxes = boxes;
  st.dims2 = 2 * ix->dims;
  st.arrival = arrival_s;
  st.latency_ms = latency_ms;
  if (opts) st.o = *opts;
  if (st.o.streams == 0) st.o.streams = 4;
  if (st.o.streams > 64) st.o.streams = 64;
  if (st.o.max_batch == 0) st.o.max_batch = 16384;
  if (st.o.output_cap_bytes == 0) st.o.output_cap_bytes = 2ull << 30;
  int dev = 0;
  cudaGetDevice(&dev);
  std::vector<std::thread> pool;
  st.t0 = Clock::now();
  st.last_done = st.t0;
  for (uint32_t w = 0; w < st.o.streams; ++w)
    pool.emplace_back([&st, dev] {
      cudaSetDevice(dev);
      worker(&st);
    });
  // feeder: open-loop arrivals
  uint32_t next = 0;
  while (next < q) {
    const double now = since(st, Clock::now());
    uint32_t end = next;
    while (end < q && arrival_s[end] <= now) ++end;
    if (end > next) {
      std::lock_guard<std::mutex> g(st.mu);
      if (st.error != QCP_OK) break;
      for (uint32_t i = next; i < end; ++i) st.pending.push_back(i);
      next = end;
      st.cv.notify_all();
      continue;
    }
    const double wait = arrival_s[next] - now;
    if (wait > 2e-4) std::this_thread::sleep_for(std::chrono::duration<double>(wait - 1e-4));
  }
  {
    std::lock_guard<std::mutex> g(st.mu);
    st.fed = true;
    st.cv.notify_all();
  }
  for (auto& t : pool) t.join();
  if (st.error != QCP_OK) {
    qcp::set_error(std::string("qcp_serve_replay: ") + st.error_msg);
    return st.error;
  }
  if (stats) {
    memset(stats, 0, sizeof(*stats));
    stats->requests = st.done;
    stats->hits = st.hits;
    stats->batches = st.batches;
    stats->mean_batch = st.batches ? (double)st.batch_sum / (double)st.batches : 0.0;
    const double first = q ? arrival_s[0] : 0.0;
    stats->seconds = since(st, st.last_done) - first;
    stats->qps = stats->seconds > 0 ? (double)st.done / stats->seconds : 0.0;
    stats->max_inflight = st.max_inflight;
    stats->max_output_bytes = st.max_held;
    if (latency_ms && q) {
      std::vector<float> l(latency_ms, latency_ms + q);
      std::sort(l.begin(), l.end());
      auto pct = [&](double p) { return (double)l[std::min<size_t>(q - 1, (size_t)(p * (q - 1) + 0.5))]; };
      stats->p50_ms = pct(0.50);
      stats->p99_ms = pct(0.99);
      stats->max_ms = l[q - 1];
      double sum = 0;
      for (float v : l) sum += v;
      stats->mean_ms = sum / q;
    }
  }
  return QCP_OK;
}
