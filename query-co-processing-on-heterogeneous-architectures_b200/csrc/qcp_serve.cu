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
//   workers   `streams` host threads, each with its own CUDA stream and two
//             captured query plans (qcp_plan: up to 256 and up to max_batch
//             queries) whose result buffers are reserved before the clock
//             starts.  A free worker takes every pending request (up to
//             max_batch) and runs them as one plan replay; results are
//             copied to the worker's pinned buffers, handed to the deliver
//             callback, and the requests complete together.  A batch whose
//             hits do not fit its plan is split in halves and replayed; a
//             single request larger than a plan runs alone through
//             qcp_query_batch after waiting until its result bytes fit the
//             output cap next to what other workers hold.
//
// Admission by output memory: every worker's plans hold result buffers for
// at most output_cap / streams bytes of results (ids and offsets).  Every
// batch's result bytes are admitted before they are copied out: they wait
// until they fit under the cap next to what other workers hold, so the
// results held at once never exceed the cap, except for a request larger
// than the cap, which is admitted when nothing else is held and so runs
// alone.
//
// Batches on different workers overlap on the device: every worker has its
// own plans, workspace and stream.  Latency of a request = time its results
// are on the host - its arrival time.
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
  uint32_t alone_waiting = 0;  // requests above the cap waiting to run alone

  std::atomic<uint64_t> trace_next{0};  // next qcp_serve_batch record

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

constexpr uint32_t kLargePlan = 4096;  // queries of a worker's larger plan

struct WorkerRes {
  cudaStream_t stream = nullptr;
  qcp_plan* plans[2] = {nullptr, nullptr};  // small, large
  uint32_t plan_q[2] = {0, 0};
  uint64_t plan_hits = 0;
  uint64_t* h_offs = nullptr;  // pinned, plan_q[1] + 1
  int32_t* h_ids = nullptr;    // pinned, plan_hits
};

void free_res(WorkerRes& r) {
  for (qcp_plan* p : r.plans)
    if (p) qcp_plan_free(p);
  if (r.h_offs) cudaFreeHost(r.h_offs);
  if (r.h_ids) cudaFreeHost(r.h_ids);
  if (r.stream) cudaStreamDestroy(r.stream);
  r = WorkerRes();
}

// Streams, plans and pinned buffers of one worker, before the clock starts.
qcp_status make_res(ServeState& st, WorkerRes& r) {
  if (cudaStreamCreateWithFlags(&r.stream, cudaStreamNonBlocking) != cudaSuccess)
    return qcp::cuda_status(cudaGetLastError(), "serve stream");
  const uint64_t budget = st.o.output_cap_bytes / st.o.streams;  // result bytes of one worker
  r.plan_hits = budget / 16;                                       // ids: <= budget / 4 bytes
  if (r.plan_hits < 2) return QCP_OK;                              // no plans: every batch runs directly
  uint64_t qmax = budget / 16 - 1;                                 // offsets: <= budget / 2 bytes
  if (qmax > st.o.max_batch) qmax = st.o.max_batch;
  r.plan_q[0] = qmax < 256 ? (uint32_t)qmax : 256u;
  r.plan_q[1] = qmax < kLargePlan ? (uint32_t)qmax : kLargePlan;
  for (int k = 0; k < 2; ++k) {
    if (k == 1 && r.plan_q[1] == r.plan_q[0]) break;
    qcp_status s = qcp_plan_create(st.ix, r.plan_q[k], r.plan_hits, nullptr, &r.plans[k]);
    if (s != QCP_OK) return s;
  }
  if (cudaHostAlloc((void**)&r.h_offs, sizeof(uint64_t) * ((size_t)r.plan_q[1] + 1), cudaHostAllocDefault) !=
          cudaSuccess ||
      cudaHostAlloc((void**)&r.h_ids, sizeof(int32_t) * r.plan_hits, cudaHostAllocDefault) != cudaSuccess)
    return qcp::cuda_status(cudaGetLastError(), "serve pinned buffers");
  return QCP_OK;
}

struct Worker {
  ServeState& st;
  WorkerRes& r;
  std::vector<float> boxes;      // gathered boxes of the current batch
  std::vector<uint32_t> batch;   // request indices of the current batch
  std::vector<uint64_t> counts;
  uint32_t index = 0;     // worker index
  double t_taken = 0.0;   // the current batch left the queue

  // one qcp_serve_batch record, if tracing
  void record(uint32_t nb, uint32_t path, uint32_t split, uint64_t total, double t_start, double t_run,
              double t_admitted, double t_done) {
    if (!st.o.trace) return;
    const uint64_t k = st.trace_next.fetch_add(1);
    if (k >= st.o.trace_cap) return;
    qcp_serve_batch& b = st.o.trace[k];
    b.worker = index;
    b.requests = nb;
    b.path = path;
    b.split = split;
    b.hits = total;
    b.t_taken = t_taken;
    b.t_start = t_start;
    b.t_run = t_run;
    b.t_admitted = t_admitted;
    b.t_done = t_done;
  }

  void account(uint32_t nb, uint64_t total, Clock::time_point now) {
    std::lock_guard<std::mutex> g(st.mu);
    st.done += nb;
    st.hits += total;
    ++st.batches;
    st.batch_sum += nb;
    st.last_done = now;
  }

  void finish(uint32_t first, uint32_t nb, const uint64_t* offs, const int32_t* ids, Clock::time_point now) {
    const double t_done = since(st, now);
    for (uint32_t k = 0; k < nb; ++k) {
      const uint32_t req = batch[first + k];
      if (st.latency_ms) st.latency_ms[req] = (float)((t_done - st.arrival[req]) * 1e3);
      if (st.o.deliver) st.o.deliver(st.o.user, req, ids + (offs[k] - offs[0]), offs[k + 1] - offs[k]);
    }
  }

  // Admission of `bytes` of results: waits until they fit under the cap
  // next to the results other workers hold, or until nothing is held (a
  // request larger than the cap then runs alone).  False on a failure.
  bool admit(uint64_t bytes) {
    std::unique_lock<std::mutex> lk(st.mem_mu);
    if (bytes > st.o.output_cap_bytes) {
      // alone: later batches wait behind it, so that the results held drain
      ++st.alone_waiting;
      st.mem_cv.wait(lk, [&] { return st.failed.load() || st.held == 0; });
      --st.alone_waiting;
    } else {
      st.mem_cv.wait(lk, [&] {
        return st.failed.load() ||
               (st.alone_waiting == 0 && (st.held == 0 || st.held + bytes <= st.o.output_cap_bytes));
      });
    }
    if (st.failed.load()) return false;
    st.held += bytes;
    std::lock_guard<std::mutex> g(st.mu);
    st.max_held = std::max(st.max_held, st.held);
    return true;
  }

  void release(uint64_t bytes) {
    {
      std::lock_guard<std::mutex> g(st.mem_mu);
      st.held -= bytes;
    }
    st.mem_cv.notify_all();
  }

  // requests batch[first, first + nb) through a plan; false on a failure
  bool run_planned(uint32_t first, uint32_t nb, uint32_t split) {
    const uint32_t pmax = r.plans[1] ? r.plan_q[1] : r.plan_q[0];
    if (nb > pmax) {  // larger than the largest plan: consecutive chunks
      for (uint32_t c = 0; c < nb; c += pmax)
        if (!run_planned(first + c, nb - c < pmax ? nb - c : pmax, split)) return false;
      return true;
    }
    const uint32_t path = (nb <= r.plan_q[0]) ? 0u : 1u;
    qcp_plan* plan = r.plans[path];
    uint64_t total = 0;
    const uint64_t* d_offs = nullptr;
    const int32_t* d_ids = nullptr;
    const float* b = boxes.data() + (size_t)first * st.dims2;
    const double t_start = since(st, Clock::now());
    qcp_status s = qcp_plan_run(plan, b, nb, QCP_MEM_HOST, r.stream, &total, &d_offs, &d_ids);
    if (s == QCP_ERR_OUTPUT_OVERFLOW) {  // split and replay
      if (nb == 1) return run_direct(first, 1, 1);
      const uint32_t h = nb / 2;
      return run_planned(first, h, 1) && run_planned(first + h, nb - h, 1);
    }
    if (s != QCP_OK) {
      fail(st, s);
      return false;
    }
    const double t_run = since(st, Clock::now());
    const uint64_t bytes = total * 4 + ((uint64_t)nb + 1) * 8;
    if (!admit(bytes)) return false;
    const double t_admitted = since(st, Clock::now());
    if (cudaMemcpyAsync(r.h_offs, d_offs, sizeof(uint64_t) * ((size_t)nb + 1), cudaMemcpyDeviceToHost, r.stream) !=
            cudaSuccess ||
        (total && cudaMemcpyAsync(r.h_ids, d_ids, sizeof(int32_t) * total, cudaMemcpyDeviceToHost, r.stream) !=
                      cudaSuccess) ||
        cudaStreamSynchronize(r.stream) != cudaSuccess) {
      release(bytes);
      fail(st, qcp::cuda_status(cudaGetLastError(), "serve result copy"));
      return false;
    }
    const Clock::time_point now = Clock::now();
    finish(first, nb, r.h_offs, r.h_ids, now);
    release(bytes);
    account(nb, total, now);
    record(nb, path, split, total, t_start, t_run, t_admitted, since(st, now));
    return true;
  }

  // requests batch[first, first + nb) through qcp_query_batch, admitted by
  // their counted result bytes against the output cap
  bool run_direct(uint32_t first, uint32_t nb, uint32_t split) {
    qcp_query_opts qo;
    memset(&qo, 0, sizeof(qo));
    qo.stream = r.stream;
    const float* b = boxes.data() + (size_t)first * st.dims2;
    counts.resize(nb);
    const double t_start = since(st, Clock::now());
    qcp_status s = qcp_query_counts(st.ix, b, nb, &qo, counts.data());
    if (s != QCP_OK) {
      fail(st, s);
      return false;
    }
    const double t_run = since(st, Clock::now());
    uint64_t bytes = ((uint64_t)nb + 1) * 8;
    for (uint32_t k = 0; k < nb; ++k) bytes += counts[k] * 4;
    if (!admit(bytes)) return false;
    const double t_admitted = since(st, Clock::now());
    qcp_result res;
    memset(&res, 0, sizeof(res));
    s = qcp_query_batch(st.ix, b, nb, &qo, &res);
    const Clock::time_point now = Clock::now();
    if (s != QCP_OK) {
      release(bytes);
      fail(st, s);
      return false;
    }
    finish(first, nb, reinterpret_cast<const uint64_t*>(res.offsets), reinterpret_cast<const int32_t*>(res.ids),
           now);
    const uint64_t total = res.total_hits;
    qcp_result_release(&res);
    release(bytes);
    account(nb, total, now);
    record(nb, 2, split, total, t_start, t_run, t_admitted, since(st, now));
    return true;
  }

  void loop() {
    const uint32_t cap = st.o.max_batch;
    boxes.resize((size_t)cap * st.dims2);
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
        ++st.inflight;
        st.max_inflight = std::max(st.max_inflight, st.inflight);
      }
      t_taken = since(st, Clock::now());
      const uint32_t nb = (uint32_t)batch.size();
      for (uint32_t k = 0; k < nb; ++k)
        std::copy(st.boxes + (size_t)batch[k] * st.dims2, st.boxes + (size_t)(batch[k] + 1) * st.dims2,
                  boxes.begin() + (size_t)k * st.dims2);
      const bool ok = r.plans[0] ? run_planned(0, nb, 0) : run_direct(0, nb, 0);
      {
        std::lock_guard<std::mutex> g(st.mu);
        --st.inflight;
      }
      if (!ok) break;
    }
  }
};

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
  std::vector<WorkerRes> res(st.o.streams);
  for (auto& r : res) {
    const qcp_status s = make_res(st, r);
    if (s != QCP_OK) {
      const std::string msg = qcp_last_error();
      for (auto& x : res) free_res(x);
      qcp::set_error(std::string("qcp_serve_replay: ") + msg);
      return s;
    }
  }
  std::vector<std::thread> pool;
  st.t0 = Clock::now();
  st.last_done = st.t0;
  for (uint32_t w = 0; w < st.o.streams; ++w)
    pool.emplace_back([&st, &res, w, dev] {
      cudaSetDevice(dev);
      Worker wk{st, res[w], {}, {}, {}, w, 0.0};
      wk.loop();
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
  for (auto& r : res) free_res(r);
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
