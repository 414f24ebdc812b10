#include "tree.h"

#include <chrono>
#include <cstdio>
#include <stdexcept>

namespace ursus {
namespace tree {

namespace {
void Check(qcp_status st, const char* what) {
  if (st != QCP_OK) throw std::runtime_error(std::string(what) + ": " + qcp_last_error());
}
}  // namespace

B200Index::B200Index(uint32_t fanout, qcp_algo algo) : fanout_(fanout), algo_(algo) {
  tree_type = TREE_TYPE_B200;
}

B200Index::~B200Index() {
  if (index_) qcp_index_free(index_);
}

bool B200Index::Build(std::shared_ptr<io::DataSet> ds) {
  if (!ds || ds->GetNumberOfData() == 0) return false;
  if (index_) {
    qcp_index_free(index_);
    index_ = nullptr;
  }
  qcp_build_opts opts{};
  opts.fanout = fanout_;
  opts.key_mode = QCP_KEY_NORM;
  opts.input_mem = QCP_MEM_HOST;
  dims_ = ds->GetNumberOfDims();
  qcp_status st = qcp_index_build(ds->GetPoints().data(), ds->GetNumberOfData(), dims_, 0, &opts, &index_);
  if (st != QCP_OK) {
    std::fprintf(stderr, "B200Index::Build: %s\n", qcp_last_error());
    index_ = nullptr;
    return false;
  }
  return true;
}

bool B200Index::DumpFromFile(std::string name) {
  qcp_index* ix = nullptr;
  if (qcp_index_load(name.c_str(), nullptr, &ix) != QCP_OK) return false;
  if (index_) qcp_index_free(index_);
  index_ = ix;
  qcp_index_info info{};
  qcp_index_get_info(index_, &info);
  dims_ = info.dims;
  fanout_ = info.fanout;
  return true;
}

bool B200Index::DumpToFile(std::string name) {
  return index_ && qcp_index_save(index_, name.c_str()) == QCP_OK;
}

HitLists B200Index::SearchIds(const std::vector<Point>& rows, ui number_of_search) {
  if (!index_) throw std::runtime_error("SearchIds before Build");
  const size_t w = 2 * (size_t)dims_;
  if (rows.size() < w * number_of_search) throw std::runtime_error("query set too small");
  HitLists out;
  out.offsets.assign(1, 0);
  report_ = SearchReport{};
  double ms = 0.0;
  for (ui q0 = 0; q0 < number_of_search; q0 += batch_) {
    const ui nq = (number_of_search - q0 < batch_) ? number_of_search - q0 : batch_;
    qcp_query_opts o{};
    o.algo = algo_;
    o.boxes_mem = QCP_MEM_HOST;
    o.result_mem = QCP_MEM_HOST;
    o.flags = QCP_QUERY_TIMING;
    qcp_result r{};
    Check(qcp_query_batch(index_, rows.data() + w * q0, nq, &o, &r), "qcp_query_batch");
    qcp_query_stats st{};
    qcp_query_stats_last(&st);
    ms += st.ms_total;
    const uint64_t base = out.offsets.back();
    for (ui i = 1; i <= nq; ++i) out.offsets.push_back(base + r.offsets[i]);
    out.ids.insert(out.ids.end(), r.ids, r.ids + r.total_hits);
    qcp_result_release(&r);
  }
  report_.total_hits = out.offsets.back();
  report_.avg_ms_per_query = number_of_search ? ms / number_of_search : 0.0;
  return out;
}

int B200Index::Search(std::shared_ptr<io::DataSet> qs, ui number_of_search, ui number_of_repeat) {
  if (!index_ || !qs) return 0;
  try {
    for (ui rep = 0; rep < number_of_repeat; ++rep) {
      SearchIds(qs->GetPoints(), number_of_search);
      std::printf("Hit : %llu\n", (unsigned long long)report_.total_hits);
      std::printf("Avg. Search Time on the GPU(ms) = \n%.6f\n", report_.avg_ms_per_query);
    }
  } catch (const std::exception& e) {
    std::fprintf(stderr, "B200Index::Search: %s\n", e.what());
    return 0;
  }
  return 1;
}

std::shared_ptr<Tree> MakeTree(const std::string& t, uint32_t fanout) {
  if (t == "b200" || t == "b") return std::make_shared<B200Index>(fanout, QCP_ALGO_BATCHED);
  if (t == "b200-plain" || t == "bp") return std::make_shared<B200Index>(fanout, QCP_ALGO_PLAIN);
  return nullptr;
}

}  // namespace tree
}  // namespace ursus
