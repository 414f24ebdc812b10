// tree::Tree with the reference's virtual interface (src/tree/tree.h:15-48),
// and B200Index, a tree type backed by the CUDA library through its C ABI
// (include/qcp.h).  B200Index takes the place of MPHR (src/tree/mphr.h)
// behind an Evaluator-style driver: Build() bulk-loads on the device and
// keeps the index resident (the role of manager::ChunkManager,
// src/manager/chunk_manager.cpp:16-40), Search() answers a query set in
// batches and logs the same totals MPHR::Search logs (src/tree/mphr.cpp:265-268),
// SearchIds() returns the per-query id lists.
#pragma once

#include <cstdint>
#include <memory>
#include <string>
#include <vector>

#include "dataset.h"
#include "qcp.h"

namespace ursus {

enum TreeType {
  TREE_TYPE_INVALID = -1,
  TREE_TYPE_HYBRID = 1,
  TREE_TYPE_MPHR = 2,
  TREE_TYPE_MPHR_PARTITION = 3,
  TREE_TYPE_BVH = 4,
  TREE_TYPE_RTREE = 5,
  TREE_TYPE_RTREE_LS = 6,
  TREE_TYPE_B200 = 7,  // this library
};

namespace tree {

class Tree {
 public:
  virtual ~Tree() = default;
  virtual bool Build(std::shared_ptr<io::DataSet> input_data_set) = 0;
  virtual bool DumpFromFile(std::string index_name) = 0;
  virtual bool DumpToFile(std::string index_name) = 0;
  virtual int Search(std::shared_ptr<io::DataSet> query_data_set, ui number_of_search,
                     ui number_of_repeat) = 0;
  TreeType GetTreeType() const { return tree_type; }

 protected:
  TreeType tree_type = TREE_TYPE_INVALID;
};

// Per-query hit lists in CSR form.
struct HitLists {
  std::vector<uint64_t> offsets;  // number_of_search + 1
  std::vector<int32_t> ids;       // ascending per query
};

struct SearchReport {
  uint64_t total_hits = 0;
  double avg_ms_per_query = 0.0;  // device time of the batches / queries
};

class B200Index : public Tree {
 public:
  explicit B200Index(uint32_t fanout = 128, qcp_algo algo = QCP_ALGO_BATCHED);
  ~B200Index() override;
  B200Index(const B200Index&) = delete;
  B200Index& operator=(const B200Index&) = delete;

  bool Build(std::shared_ptr<io::DataSet> input_data_set) override;
  bool DumpFromFile(std::string index_name) override;
  bool DumpToFile(std::string index_name) override;
  // Logs "Hit : <total>" and the average time per query; returns 1 on
  // success like the reference's Search functions, 0 on failure.
  int Search(std::shared_ptr<io::DataSet> query_data_set, ui number_of_search,
             ui number_of_repeat) override;

  // Query rows are [lo0..lo(D-1), hi0..hi(D-1)], i.e. two data-set rows per
  // query as in the reference's query files (src/io/dataset.cpp:82-88).
  HitLists SearchIds(const std::vector<Point>& query_rows, ui number_of_search);
  SearchReport last_report() const { return report_; }

  void SetAlgorithm(qcp_algo algo) { algo_ = algo; }
  void SetBatchSize(ui batch) { batch_ = batch ? batch : 1; }
  qcp_index* handle() const { return index_; }

 private:
  uint32_t fanout_;
  qcp_algo algo_;
  ui batch_ = 65536;
  ui dims_ = 0;
  qcp_index* index_ = nullptr;
  SearchReport report_;
};

// String factory in the manner of Evaluator::AddTrees (src/evaluator/evaluator.cpp:411-444):
// "b200" / "b" -> batched traversal, "b200-plain" / "bp" -> one query per block.
std::shared_ptr<Tree> MakeTree(const std::string& index_type, uint32_t fanout = 128);

}  // namespace tree
}  // namespace ursus
