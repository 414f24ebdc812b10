// Evaluator-style driver (src/evaluator/evaluator.cpp, src/main/main.cpp):
// read a data set and a query set in the reference's binary formats, build
// the requested trees, search, and log hit totals and time per query.
//
//   qcp_eval -d <number of data, "m" suffix = millions> -q <queries>
//            -D <data file> -Q <query file> [-k dims] [-i b200|b200-plain]...
//            [-F fanout] [-r repeat] [-o hits.bin]
//
// Flags follow ParseArgs (evaluator.cpp:328-409) where they overlap; the
// reference's hard-coded data paths (:479-505) become -D/-Q.  -o writes the
// per-query hit lists: u64 query count, u64 offsets[q+1], i32 ids[].
#include <unistd.h>

#include <cstdio>
#include <cstdlib>
#include <memory>
#include <string>
#include <vector>

#include "dataset.h"
#include "tree.h"

using namespace ursus;

static void PrintHelp(const char* argv0) {
  std::fprintf(stderr,
               "Usage:\n%s -d number of data -q number of queries -D data file -Q query file\n"
               " [-k dims, default 3] [-i index type: b200 | b200-plain, repeatable]\n"
               " [-F fanout, default 128] [-r repeat, default 1] [-o hit lists file]\n",
               argv0);
}

int main(int argc, char** argv) {
  std::string n_str, data_path, query_path, out_path;
  ui nq = 0, dims = 3, repeat = 1, fanout = 128;
  std::vector<std::string> types;
  int c;
  while ((c = getopt(argc, argv, "d:D:q:Q:k:i:F:r:o:h")) != -1) {
    switch (c) {
      case 'd': n_str = optarg; break;
      case 'D': data_path = optarg; break;
      case 'q': nq = (ui)std::strtoul(optarg, nullptr, 10); break;
      case 'Q': query_path = optarg; break;
      case 'k': dims = (ui)std::strtoul(optarg, nullptr, 10); break;
      case 'i': types.push_back(optarg); break;
      case 'F': fanout = (ui)std::strtoul(optarg, nullptr, 10); break;
      case 'r': repeat = (ui)std::strtoul(optarg, nullptr, 10); break;
      case 'o': out_path = optarg; break;
      default: PrintHelp(argv[0]); return 2;
    }
  }
  if (n_str.empty() || data_path.empty()) {
    PrintHelp(argv[0]);
    return 2;
  }
  ui n = 0;
  auto m = n_str.find('m');
  if (m == std::string::npos) {
    n = (ui)std::stoul(n_str);
  } else {
    n = (ui)std::stoul(n_str.substr(0, m)) * 1000000u;
  }
  if (types.empty()) types.push_back("b200");
  try {
    auto data = std::make_shared<io::DataSet>(dims, n, data_path, DATASET_TYPE_BINARY,
                                              DATA_TYPE_SYNTHETIC, CLUSTER_TYPE_HILBERT, "no");
    std::shared_ptr<io::DataSet> queries;
    if (nq > 0) {
      if (query_path.empty()) {
        PrintHelp(argv[0]);
        return 2;
      }
      queries = std::make_shared<io::DataSet>(dims, 2 * nq, query_path, DATASET_TYPE_BINARY,
                                              DATA_TYPE_SYNTHETIC, CLUSTER_TYPE_HILBERT, "no");
    }
    std::printf(" Evaluator : \n number of data = %u\n number of searches = %u\n fanout = %u\n", n, nq,
                fanout);
    int rc = 0;
    for (const auto& t : types) {
      auto tree = tree::MakeTree(t, fanout);
      if (!tree) {
        std::fprintf(stderr, "unknown index type %s\n", t.c_str());
        return 2;
      }
      if (!tree->Build(data)) return 1;
      std::printf("Built %s\n", t.c_str());
      if (!queries) continue;
      if (!tree->Search(queries, nq, repeat)) rc = 1;
      if (!out_path.empty()) {
        auto* b = static_cast<tree::B200Index*>(tree.get());
        tree::HitLists h = b->SearchIds(queries->GetPoints(), nq);
        FILE* f = std::fopen(out_path.c_str(), "wb");
        if (!f) return 1;
        uint64_t q64 = nq;
        std::fwrite(&q64, sizeof(q64), 1, f);
        std::fwrite(h.offsets.data(), sizeof(uint64_t), h.offsets.size(), f);
        std::fwrite(h.ids.data(), sizeof(int32_t), h.ids.size(), f);
        std::fclose(f);
      }
    }
    return rc;
  } catch (const std::exception& e) {
    std::fprintf(stderr, "%s\n", e.what());
    return 1;
  }
}
