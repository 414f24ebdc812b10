// Harness around the reference implementation, compiled from the reference's
// own sources by oracle/Makefile into oracle/_ref/libqcpref_d<D>.so.
//
// TEST INFRASTRUCTURE ONLY.  It drives the reference's own classes through
// their public interface so that the tests can pin the oracle against the
// reference and bench.py can time the reference's CPU traversal.  Nothing in
// the product links it.
//
// What it exposes (extern "C", plain pointers):
//   ref_dims                 the compile-time dimension count of this build
//   ref_hilbert_keys         HilbertMapper::MappingIntoSingle per point
//                            (src/mapper/hilbert_mapper.cpp:15-68)
//   ref_bvh_build/_counts/_search_seconds/_free
//                            the CPU Hilbert-BVH (src/tree/bvh.cpp), built by
//                            the steps of BVH::Build (bvh.cpp:25-63) with the
//                            CPU branch of sort::Sorter::Sort (sorter.cpp:22-23),
//                            searched by BVH::TraverseInternalNodes
//                            (bvh.cpp:256-278) and timed through BVH::Search
//                            (bvh.cpp:165-236)
//   ref_mphr_build/_counts   the GPU MPHR tree (src/tree/mphr.cpp): MPHR::Build
//                            (:35-136) and the per-block hit counts of the MPRS
//                            kernel launched in batches as MPHR::Search does
//                            (:231-258)
//
// The reference prints its log lines on stdout; every entry point moves them
// to stderr so that the caller's stdout stays clean.

#include "io/dataset.h"
#include "mapper/hilbert_mapper.h"
#include "node/node.h"
#include "sort/parallel_sorter.h"
#include "tree/bvh.h"
#include "tree/mphr.h"

#include <cuda_runtime.h>
#include <unistd.h>

#include <chrono>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <iostream>
#include <memory>
#include <string>
#include <thread>
#include <vector>

using namespace ursus;

namespace {

// Redirect fd 1 to fd 2 for the lifetime of the object.
struct StdoutToStderr {
  int saved = -1;
  StdoutToStderr() {
    fflush(stdout);
    std::cout.flush();
    saved = dup(1);
    dup2(2, 1);
  }
  ~StdoutToStderr() {
    fflush(stdout);
    std::cout.flush();
    if (saved >= 0) {
      dup2(saved, 1);
      close(saved);
    }
  }
};

// io::DataSet only reads from a file (src/io/dataset.cpp:10-43), so inputs are
// written to a temporary file in the reference's binary format first.
std::shared_ptr<io::DataSet> MakeDataSet(const float* rows, uint64_t nrows, const char* tag) {
  char path[] = "/tmp/qcpref_XXXXXX";
  int fd = mkstemp(path);
  if (fd < 0) return nullptr;
  const size_t bytes = sizeof(float) * nrows * GetNumberOfDims();
  size_t off = 0;
  const char* p = reinterpret_cast<const char*>(rows);
  while (off < bytes) {
    ssize_t w = write(fd, p + off, bytes - off);
    if (w <= 0) {
      close(fd);
      unlink(path);
      return nullptr;
    }
    off += (size_t)w;
  }
  close(fd);
  std::shared_ptr<io::DataSet> ds(new io::DataSet(GetNumberOfDims(), (ui)nrows, path,
                                                  DATASET_TYPE_BINARY, DATA_TYPE_SYNTHETIC,
                                                  CLUSTER_TYPE_HILBERT, "yes"));
  unlink(path);
  (void)tag;
  return ds;
}

class HarnessBVH : public tree::BVH {
 public:
  bool DumpFromFile(std::string) { return false; }  // no cached index files
  bool DumpToFile(std::string) { return true; }

  // The steps of BVH::Build (bvh.cpp:37-56), sorting on the CPU.  The
  // top-down step calls Tree::CreateNode directly, which is what
  // Tree::BVH_Top_Down does (tree.cpp:113); BVH_Top_Down itself falls off the
  // end of a bool function, which current g++ compiles to a trap.
  bool BuildOnHost(std::shared_ptr<io::DataSet> ds) {
    std::vector<node::Branch> branches = CreateBranches(ds);
    AssignHilbertIndexToBranches(branches);
    sort::Parallel_Sorter::Sort(branches);
    std::vector<ui> level_node_count;
    node_ptr = CreateNode(branches, 0, (ui)branches.size() - 1, 0, level_node_count);
    host_height = (ui)level_node_count.size();
    return node_ptr != nullptr;
  }
  node::Node* Root() const { return node_ptr; }
};

class HarnessMPHR : public tree::MPHR {
 public:
  bool DumpFromFile(std::string) { return false; }
  bool DumpToFile(std::string) { return true; }
};

}  // namespace

extern "C" {

uint32_t ref_dims(void) { return GetNumberOfDims(); }

int ref_hilbert_keys(uint32_t bits, const float* pts, uint64_t n, int64_t* out) {
  const uint32_t D = GetNumberOfDims();
  std::vector<Point> p(D);
  for (uint64_t i = 0; i < n; ++i) {
    for (uint32_t d = 0; d < D; ++d) p[d] = pts[i * D + d];
    out[i] = mapper::HilbertMapper::MappingIntoSingle(D, bits, p);
  }
  return 0;
}

void* ref_bvh_build(const float* pts, uint64_t n) {
  StdoutToStderr quiet;
  auto ds = MakeDataSet(pts, n, "data");
  if (!ds) return nullptr;
  auto* t = new HarnessBVH();
  t->SetNumberOfCPUThreads(1);
  if (!t->BuildOnHost(ds)) {
    delete t;
    return nullptr;
  }
  return t;
}

// Per-query hit counts from BVH::TraverseInternalNodes, queries split over
// `threads` host threads in contiguous slices as bvh.cpp:195-220 does.
int ref_bvh_counts(void* h, const float* boxes, uint32_t q, uint32_t threads, uint32_t* counts) {
  auto* t = static_cast<HarnessBVH*>(h);
  if (!t) return -1;
  const uint32_t D2 = 2 * GetNumberOfDims();
  if (threads == 0) threads = 1;
  std::vector<std::thread> pool;
  for (uint32_t k = 0; k < threads; ++k) {
    uint32_t q0 = (uint32_t)((uint64_t)q * k / threads);
    uint32_t q1 = (uint32_t)((uint64_t)q * (k + 1) / threads);
    pool.emplace_back([=]() {
      std::vector<Point> box(D2);
      for (uint32_t i = q0; i < q1; ++i) {
        for (uint32_t d = 0; d < D2; ++d) box[d] = boxes[(uint64_t)i * D2 + d];
        ui visits = 0;
        counts[i] = t->TraverseInternalNodes(t->Root(), box.data(), &visits);
      }
    });
  }
  for (auto& th : pool) th.join();
  return 0;
}

// Wall time in seconds of the reference's own BVH::Search over q queries with
// `threads` host threads (steady_clock around the call).
double ref_bvh_search_seconds(void* h, const float* boxes, uint32_t q, uint32_t threads) {
  auto* t = static_cast<HarnessBVH*>(h);
  if (!t || q == 0) return -1.0;
  StdoutToStderr quiet;
  auto qs = MakeDataSet(boxes, 2ull * q, "query");
  if (!qs) return -1.0;
  t->SetNumberOfCPUThreads(threads ? threads : 1);
  auto t0 = std::chrono::steady_clock::now();
  t->Search(qs, q, 1);
  auto t1 = std::chrono::steady_clock::now();
  return std::chrono::duration<double>(t1 - t0).count();
}

void ref_bvh_free(void* h) {
  // Tree nodes are never freed by the reference (bvh.cpp has no destructor);
  // the handle alone is released here.
  delete static_cast<HarnessBVH*>(h);
}

void* ref_mphr_build(const float* pts, uint64_t n) {
  StdoutToStderr quiet;
  auto ds = MakeDataSet(pts, n, "data");
  if (!ds) return nullptr;
  auto* t = new HarnessMPHR();
  t->SetNumberOfCUDABlocks(128);  // the evaluator's default (evaluator.h:94)
  t->SetNumberOfPartition(1);
  t->Build(ds);
  if (cudaDeviceSynchronize() != cudaSuccess) {
    delete t;
    return nullptr;
  }
  return t;
}

// Per-query hit counts of global_RestartScanning_and_ParentCheck, launched in
// batches of 128 queries x 192 threads as MPHR::Search does (mphr.cpp:231-258);
// *ms receives the cudaEvent time of the batch loop, D2H copies included.
int ref_mphr_counts(void* h, const float* boxes, uint32_t q, uint32_t* counts, float* ms) {
  auto* t = static_cast<HarnessMPHR*>(h);
  if (!t) return -1;
  StdoutToStderr quiet;
  const uint32_t D2 = 2 * GetNumberOfDims();
  const uint32_t B = 128;
  Point* d_query = nullptr;
  ui *d_hit = nullptr, *d_root = nullptr, *d_node = nullptr;
  if (cudaMalloc(&d_query, sizeof(Point) * D2 * (size_t)(q ? q : 1)) != cudaSuccess) return -2;
  cudaMemcpy(d_query, boxes, sizeof(Point) * D2 * (size_t)q, cudaMemcpyHostToDevice);
  cudaMalloc(&d_hit, sizeof(ui) * B);
  cudaMalloc(&d_root, sizeof(ui) * B);
  cudaMalloc(&d_node, sizeof(ui) * B);
  cudaEvent_t e0, e1;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  cudaEventRecord(e0, 0);
  for (uint32_t q0 = 0; q0 < q; q0 += B) {
    uint32_t nb = (q - q0 < B) ? (q - q0) : B;
    tree::global_RestartScanning_and_ParentCheck<<<nb, GetNumberOfThreads()>>>(
        &d_query[(size_t)q0 * D2], 1, d_hit, d_root, d_node);
    const cudaError_t le = cudaGetLastError();
    if (le != cudaSuccess) {
      fprintf(stderr, "ref_mphr_counts: kernel launch failed: %s\n", cudaGetErrorString(le));
      cudaFree(d_query);
      cudaFree(d_hit);
      cudaFree(d_root);
      cudaFree(d_node);
      return -3;
    }
    cudaMemcpy(counts + q0, d_hit, sizeof(ui) * nb, cudaMemcpyDeviceToHost);
  }
  cudaEventRecord(e1, 0);
  cudaEventSynchronize(e1);
  float elapsed = 0.f;
  cudaEventElapsedTime(&elapsed, e0, e1);
  if (ms) *ms = elapsed;
  cudaError_t err = cudaGetLastError();
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  cudaFree(d_query);
  cudaFree(d_hit);
  cudaFree(d_root);
  cudaFree(d_node);
  return err == cudaSuccess ? 0 : -3;
}

void ref_mphr_free(void* h) { delete static_cast<HarnessMPHR*>(h); }

}  // extern "C"
