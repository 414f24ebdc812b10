// qcp_query_counts_noalloc: per-query hit counts with no memory allocation.
//
// Some callers cannot call cudaMalloc while they query: a process whose
// device memory is owned by another allocator (a framework's caching
// allocator that must see every byte), a serving loop that may not take the
// device-wide synchronisation cudaMalloc/cudaFree imply, or code that has
// finished all allocation at start-up by policy.  For them this entry point
// runs the batched traversal's counting pass with its scratch (the query
// frontier, per-item counts and counters) in one fixed array of device
// memory that is part of this library's image, so a call allocates nothing;
// the caller passes the query boxes and receives the counts in its own
// device buffers.
//
// The fixed scratch costs kNoAllocScratchBytes (about 20 MiB) on every GPU
// that loads the library, for as long as the process runs.  It is shared by
// every call: calls that overlap on the GPU (several streams or host threads
// at once) race on it and must be serialised by the caller.  The counters a
// call needs at zero are cleared on the call's stream at its start.
#include <mutex>

#include "qcp_internal.cuh"

namespace qcp {

namespace {

constexpr size_t kNoAllocMaxItems = size_t(1) << 20;     // (query, node) items per frontier level
constexpr uint32_t kNoAllocMaxQueries = 1u << 18;         // queries per call

struct NoAllocScratch {
  uint2 items[2][kNoAllocMaxItems];
  uint32_t item_hits[kNoAllocMaxItems];
  uint32_t ctr[kCtrCount];
  unsigned long long stats[kStatCount];
};

constexpr size_t kNoAllocScratchBytes = sizeof(NoAllocScratch);

// The scratch itself.  In host code this name is only a handle for the
// runtime, not a device address: the address comes from cudaGetSymbolAddress.
static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocScratchBytes];

constexpr int kMaxDevices = 64;
std::mutex g_setup_mu;
void* g_scratch_addr[kMaxDevices] = {nullptr};

// Device address of the scratch on the current device, looked up once per
// device (the first call on a device does it; make that first call before
// any stream capture).
qcp_status scratch_on_current_device(NoAllocScratch** out) {
  int dev = 0;
  QCP_CUDA(cudaGetDevice(&dev));
  if (dev < 0 || dev >= kMaxDevices) {
    set_error("device ordinal beyond the no-alloc entry point's table");
    return QCP_ERR_BAD_ARG;
  }
  std::lock_guard<std::mutex> g(g_setup_mu);
  if (!g_scratch_addr[dev]) {
    void* p = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess) return cuda_status(e, "cudaGetSymbolAddress(no-alloc scratch)");
    g_scratch_addr[dev] = p;
  }
  *out = reinterpret_cast<NoAllocScratch*>(g_scratch_addr[dev]);
  return QCP_OK;
}

// Memory the kernels on `device` may read and write: device memory of that
// GPU, or managed memory.  Device memory of another GPU is refused: without
// peer access a kernel that touched it would fault.
bool is_device_pointer_on(const void* p, int device) {
  cudaPointerAttributes a;
  if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
    cudaGetLastError();
    return false;
  }
  if (a.type == cudaMemoryTypeManaged) return true;
  return a.type == cudaMemoryTypeDevice && a.device == device;
}

}  // namespace

}  // namespace qcp

using namespace qcp;

extern "C" qcp_status qcp_query_counts_noalloc(qcp_index* index, const float* d_boxes, uint32_t q,
                                               uint64_t* d_counts, void* stream) {
  clear_error();
  if (!index) {
    set_error("index is NULL");
    return QCP_ERR_BAD_ARG;
  }
  if (q == 0) return QCP_OK;
  if (q > kNoAllocMaxQueries) {
    set_error("qcp_query_counts_noalloc takes at most 262144 queries per call");
    return QCP_ERR_BAD_ARG;
  }
  int dev = 0;
  QCP_CUDA(cudaGetDevice(&dev));
  if (dev != index->device) {
    set_error("index lives on another device than the current one");
    return QCP_ERR_BAD_ARG;
  }
  if (!d_boxes || !d_counts || !is_device_pointer_on(d_boxes, dev) || !is_device_pointer_on(d_counts, dev)) {
    set_error("qcp_query_counts_noalloc needs boxes and counts in device memory of the index's device");
    return QCP_ERR_BAD_ARG;
  }
  NoAllocScratch* sc = nullptr;
  QCP_TRY(scratch_on_current_device(&sc));
  return run_batched_counts_into(index, d_boxes, q, d_counts, sc->items[0], sc->items[1], sc->item_hits,
                                 kNoAllocMaxItems, sc->ctr, sc->stats, (cudaStream_t)stream);
}
