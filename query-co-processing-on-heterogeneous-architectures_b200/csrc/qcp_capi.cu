// C ABI: index lifecycle, device/pinned pools, per-call workspaces, query
// entry points, index files.  Every function returns a qcp_status and records
// a message for qcp_last_error; nothing calls exit() (the reference's
// cudaErrCheck exits the process, src/common/macro.h:100-108).
#include <cstdio>
#include <cstring>
#include <new>

#include "qcp_internal.cuh"

namespace qcp {

namespace {
thread_local std::string t_error;
thread_local uint64_t t_launches = 0;
thread_local qcp_query_stats t_stats;
}  // namespace

void set_error(const std::string& msg) { t_error = msg; }
void clear_error() { t_error.clear(); }

qcp_status cuda_status(cudaError_t e, const char* what) {
  set_error(std::string(what) + ": " + cudaGetErrorString(e));
  if (e == cudaErrorMemoryAllocation) {
    cudaGetLastError();  // not sticky
    return QCP_ERR_OOM;
  }
  if (e == cudaErrorNoDevice || e == cudaErrorInsufficientDriver) return QCP_ERR_NO_DEVICE;
  return QCP_ERR_CUDA;
}

void note_launch(uint32_t k) { t_launches += k; }

qcp_status check_launch(const char* what) {
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return cuda_status(e, what);
  return QCP_OK;
}

// ---------------------------------------------------------------------------
// Pools
// ---------------------------------------------------------------------------
static size_t round_alloc(size_t bytes) {
  size_t r = 256;
  while (r < bytes) r <<= 1;
  if (r > bytes + (bytes >> 2) + (64u << 20)) {
    // large requests: round to 2 MiB instead of the next power of two
    r = (bytes + (2u << 20) - 1) & ~((size_t)(2u << 20) - 1);
  }
  return r;
}

qcp_status DevPool::get(size_t bytes, void** out) {
  if (bytes == 0) bytes = 1;
  {
    std::lock_guard<std::mutex> g(mu);
    size_t best = (size_t)-1, bi = 0;
    for (size_t i = 0; i < free_list.size(); ++i) {
      const size_t sz = free_list[i].first;
      if (sz >= bytes && sz <= 2 * bytes + (1u << 20) && sz < best) {
        best = sz;
        bi = i;
      }
    }
    if (best != (size_t)-1) {
      *out = free_list[bi].second;
      cached_bytes -= best;
      free_list.erase(free_list.begin() + bi);
      return QCP_OK;
    }
  }
  const size_t sz = round_alloc(bytes);
  void* p = nullptr;
  cudaError_t e = cudaMalloc(&p, sz);
  if (e == cudaErrorMemoryAllocation) {
    cudaGetLastError();
    trim();
    e = cudaMalloc(&p, sz);
  }
  if (e != cudaSuccess) return cuda_status(e, "cudaMalloc");
  // remember the real size through the free list protocol: callers hand the
  // requested size back, so record the mapping here
  {
    std::lock_guard<std::mutex> g(mu);
    sizes.emplace_back(p, sz);
  }
  *out = p;
  return QCP_OK;
}

void DevPool::put(size_t bytes, void* p) {
  (void)bytes;
  if (!p) return;
  std::lock_guard<std::mutex> g(mu);
  size_t sz = 0;
  for (auto& kv : sizes)
    if (kv.first == p) sz = kv.second;
  free_list.emplace_back(sz, p);
  cached_bytes += sz;
}

void DevPool::trim() {
  std::lock_guard<std::mutex> g(mu);
  for (auto& kv : free_list) {
    cudaFree(kv.second);
    for (size_t i = 0; i < sizes.size(); ++i)
      if (sizes[i].first == kv.second) {
        sizes.erase(sizes.begin() + i);
        break;
      }
  }
  free_list.clear();
  cached_bytes = 0;
}

qcp_status HostPool::get(size_t bytes, void** out) {
  if (bytes == 0) bytes = 1;
  {
    std::lock_guard<std::mutex> g(mu);
    size_t best = (size_t)-1, bi = 0;
    for (size_t i = 0; i < free_list.size(); ++i) {
      const size_t sz = free_list[i].first;
      if (sz >= bytes && sz <= 2 * bytes + (1u << 20) && sz < best) {
        best = sz;
        bi = i;
      }
    }
    if (best != (size_t)-1) {
      *out = free_list[bi].second;
      free_list.erase(free_list.begin() + bi);
      return QCP_OK;
    }
  }
  const size_t sz = round_alloc(bytes);
  void* p = nullptr;
  cudaError_t e = cudaHostAlloc(&p, sz, cudaHostAllocDefault);
  if (e == cudaErrorMemoryAllocation) {
    cudaGetLastError();
    trim();
    e = cudaHostAlloc(&p, sz, cudaHostAllocDefault);
  }
  if (e != cudaSuccess) return cuda_status(e, "cudaHostAlloc");
  {
    std::lock_guard<std::mutex> g(mu);
    sizes.emplace_back(p, sz);
  }
  *out = p;
  return QCP_OK;
}

void HostPool::put(size_t bytes, void* p) {
  (void)bytes;
  if (!p) return;
  std::lock_guard<std::mutex> g(mu);
  size_t sz = 0;
  for (auto& kv : sizes)
    if (kv.first == p) sz = kv.second;
  free_list.emplace_back(sz, p);
}

void HostPool::trim() {
  std::lock_guard<std::mutex> g(mu);
  for (auto& kv : free_list) {
    cudaFreeHost(kv.second);
    for (size_t i = 0; i < sizes.size(); ++i)
      if (sizes[i].first == kv.second) {
        sizes.erase(sizes.begin() + i);
        break;
      }
  }
  free_list.clear();
}

static HostPool& host_pool() {
  static HostPool* p = new HostPool();  // lives until exit
  return *p;
}

// ---------------------------------------------------------------------------
// Workspaces
// ---------------------------------------------------------------------------
template <class T>
static qcp_status grow(T** p, size_t* cap, size_t need, size_t elems_min = 1) {
  if (*p && *cap >= need) return QCP_OK;
  size_t n = need < elems_min ? elems_min : need;
  n += n >> 2;  // headroom
  if (*p) cudaFree(*p);
  *p = nullptr;
  *cap = 0;
  cudaError_t e = cudaMalloc((void**)p, sizeof(T) * n);
  if (e != cudaSuccess) return cuda_status(e, "workspace cudaMalloc");
  *cap = n;
  return QCP_OK;
}

qcp_status ws_reserve_items(qcp_index* ix, Workspace* ws, size_t items) {
  (void)ix;
  if (items == 0 || (ws->items[0] && ws->items_cap >= items)) return QCP_OK;
  size_t n = items + (items >> 2) + 1024;
  cudaFree(ws->items[0]);
  cudaFree(ws->items[1]);
  cudaFree(ws->item_hits);
  ws->items[0] = ws->items[1] = nullptr;
  ws->item_hits = nullptr;
  ws->items_cap = ws->item_hits_cap = 0;
  QCP_CUDA(cudaMalloc(&ws->items[0], sizeof(uint2) * n));
  QCP_CUDA(cudaMalloc(&ws->items[1], sizeof(uint2) * n));
  QCP_CUDA(cudaMalloc(&ws->item_hits, sizeof(uint32_t) * n));
  ws->items_cap = ws->item_hits_cap = n;
  return QCP_OK;
}

qcp_status ws_reserve_queries(qcp_index* ix, Workspace* ws, uint32_t q) {
  const size_t need = (size_t)q + 1;
  if (!ws->qcount || ws->q_cap < need) {
    const size_t n = need + (need >> 2) + 64;
    cudaFree(ws->qcount);
    cudaFree(ws->qcursor);
    ws->qcount = ws->qcursor = nullptr;
    ws->q_cap = 0;
    QCP_CUDA(cudaMalloc(&ws->qcount, sizeof(uint64_t) * n));
    QCP_CUDA(cudaMalloc(&ws->qcursor, sizeof(uint64_t) * n));
    ws->q_cap = n;
  }
  if (!ws->offsets || ws->offsets_cap < need) {
    if (ws->offsets) ix->pool.put(0, ws->offsets);
    ws->offsets = nullptr;
    ws->offsets_cap = 0;
    void* p = nullptr;
    QCP_TRY(ix->pool.get(sizeof(uint64_t) * need, &p));
    ws->offsets = (uint64_t*)p;
    ws->offsets_cap = need;
  }
  QCP_TRY(grow(&ws->boxes, &ws->boxes_cap, (size_t)q * 2 * ix->dims, 64));
  if (!ws->ctr) {
    QCP_CUDA(cudaMalloc(&ws->ctr, sizeof(uint32_t) * kCtrCount));
    QCP_CUDA(cudaHostAlloc(&ws->h_ctr, sizeof(uint32_t) * kCtrCount, cudaHostAllocDefault));
    QCP_CUDA(cudaHostAlloc(&ws->h_total, sizeof(uint64_t), cudaHostAllocDefault));
    QCP_CUDA(cudaMalloc(&ws->d_stats, sizeof(unsigned long long) * kStatCount));
    QCP_CUDA(cudaMemset(ws->d_stats, 0, sizeof(unsigned long long) * kStatCount));
    QCP_CUDA(cudaHostAlloc(&ws->h_stats, sizeof(unsigned long long) * kStatCount, cudaHostAllocDefault));
    for (int i = 0; i < kEvCountSlots; ++i) QCP_CUDA(cudaEventCreate(&ws->ev[i]));
  }
  // the root frontier holds one item per query
  if (!ws->items[0] || ws->items_cap < q) {
    const size_t want = (size_t)q * 64 + (1u << 16);
    QCP_TRY(ws_reserve_items(ix, ws, want));
  }
  return QCP_OK;
}

qcp_status ws_reserve_out(qcp_index* ix, Workspace* ws, size_t ids) {
  if (ws->out_ids && ws->out_cap >= ids) return QCP_OK;
  size_t n = ids + (ids >> 3) + 1024;
  if (ws->out_ids) ix->pool.put(sizeof(int32_t) * ws->out_cap, ws->out_ids);
  if (ws->tmp_ids) ix->pool.put(sizeof(int32_t) * ws->out_cap, ws->tmp_ids);
  ws->out_ids = ws->tmp_ids = nullptr;
  ws->out_cap = 0;
  void* a = nullptr;
  void* b = nullptr;
  QCP_TRY(ix->pool.get(sizeof(int32_t) * n, &a));
  qcp_status st = ix->pool.get(sizeof(int32_t) * n, &b);
  if (st != QCP_OK) {
    ix->pool.put(sizeof(int32_t) * n, a);
    return st;
  }
  ws->out_ids = (int32_t*)a;
  ws->tmp_ids = (int32_t*)b;
  ws->out_cap = n;
  return QCP_OK;
}

qcp_status ws_reserve_sort(qcp_index* ix, Workspace* ws, size_t jobs, size_t tiles) {
  (void)ix;
  if (jobs && (!ws->jobs[0] || ws->jobs_cap < jobs)) {
    size_t n = jobs + (jobs >> 2) + 256;
    cudaFree(ws->jobs[0]);
    cudaFree(ws->jobs[1]);
    ws->jobs[0] = ws->jobs[1] = nullptr;
    ws->jobs_cap = 0;
    QCP_CUDA(cudaMalloc(&ws->jobs[0], sizeof(uint4) * n));
    QCP_CUDA(cudaMalloc(&ws->jobs[1], sizeof(uint4) * n));
    ws->jobs_cap = n;
  }
  if (tiles) {
    size_t cap = ws->seg_hist_cap;
    QCP_TRY(grow(&ws->seg_hist, &cap, tiles, 1024));
    ws->seg_hist_cap = cap;
  }
  return QCP_OK;
}

// The count pass's hit cache: group records for `items` items and
// `mask_words` words of partial-leaf hit masks (each grown on its own).
qcp_status ws_reserve_hitcache(Workspace* ws, size_t items, size_t mask_words) {
  if (items && (!ws->item_grp || ws->item_grp_cap < items)) {
    cudaFree(ws->item_grp);
    ws->item_grp = nullptr;
    ws->item_grp_cap = 0;
    QCP_CUDA(cudaMalloc(&ws->item_grp, sizeof(uint32_t) * kMaxGroups * kGrpWords * items));
    ws->item_grp_cap = items;
  }
  if (mask_words && (!ws->hmask || ws->hmask_cap < mask_words)) {
    cudaFree(ws->hmask);
    ws->hmask = nullptr;
    ws->hmask_cap = 0;
    const size_t n = mask_words + (mask_words >> 2) + 4096;
    QCP_CUDA(cudaMalloc(&ws->hmask, sizeof(uint32_t) * n));
    ws->hmask_cap = n;
  }
  return QCP_OK;
}

qcp_status ws_reserve_qwhist(Workspace* ws, size_t n) {
  size_t cap = ws->qwhist_cap;
  QCP_TRY(grow(&ws->qwhist, &cap, n, 4096));
  ws->qwhist_cap = cap;
  return QCP_OK;
}

void ws_destroy(Workspace* ws, qcp_index* ix) {
  cudaFree(ws->qwhist);
  cudaFree(ws->scan_tmp);
  cudaFree(ws->boxes);
  cudaFree(ws->items[0]);
  cudaFree(ws->items[1]);
  cudaFree(ws->item_hits);
  cudaFree(ws->item_grp);
  cudaFree(ws->hmask);
  cudaFree(ws->qcount);
  cudaFree(ws->qcursor);
  if (ws->offsets) ix->pool.put(0, ws->offsets);
  if (ws->out_ids) ix->pool.put(0, ws->out_ids);
  if (ws->tmp_ids) ix->pool.put(0, ws->tmp_ids);
  cudaFree(ws->jobs[0]);
  cudaFree(ws->jobs[1]);
  cudaFree(ws->seg_hist);
  cudaFree(ws->ctr);
  if (ws->h_ctr) cudaFreeHost(ws->h_ctr);
  if (ws->h_total) cudaFreeHost(ws->h_total);
  cudaFree(ws->d_stats);
  if (ws->h_stats) cudaFreeHost(ws->h_stats);
  for (int i = 0; i < kEvCountSlots; ++i)
    if (ws->ev[i]) cudaEventDestroy(ws->ev[i]);
  delete ws;
}

static Workspace* ws_acquire(qcp_index* ix) {
  std::lock_guard<std::mutex> g(ix->ws_mu);
  if (!ix->ws_free.empty()) {
    Workspace* w = ix->ws_free.back();
    ix->ws_free.pop_back();
    return w;
  }
  Workspace* w = new (std::nothrow) Workspace();
  if (w) ix->ws_all.push_back(w);
  return w;
}

static void ws_release(qcp_index* ix, Workspace* ws) {
  std::lock_guard<std::mutex> g(ix->ws_mu);
  ix->ws_free.push_back(ws);
}

// Result arena owned by a qcp_result.
struct ResultArena {
  qcp_index* ix = nullptr;
  uint32_t mem = QCP_MEM_HOST;
  void* host = nullptr;      // pinned: offsets then ids
  size_t host_bytes = 0;
  uint64_t* d_offsets = nullptr;
  size_t d_offsets_cap = 0;
  int32_t* d_ids = nullptr;
  int32_t* d_tmp = nullptr;
  size_t d_ids_cap = 0;
};

static void index_release(qcp_index* ix) {
  for (Workspace* w : ix->ws_all) ws_destroy(w, ix);
  ix->ws_all.clear();
  ix->ws_free.clear();
  cudaFree(ix->coords);
  cudaFree(ix->ids);
  cudaFree(ix->keys);
  for (int l = 0; l < kMaxLevels; ++l) cudaFree(ix->mbr[l]);
  ix->pool.trim();
  delete ix;
}

static qcp_status index_alloc(qcp_index* ix) {
  const uint64_t F = ix->fanout;
  // level sizes, leaves first: ceil(n / F) until one node is left
  uint64_t cur = ix->n;
  uint32_t L = 0;
  do {
    cur = (cur + F - 1) / F;
    if (L >= (uint32_t)kMaxLevels) {
      set_error("tree deeper than 16 levels");
      return QCP_ERR_BAD_ARG;
    }
    ix->level_nodes[L] = cur;
    ix->level_pad[L] = ((cur + F - 1) / F) * F;
    ++L;
  } while (cur > 1);
  ix->levels = L;
  ix->npad = ix->level_nodes[0] * F;
  ix->device_bytes = 0;
  QCP_CUDA(cudaMalloc(&ix->coords, sizeof(float) * ix->ncoord * ix->npad));
  QCP_CUDA(cudaMalloc(&ix->ids, sizeof(int32_t) * ix->npad));
  QCP_CUDA(cudaMalloc(&ix->keys, sizeof(uint64_t) * ix->n));
  ix->device_bytes += sizeof(float) * ix->ncoord * ix->npad + sizeof(int32_t) * ix->npad;
  for (uint32_t l = 0; l < L; ++l) {
    QCP_CUDA(cudaMalloc(&ix->mbr[l], sizeof(float) * 2 * ix->dims * ix->level_pad[l]));
    ix->device_bytes += sizeof(float) * 2 * ix->dims * ix->level_pad[l];
  }
  return QCP_OK;
}

static uint32_t default_bits(uint32_t mode, uint32_t dims) {
  if (mode == QCP_KEY_REF) return dims > 2 ? 20 : 31;  // src/tree/tree.cpp:597
  if (dims == 1) return 32;
  if (dims == 2) return 32;
  if (dims == 3) return 21;
  return 64 / dims;
}

static qcp_status build_impl(const float* objs, uint64_t n, uint32_t dims, uint32_t is_rect,
                             const qcp_build_opts* opts, qcp_index** out) {
  if (!out) {
    set_error("out is NULL");
    return QCP_ERR_BAD_ARG;
  }
  *out = nullptr;
  qcp_build_opts o;
  memset(&o, 0, sizeof(o));
  if (opts) o = *opts;
  if (!objs || n == 0 || n >= (1ull << 31)) {
    set_error("objs must be non-NULL and 1 <= n < 2^31");
    return QCP_ERR_BAD_ARG;
  }
  if (dims < 1 || dims > (uint32_t)kMaxDims || is_rect > 1) {
    set_error("dims must be in [1, 8] and is_rect 0 or 1");
    return QCP_ERR_BAD_ARG;
  }
  const uint32_t fanout = o.fanout ? o.fanout : 128;
  if (fanout < 32 || fanout > 256 || fanout % 32) {
    set_error("fanout must be a multiple of 32 in [32, 256]");
    return QCP_ERR_BAD_ARG;
  }
  if (o.key_mode > QCP_KEY_KMEANS || o.input_mem > QCP_MEM_DEVICE) {
    set_error("invalid key_mode or input_mem");
    return QCP_ERR_BAD_ARG;
  }
  const uint32_t bits =
      o.key_bits ? o.key_bits : default_bits(o.key_mode == QCP_KEY_KMEANS ? QCP_KEY_NORM : o.key_mode, dims);
  if (bits > 32 || (uint64_t)bits * dims > 64) {
    set_error("key bits per dimension must be <= 32 and dims*bits <= 64");
    return QCP_ERR_BAD_ARG;
  }
  int count = 0;
  if (cudaGetDeviceCount(&count) != cudaSuccess || count == 0) {
    cudaGetLastError();
    set_error("no CUDA device");
    return QCP_ERR_NO_DEVICE;
  }
  cudaStream_t s = (cudaStream_t)o.stream;
  qcp_index* ix = new (std::nothrow) qcp_index();
  if (!ix) return QCP_ERR_OOM;
  cudaGetDevice(&ix->device);
  ix->n = n;
  ix->dims = dims;
  ix->is_rect = is_rect;
  ix->fanout = fanout;
  ix->key_mode = o.key_mode;
  ix->key_bits = bits;
  ix->ncoord = is_rect ? 2 * dims : dims;
  qcp_status st = index_alloc(ix);
  void *d_objs = nullptr, *keys_tmp = nullptr, *vals = nullptr, *vals_tmp = nullptr, *bad = nullptr;
  const size_t obj_bytes = sizeof(float) * ix->ncoord * n;
  bool own_objs = false;
  bool in_tmp = false;
  uint32_t h_bad = 0;
  if (st != QCP_OK) goto fail;
  if (o.input_mem == QCP_MEM_HOST) {
    st = ix->pool.get(obj_bytes, &d_objs);
    if (st != QCP_OK) goto fail;
    own_objs = true;
    if (cudaMemcpyAsync(d_objs, objs, obj_bytes, cudaMemcpyHostToDevice, s) != cudaSuccess) {
      st = cuda_status(cudaGetLastError(), "copy objects to device");
      goto fail;
    }
  } else {
    d_objs = (void*)objs;
  }
  if ((st = ix->pool.get(sizeof(uint64_t) * n, &keys_tmp)) != QCP_OK) goto fail;
  if ((st = ix->pool.get(sizeof(uint32_t) * n, &vals)) != QCP_OK) goto fail;
  if ((st = ix->pool.get(sizeof(uint32_t) * n, &vals_tmp)) != QCP_OK) goto fail;
  if ((st = ix->pool.get(sizeof(uint32_t), &bad)) != QCP_OK) goto fail;
  if (cudaMemsetAsync(bad, 0, sizeof(uint32_t), s) != cudaSuccess) {
    st = cuda_status(cudaGetLastError(), "memset");
    goto fail;
  }
  if (ix->key_mode == QCP_KEY_KMEANS) {
    const uint32_t K = o.kmeans_clusters ? o.kmeans_clusters : (uint32_t)(n < 1024 ? n : 1024);
    if ((st = build_keys_kmeans((const float*)d_objs, n, dims, is_rect, bits, K,
                                o.kmeans_iters ? o.kmeans_iters : 30u, ix->keys, (uint32_t*)vals, s)) != QCP_OK)
      goto fail;
  } else if ((st = build_keys((const float*)d_objs, n, dims, is_rect, ix->key_mode, bits, ix->keys,
                              (uint32_t*)vals, s)) != QCP_OK) {
    goto fail;
  }
  if ((st = radix_sort_pairs(ix->keys, (uint32_t*)vals, (uint64_t*)keys_tmp, (uint32_t*)vals_tmp, n,
                             ix->key_mode == QCP_KEY_KMEANS ? 64u : dims * bits, ix->pool, s, &in_tmp)) != QCP_OK)
    goto fail;
  if (in_tmp) {
    if (cudaMemcpyAsync(ix->keys, keys_tmp, sizeof(uint64_t) * n, cudaMemcpyDeviceToDevice, s) !=
        cudaSuccess) {
      st = cuda_status(cudaGetLastError(), "copy keys");
      goto fail;
    }
  }
  if ((st = build_pack(ix, (const float*)d_objs, (const uint32_t*)(in_tmp ? vals_tmp : vals), s,
                       (uint32_t*)bad)) != QCP_OK)
    goto fail;
  if ((st = build_levels(ix, s)) != QCP_OK) goto fail;
  if (cudaMemcpyAsync(&h_bad, bad, sizeof(uint32_t), cudaMemcpyDeviceToHost, s) != cudaSuccess ||
      cudaStreamSynchronize(s) != cudaSuccess) {
    st = cuda_status(cudaGetLastError(), "build");
    goto fail;
  }
  if (h_bad) {
    set_error("object coordinates must be finite");
    st = QCP_ERR_BAD_ARG;
    goto fail;
  }
  ix->pool.put(0, keys_tmp);
  ix->pool.put(0, vals);
  ix->pool.put(0, vals_tmp);
  ix->pool.put(0, bad);
  if (own_objs) ix->pool.put(0, d_objs);
  ix->pool.trim();
  *out = ix;
  return QCP_OK;
fail:
  cudaStreamSynchronize(s);
  if (keys_tmp) ix->pool.put(0, keys_tmp);
  if (vals) ix->pool.put(0, vals);
  if (vals_tmp) ix->pool.put(0, vals_tmp);
  if (bad) ix->pool.put(0, bad);
  if (own_objs && d_objs) ix->pool.put(0, d_objs);
  index_release(ix);
  return st;
}

static qcp_status run_query(qcp_index* ix, const float* boxes, uint32_t q, const qcp_query_opts* opts,
                            bool counts_only, Workspace** ws_out) {
  qcp_query_opts o;
  memset(&o, 0, sizeof(o));
  if (opts) o = *opts;
  if (!ix || (!boxes && q)) {
    set_error("index and boxes must be non-NULL");
    return QCP_ERR_BAD_ARG;
  }
  if (o.algo > QCP_ALGO_HYBRID || o.boxes_mem > QCP_MEM_DEVICE || o.result_mem > QCP_MEM_DEVICE) {
    set_error("invalid query options");
    return QCP_ERR_BAD_ARG;
  }
  int dev = 0;
  cudaGetDevice(&dev);
  if (dev != ix->device) {
    set_error("index lives on another device than the current one");
    return QCP_ERR_BAD_ARG;
  }
  cudaStream_t s = (cudaStream_t)o.stream;
  Workspace* ws = ws_acquire(ix);
  if (!ws) return QCP_ERR_OOM;
  qcp_status st = ws_reserve_queries(ix, ws, q);
  ws->timing = (o.flags & QCP_QUERY_TIMING) != 0;
  ws->blocks_per_sm = o.blocks_per_sm ? (o.blocks_per_sm > 32 ? 32u : o.blocks_per_sm) : 8u;
  ws->win_bits = o.win_bits ? (o.win_bits < 12 ? 12u : o.win_bits) : kDefaultWinBits;
  ws->leaf_ring = leaf_ring_of(o.leaf_prefetch);
  ws->lanes_per_item = lanes_per_item_of(o.lanes_per_item);
  ws->hit_cache_on = o.hit_cache != 1;
  ws->sort_small_jobs = ws->sort_msd_jobs = 0;
  ws->hybrid = o.algo == QCP_ALGO_HYBRID;
  ws->cpu_threads = o.cpu_threads;
  ws->handoff_level = o.handoff_level ? o.handoff_level : 1u;
  ws->h_boxes = nullptr;
  if (st == QCP_OK && q && ws->hybrid) {
    // the host walk reads the boxes on the host
    if (o.boxes_mem == QCP_MEM_HOST) {
      ws->h_boxes = boxes;
    } else {
      ws->h_boxes_copy.resize(2 * (size_t)ix->dims * q);
      if (cudaMemcpyAsync(ws->h_boxes_copy.data(), boxes, sizeof(float) * ws->h_boxes_copy.size(),
                          cudaMemcpyDeviceToHost, s) != cudaSuccess ||
          cudaStreamSynchronize(s) != cudaSuccess)
        st = cuda_status(cudaGetLastError(), "copy query boxes to the host");
      ws->h_boxes = ws->h_boxes_copy.data();
    }
  }
  if (st == QCP_OK && q) {
    const size_t bytes = sizeof(float) * 2 * ix->dims * (size_t)q;
    cudaError_t e = cudaMemcpyAsync(ws->boxes, boxes, bytes,
                                    o.boxes_mem == QCP_MEM_HOST ? cudaMemcpyHostToDevice
                                                                : cudaMemcpyDeviceToDevice,
                                    s);
    if (e != cudaSuccess) st = cuda_status(e, "copy query boxes");
  }
  if (st == QCP_OK) {
    if (q == 0) {
      *ws->h_total = 0;
      if (cudaMemsetAsync(ws->offsets, 0, sizeof(uint64_t), s) != cudaSuccess)
        st = cuda_status(cudaGetLastError(), "memset");
    } else if (o.algo == QCP_ALGO_PLAIN) {
      st = run_plain(ix, ws, q, counts_only, !o.unsorted, s);
    } else {
      st = run_batched(ix, ws, q, counts_only, !o.unsorted, s);
    }
  }
  if (st != QCP_OK) {
    cudaStreamSynchronize(s);
    ws_release(ix, ws);
    return st;
  }
  // work counters and phase times of this call
  memset(&t_stats, 0, sizeof(t_stats));
  t_stats.algo = o.algo;
  t_stats.num_queries = q;
  t_stats.hits = counts_only ? 0 : *ws->h_total;
  t_stats.sort_small_jobs = ws->sort_small_jobs;
  t_stats.sort_msd_jobs = ws->sort_msd_jobs;
  if (ws->timing && q) {
    if (cudaMemcpyAsync(ws->h_stats, ws->d_stats, sizeof(unsigned long long) * kStatCount,
                        cudaMemcpyDeviceToHost, s) == cudaSuccess &&
        cudaStreamSynchronize(s) == cudaSuccess) {
      t_stats.leaves_covered = ws->h_stats[kStatCovered];
      t_stats.leaves_partial = ws->h_stats[kStatPartial];
      t_stats.objects_covered = ws->h_stats[kStatObjCovered];
      t_stats.sort_window_ids = ws->h_stats[kStatWindowIds];
      t_stats.sort_window_bitmap_ids = ws->h_stats[kStatBitmapIds];
      for (int l = 0; l < 16; ++l) t_stats.frontier_items[l] = ws->h_stats[kStatLevel0 + l];
      t_stats.leaf_items = t_stats.frontier_items[1];
      auto ms = [&](int a, int b) {
        float v = 0.f;
        if (cudaEventElapsedTime(&v, ws->ev[a], ws->ev[b]) != cudaSuccess) {
          cudaGetLastError();
          v = 0.f;
        }
        return v;
      };
      t_stats.ms_expand = ms(kEvStart, kEvExpand);
      t_stats.ms_count = ms(kEvExpand, kEvCount);
      t_stats.ms_scan = ms(kEvCount, kEvScan);
      if (!counts_only && *ws->h_total) {
        t_stats.ms_write = ms(kEvScan, kEvWrite);
        t_stats.ms_sort = ms(kEvWrite, kEvSort);
        t_stats.ms_total = ms(kEvStart, kEvSort);
        if (!o.unsorted) {
          t_stats.ms_sort_small = ms(kEvWrite, kEvSortSmall);
          if (ws->sort_part_marked) {
            t_stats.ms_sort_partition = ms(kEvSortSmall, kEvSortPart);
            t_stats.ms_sort_windows = ms(kEvSortPart, kEvSort);
            t_stats.ms_sort_windows_bitmap = ms(kEvSortPart, kEvSortBitmap);
          } else {
            t_stats.ms_sort_windows = ms(kEvSortSmall, kEvSort);
          }
        }
      } else {
        t_stats.ms_total = ms(kEvStart, kEvScan);
      }
    }
  }
  *ws_out = ws;
  return QCP_OK;
}

// ---------------------------------------------------------------------------
// Captured build (qcp_build_plan_*): the device bulk load of n objects of a
// fixed shape -- keys, radix sort, packing, bottom-up MBR levels -- recorded
// once into a CUDA graph over buffers the plan owns and replayed per build.
// The reference builds on the host and copies the tree over in one piece
// (Tree::Bottom_Up, src/tree/tree.cpp:410-495; MPHR::Build,
// src/tree/mphr.cpp:60-133).
// ---------------------------------------------------------------------------
}  // namespace qcp

struct qcp_build_plan {
  qcp_index* ix = nullptr;
  uint64_t n = 0;
  uint32_t ncoord = 0;
  float* d_in = nullptr;        // objects the graph reads (n rows of ncoord floats)
  uint64_t* keys_tmp = nullptr;
  uint32_t* vals = nullptr;
  uint32_t* vals_tmp = nullptr;
  uint32_t* bad = nullptr;      // nonzero: a coordinate was not finite
  uint32_t* h_bad = nullptr;    // pinned mirror
  void* rs_scratch = nullptr;
  size_t rs_bytes = 0;
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
};

namespace qcp {

static void build_plan_destroy(qcp_build_plan* p) {
  if (!p) return;
  if (p->exec) cudaGraphExecDestroy(p->exec);
  if (p->graph) cudaGraphDestroy(p->graph);
  cudaFree(p->d_in);
  cudaFree(p->keys_tmp);
  cudaFree(p->vals);
  cudaFree(p->vals_tmp);
  cudaFree(p->bad);
  cudaFree(p->rs_scratch);
  if (p->h_bad) cudaFreeHost(p->h_bad);
  if (p->ix) index_release(p->ix);
  delete p;
}

// The build's device work on stream s, allocation- and sync-free.
static qcp_status build_plan_record(qcp_build_plan* p, cudaStream_t s) {
  qcp_index* ix = p->ix;
  QCP_CUDA(cudaMemsetAsync(p->bad, 0, sizeof(uint32_t), s));
  QCP_TRY(build_keys(p->d_in, ix->n, ix->dims, ix->is_rect, ix->key_mode, ix->key_bits, ix->keys, p->vals, s));
  bool in_tmp = false;
  QCP_TRY(radix_sort_pairs(ix->keys, p->vals, p->keys_tmp, p->vals_tmp, ix->n, ix->dims * ix->key_bits, ix->pool, s,
                           &in_tmp, p->rs_scratch, p->rs_bytes));
  if (in_tmp)
    QCP_CUDA(cudaMemcpyAsync(ix->keys, p->keys_tmp, sizeof(uint64_t) * ix->n, cudaMemcpyDeviceToDevice, s));
  QCP_TRY(build_pack(ix, p->d_in, in_tmp ? p->vals_tmp : p->vals, s, p->bad));
  QCP_TRY(build_levels(ix, s));
  return QCP_OK;
}

}  // namespace qcp

using namespace qcp;

extern "C" {

qcp_status qcp_build_plan_create(uint64_t n, uint32_t dims, uint32_t is_rect, const qcp_build_opts* opts,
                                 qcp_build_plan** out) {
  clear_error();
  if (!out) {
    set_error("out is NULL");
    return QCP_ERR_BAD_ARG;
  }
  *out = nullptr;
  qcp_build_opts o;
  memset(&o, 0, sizeof(o));
  if (opts) o = *opts;
  if (n == 0 || n >= (1ull << 31) || dims < 1 || dims > (uint32_t)kMaxDims || is_rect > 1) {
    set_error("qcp_build_plan_create: 1 <= n < 2^31, dims in [1, 8], is_rect 0 or 1");
    return QCP_ERR_BAD_ARG;
  }
  const uint32_t fanout = o.fanout ? o.fanout : 128;
  if (fanout < 32 || fanout > 256 || fanout % 32) {
    set_error("fanout must be a multiple of 32 in [32, 256]");
    return QCP_ERR_BAD_ARG;
  }
  if (o.key_mode > QCP_KEY_REF) {
    set_error("qcp_build_plan_create: key_mode must be QCP_KEY_NORM or QCP_KEY_REF (the k-means keys iterate "
              "to convergence on the host)");
    return QCP_ERR_BAD_ARG;
  }
  const uint32_t bits = o.key_bits ? o.key_bits : default_bits(o.key_mode, dims);
  if (bits > 32 || (uint64_t)bits * dims > 64) {
    set_error("key bits per dimension must be <= 32 and dims*bits <= 64");
    return QCP_ERR_BAD_ARG;
  }
  int count = 0;
  if (cudaGetDeviceCount(&count) != cudaSuccess || count == 0) {
    cudaGetLastError();
    set_error("no CUDA device");
    return QCP_ERR_NO_DEVICE;
  }
  qcp_build_plan* p = new (std::nothrow) qcp_build_plan();
  if (!p) return QCP_ERR_OOM;
  qcp_index* ix = new (std::nothrow) qcp_index();
  if (!ix) {
    delete p;
    return QCP_ERR_OOM;
  }
  p->ix = ix;
  cudaGetDevice(&ix->device);
  ix->n = n;
  ix->dims = dims;
  ix->is_rect = is_rect;
  ix->fanout = fanout;
  ix->key_mode = o.key_mode;
  ix->key_bits = bits;
  ix->ncoord = is_rect ? 2 * dims : dims;
  p->n = n;
  p->ncoord = ix->ncoord;
  p->rs_bytes = radix_scratch_bytes(n);
  qcp_status st = index_alloc(ix);
  cudaStream_t cap = nullptr;
  if (st == QCP_OK) {
    if (cudaMalloc(&p->d_in, sizeof(float) * p->ncoord * n) != cudaSuccess ||
        cudaMalloc(&p->keys_tmp, sizeof(uint64_t) * n) != cudaSuccess ||
        cudaMalloc(&p->vals, sizeof(uint32_t) * n) != cudaSuccess ||
        cudaMalloc(&p->vals_tmp, sizeof(uint32_t) * n) != cudaSuccess ||
        cudaMalloc(&p->bad, sizeof(uint32_t)) != cudaSuccess ||
        cudaMalloc(&p->rs_scratch, p->rs_bytes) != cudaSuccess ||
        cudaMallocHost(&p->h_bad, sizeof(uint32_t)) != cudaSuccess) {
      st = cuda_status(cudaGetLastError(), "qcp_build_plan_create allocation");
      if (st == QCP_OK) st = QCP_ERR_OOM;
    }
  }
  if (st == QCP_OK && cudaStreamCreateWithFlags(&cap, cudaStreamNonBlocking) != cudaSuccess)
    st = cuda_status(cudaGetLastError(), "cudaStreamCreate");
  if (st == QCP_OK) {
    // the build's attributes and lazily loaded kernels are set up by one
    // uncaptured run over the (zeroed) input before the capture
    cudaMemsetAsync(p->d_in, 0, sizeof(float) * p->ncoord * n, cap);
    st = build_plan_record(p, cap);
    if (st == QCP_OK && cudaStreamSynchronize(cap) != cudaSuccess) st = cuda_status(cudaGetLastError(), "build");
  }
  if (st == QCP_OK) {
    if (cudaStreamBeginCapture(cap, cudaStreamCaptureModeThreadLocal) != cudaSuccess) {
      st = cuda_status(cudaGetLastError(), "cudaStreamBeginCapture");
    } else {
      st = build_plan_record(p, cap);
      cudaGraph_t g = nullptr;
      const cudaError_t e = cudaStreamEndCapture(cap, &g);
      if (st == QCP_OK && e != cudaSuccess) st = cuda_status(e, "cudaStreamEndCapture");
      p->graph = g;
      if (st == QCP_OK && cudaGraphInstantiate(&p->exec, p->graph, 0) != cudaSuccess)
        st = cuda_status(cudaGetLastError(), "cudaGraphInstantiate");
    }
  }
  if (cap) cudaStreamDestroy(cap);
  if (st != QCP_OK) {
    build_plan_destroy(p);
    return st;
  }
  *out = p;
  return QCP_OK;
}

float* qcp_build_plan_input(qcp_build_plan* p) { return p ? p->d_in : nullptr; }

qcp_status qcp_build_plan_run(qcp_build_plan* p, const float* objs, uint32_t objs_mem, void* stream,
                              qcp_index** index) {
  clear_error();
  if (!p || !index || objs_mem > QCP_MEM_DEVICE) {
    set_error("qcp_build_plan_run: plan and index must be non-NULL, objs_mem a qcp_mem");
    return QCP_ERR_BAD_ARG;
  }
  *index = nullptr;
  cudaStream_t s = (cudaStream_t)stream;
  if (objs && objs != p->d_in)
    QCP_CUDA(cudaMemcpyAsync(p->d_in, objs, sizeof(float) * p->ncoord * p->n,
                             objs_mem == QCP_MEM_DEVICE ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice, s));
  QCP_CUDA(cudaGraphLaunch(p->exec, s));
  note_launch();
  QCP_CUDA(cudaMemcpyAsync(p->h_bad, p->bad, sizeof(uint32_t), cudaMemcpyDeviceToHost, s));
  QCP_CUDA(cudaStreamSynchronize(s));
  {
    std::lock_guard<std::mutex> g(p->ix->host_mbr_mu);
    p->ix->host_mbr_ready = false;  // host copies of the old levels are stale
  }
  if (*p->h_bad) {
    set_error("object coordinates must be finite");
    return QCP_ERR_BAD_ARG;
  }
  *index = p->ix;
  return QCP_OK;
}

qcp_status qcp_build_plan_free(qcp_build_plan* p) {
  clear_error();
  if (!p) return QCP_OK;
  cudaDeviceSynchronize();
  build_plan_destroy(p);
  return QCP_OK;
}

const char* qcp_last_error(void) { return t_error.c_str(); }

uint64_t qcp_launch_count(int reset) {
  uint64_t v = t_launches;
  if (reset) t_launches = 0;
  return v;
}

const char* qcp_version(void) { return "qcp-b200 0.1 (sm_100a)"; }

qcp_status qcp_query_stats_last(qcp_query_stats* out) {
  if (!out) return QCP_ERR_BAD_ARG;
  *out = t_stats;
  return QCP_OK;
}

qcp_status qcp_index_build(const float* objs, uint64_t n, uint32_t dims, uint32_t is_rect,
                           const qcp_build_opts* opts, qcp_index** out) {
  clear_error();
  return build_impl(objs, n, dims, is_rect, opts, out);
}

qcp_status qcp_index_free(qcp_index* index) {
  clear_error();
  if (!index) return QCP_OK;
  cudaDeviceSynchronize();
  index_release(index);
  return QCP_OK;
}

qcp_status qcp_index_get_info(const qcp_index* ix, qcp_index_info* info) {
  clear_error();
  if (!ix || !info) {
    set_error("index and info must be non-NULL");
    return QCP_ERR_BAD_ARG;
  }
  memset(info, 0, sizeof(*info));
  info->n = ix->n;
  info->dims = ix->dims;
  info->is_rect = ix->is_rect;
  info->fanout = ix->fanout;
  info->levels = ix->levels;
  for (uint32_t l = 0; l < ix->levels && l < 16; ++l) info->level_nodes[l] = ix->level_nodes[l];
  info->device_bytes = ix->device_bytes;
  info->key_mode = ix->key_mode;
  info->key_bits = ix->key_bits;
  return QCP_OK;
}

qcp_status qcp_query_batch(qcp_index* ix, const float* boxes, uint32_t q, const qcp_query_opts* opts,
                           qcp_result* out) {
  clear_error();
  if (!out) {
    set_error("out is NULL");
    return QCP_ERR_BAD_ARG;
  }
  memset(out, 0, sizeof(*out));
  Workspace* ws = nullptr;
  QCP_TRY(run_query(ix, boxes, q, opts, false, &ws));
  const uint32_t mem = opts ? opts->result_mem : (uint32_t)QCP_MEM_HOST;
  cudaStream_t s = opts ? (cudaStream_t)opts->stream : nullptr;
  const uint64_t total = *ws->h_total;
  ResultArena* a = new (std::nothrow) ResultArena();
  qcp_status st = a ? QCP_OK : QCP_ERR_OOM;
  if (st == QCP_OK) {
    a->ix = ix;
    a->mem = mem;
    if (mem == QCP_MEM_HOST) {
      a->host_bytes = sizeof(uint64_t) * ((size_t)q + 1) + sizeof(int32_t) * total;
      st = host_pool().get(a->host_bytes, &a->host);
      if (st == QCP_OK) {
        uint64_t* h_off = (uint64_t*)a->host;
        int32_t* h_ids = (int32_t*)(h_off + q + 1);
        cudaError_t e = cudaMemcpyAsync(h_off, ws->offsets, sizeof(uint64_t) * ((size_t)q + 1),
                                        cudaMemcpyDeviceToHost, s);
        if (e == cudaSuccess && total)
          e = cudaMemcpyAsync(h_ids, ws->out_ids, sizeof(int32_t) * total, cudaMemcpyDeviceToHost, s);
        if (e == cudaSuccess) e = cudaStreamSynchronize(s);
        if (e != cudaSuccess) st = cuda_status(e, "copy result to host");
        out->offsets = h_off;
        out->ids = h_ids;
      }
    } else {
      // hand the workspace's output buffers to the result; the workspace
      // takes fresh ones from the pool on its next call
      a->d_offsets = ws->offsets;
      a->d_offsets_cap = ws->offsets_cap;
      a->d_ids = ws->out_ids;
      a->d_tmp = ws->tmp_ids;
      a->d_ids_cap = ws->out_cap;
      ws->offsets = nullptr;
      ws->offsets_cap = 0;
      ws->out_ids = ws->tmp_ids = nullptr;
      ws->out_cap = 0;
      cudaError_t e = cudaStreamSynchronize(s);
      if (e != cudaSuccess) st = cuda_status(e, "query");
      out->offsets = a->d_offsets;
      out->ids = a->d_ids;
    }
  }
  ws_release(ix, ws);
  if (st != QCP_OK) {
    if (a) {
      qcp_result tmp;
      memset(&tmp, 0, sizeof(tmp));
      tmp.owner_ = a;
      qcp_result_release(&tmp);
    }
    memset(out, 0, sizeof(*out));
    return st;
  }
  out->num_queries = q;
  out->mem = mem;
  out->total_hits = total;
  out->owner_ = a;
  return QCP_OK;
}

qcp_status qcp_query_counts(qcp_index* ix, const float* boxes, uint32_t q, const qcp_query_opts* opts,
                            uint64_t* counts) {
  clear_error();
  if (!counts && q) {
    set_error("counts is NULL");
    return QCP_ERR_BAD_ARG;
  }
  Workspace* ws = nullptr;
  QCP_TRY(run_query(ix, boxes, q, opts, true, &ws));
  const uint32_t mem = opts ? opts->result_mem : (uint32_t)QCP_MEM_HOST;
  cudaStream_t s = opts ? (cudaStream_t)opts->stream : nullptr;
  qcp_status st = QCP_OK;
  if (q) {
    cudaError_t e = cudaMemcpyAsync(counts, ws->qcount, sizeof(uint64_t) * q,
                                    mem == QCP_MEM_HOST ? cudaMemcpyDeviceToHost
                                                        : cudaMemcpyDeviceToDevice,
                                    s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) st = cuda_status(e, "copy counts");
  }
  ws_release(ix, ws);
  return st;
}

qcp_status qcp_result_release(qcp_result* r) {
  if (!r || !r->owner_) return QCP_OK;
  ResultArena* a = (ResultArena*)r->owner_;
  if (a->host) host_pool().put(a->host_bytes, a->host);
  if (a->d_offsets && a->ix) a->ix->pool.put(0, a->d_offsets);
  if (a->d_ids && a->ix) a->ix->pool.put(0, a->d_ids);
  if (a->d_tmp && a->ix) a->ix->pool.put(0, a->d_tmp);
  delete a;
  memset(r, 0, sizeof(*r));
  return QCP_OK;
}

// ---------------------------------------------------------------------------
// Index files: "QCPIDX1\0", a header of little-endian fields, then the
// sorted keys, ids, coordinates and the MBR levels exactly as resident.
// ---------------------------------------------------------------------------
namespace {
const char kMagic[8] = {'Q', 'C', 'P', 'I', 'D', 'X', '1', 0};
struct FileHeader {
  char magic[8];
  uint32_t version, dims, is_rect, fanout, levels, key_mode, key_bits, ncoord;
  uint64_t n, npad;
  uint64_t level_nodes[kMaxLevels];
  uint64_t level_pad[kMaxLevels];
};
}  // namespace

qcp_status qcp_index_save(const qcp_index* ix, const char* path) {
  clear_error();
  if (!ix || !path) {
    set_error("index and path must be non-NULL");
    return QCP_ERR_BAD_ARG;
  }
  FILE* f = fopen(path, "wb");
  if (!f) {
    set_error(std::string("cannot open ") + path);
    return QCP_ERR_IO;
  }
  FileHeader h;
  memset(&h, 0, sizeof(h));
  memcpy(h.magic, kMagic, 8);
  h.version = 1;
  h.dims = ix->dims;
  h.is_rect = ix->is_rect;
  h.fanout = ix->fanout;
  h.levels = ix->levels;
  h.key_mode = ix->key_mode;
  h.key_bits = ix->key_bits;
  h.ncoord = ix->ncoord;
  h.n = ix->n;
  h.npad = ix->npad;
  memcpy(h.level_nodes, ix->level_nodes, sizeof(h.level_nodes));
  memcpy(h.level_pad, ix->level_pad, sizeof(h.level_pad));
  bool ok = fwrite(&h, sizeof(h), 1, f) == 1;
  auto dump = [&](const void* dptr, size_t bytes) {
    if (!ok || bytes == 0) return;
    std::vector<char> buf(bytes);
    if (cudaMemcpy(buf.data(), dptr, bytes, cudaMemcpyDeviceToHost) != cudaSuccess) {
      ok = false;
      return;
    }
    ok = fwrite(buf.data(), 1, bytes, f) == bytes;
  };
  dump(ix->keys, sizeof(uint64_t) * ix->n);
  dump(ix->ids, sizeof(int32_t) * ix->npad);
  dump(ix->coords, sizeof(float) * ix->ncoord * ix->npad);
  for (uint32_t l = 0; l < ix->levels; ++l) dump(ix->mbr[l], sizeof(float) * 2 * ix->dims * ix->level_pad[l]);
  ok = (fclose(f) == 0) && ok;
  if (!ok) {
    set_error(std::string("failed writing ") + path);
    return QCP_ERR_IO;
  }
  return QCP_OK;
}

qcp_status qcp_index_load(const char* path, void* stream, qcp_index** out) {
  clear_error();
  (void)stream;
  if (!path || !out) {
    set_error("path and out must be non-NULL");
    return QCP_ERR_BAD_ARG;
  }
  *out = nullptr;
  FILE* f = fopen(path, "rb");
  if (!f) {
    set_error(std::string("cannot open ") + path);
    return QCP_ERR_IO;
  }
  FileHeader h;
  if (fread(&h, sizeof(h), 1, f) != 1 || memcmp(h.magic, kMagic, 8) != 0 || h.version != 1 ||
      h.dims < 1 || h.dims > (uint32_t)kMaxDims || h.levels < 1 || h.levels > (uint32_t)kMaxLevels ||
      h.n == 0 || h.n >= (1ull << 31) || h.fanout < 32 || h.fanout > 256 || h.fanout % 32 ||
      h.ncoord != (h.is_rect ? 2 * h.dims : h.dims)) {
    fclose(f);
    set_error(std::string("not a valid index file: ") + path);
    return QCP_ERR_IO;
  }
  qcp_index* ix = new (std::nothrow) qcp_index();
  if (!ix) {
    fclose(f);
    return QCP_ERR_OOM;
  }
  cudaGetDevice(&ix->device);
  ix->n = h.n;
  ix->dims = h.dims;
  ix->is_rect = h.is_rect;
  ix->fanout = h.fanout;
  ix->key_mode = h.key_mode;
  ix->key_bits = h.key_bits;
  ix->ncoord = h.ncoord;
  qcp_status st = index_alloc(ix);
  if (st == QCP_OK && (ix->levels != h.levels || ix->npad != h.npad ||
                       memcmp(ix->level_nodes, h.level_nodes, sizeof(h.level_nodes)) != 0)) {
    set_error(std::string("inconsistent index file: ") + path);
    st = QCP_ERR_IO;
  }
  bool ok = st == QCP_OK;
  auto load = [&](void* dptr, size_t bytes) {
    if (!ok || bytes == 0) return;
    std::vector<char> buf(bytes);
    if (fread(buf.data(), 1, bytes, f) != bytes ||
        cudaMemcpy(dptr, buf.data(), bytes, cudaMemcpyHostToDevice) != cudaSuccess)
      ok = false;
  };
  load(ix->keys, sizeof(uint64_t) * ix->n);
  load(ix->ids, sizeof(int32_t) * ix->npad);
  load(ix->coords, sizeof(float) * ix->ncoord * ix->npad);
  for (uint32_t l = 0; l < ix->levels && ok; ++l) load(ix->mbr[l], sizeof(float) * 2 * ix->dims * ix->level_pad[l]);
  fclose(f);
  if (!ok) {
    if (st == QCP_OK) {
      set_error(std::string("failed reading ") + path);
      st = QCP_ERR_IO;
    }
    index_release(ix);
    return st;
  }
  *out = ix;
  return QCP_OK;
}

qcp_status qcp_index_export(const qcp_index* ix, uint64_t* keys, int32_t* ids, uint32_t level, float* mbr) {
  clear_error();
  if (!ix) {
    set_error("index is NULL");
    return QCP_ERR_BAD_ARG;
  }
  if (keys) QCP_CUDA(cudaMemcpy(keys, ix->keys, sizeof(uint64_t) * ix->n, cudaMemcpyDeviceToHost));
  if (ids) QCP_CUDA(cudaMemcpy(ids, ix->ids, sizeof(int32_t) * ix->n, cudaMemcpyDeviceToHost));
  if (mbr) {
    if (level >= ix->levels) {
      set_error("level out of range");
      return QCP_ERR_BAD_ARG;
    }
    const uint64_t nodes = ix->level_nodes[level], pad = ix->level_pad[level];
    const uint32_t m = 2 * ix->dims;
    std::vector<float> soa((size_t)m * pad);
    QCP_CUDA(cudaMemcpy(soa.data(), ix->mbr[level], sizeof(float) * m * pad, cudaMemcpyDeviceToHost));
    for (uint64_t k = 0; k < nodes; ++k)
      for (uint32_t c = 0; c < m; ++c) mbr[k * m + c] = soa[(size_t)c * pad + k];
  }
  return QCP_OK;
}

}  // extern "C"
