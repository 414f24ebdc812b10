// Internal declarations shared by the library's translation units.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <mutex>
#include <string>
#include <vector>

#include "qcp.h"

namespace qcp {

constexpr int kMaxLevels = 16;
constexpr int kMaxDims = 8;
constexpr uint32_t kWarp = 32;

// ---------------------------------------------------------------------------
// Errors: every failing step records a message for qcp_last_error and returns
// a status; nothing exits the process.
// ---------------------------------------------------------------------------
void set_error(const std::string& msg);
void clear_error();
qcp_status cuda_status(cudaError_t e, const char* what);

#define QCP_CUDA(expr)                                              \
  do {                                                              \
    cudaError_t e_ = (expr);                                        \
    if (e_ != cudaSuccess) return ::qcp::cuda_status(e_, #expr);    \
  } while (0)

#define QCP_TRY(expr)                    \
  do {                                   \
    qcp_status s_ = (expr);              \
    if (s_ != QCP_OK) return s_;         \
  } while (0)

// Per-host-thread count of kernel launches made by this library.
void note_launch(uint32_t k = 1);
qcp_status check_launch(const char* what);

// ---------------------------------------------------------------------------
// Device buffers.  A small caching allocator keeps freed buffers per device
// so that repeated query batches do not call cudaMalloc each time.
// ---------------------------------------------------------------------------
struct DevPool {
  std::mutex mu;
  std::vector<std::pair<size_t, void*>> free_list;  // (bytes, ptr) ready for reuse
  std::vector<std::pair<void*, size_t>> sizes;      // every live allocation's size
  size_t cached_bytes = 0;
  qcp_status get(size_t bytes, void** out);
  void put(size_t bytes, void* p);
  void trim();
};

struct HostPool {  // pinned host memory for results
  std::mutex mu;
  std::vector<std::pair<size_t, void*>> free_list;
  std::vector<std::pair<void*, size_t>> sizes;
  qcp_status get(size_t bytes, void** out);
  void put(size_t bytes, void* p);
  void trim();
};

template <class T>
struct DevArray {
  T* ptr = nullptr;
  size_t cap = 0;  // elements
};

// Phase events of Workspace::ev.
enum EvSlot : int {
  kEvStart = 0, kEvExpand = 1, kEvCount = 2, kEvScan = 3, kEvWrite = 4, kEvSort = 5,
  kEvSortSmall = 6, kEvSortPart = 7, kEvSortBitmap = 8, kEvCountSlots = 9
};

// Scratch for one query call.  Reused across calls through the index's
// workspace list (one workspace per concurrently running call).
struct Workspace {
  float* boxes = nullptr;
  size_t boxes_cap = 0;          // floats
  uint2* items[2] = {nullptr, nullptr};
  size_t items_cap = 0;          // (query, node) items per buffer
  uint32_t* item_hits = nullptr; // per level-1 item hit counts
  size_t item_hits_cap = 0;
  uint64_t* qcount = nullptr;    // per-query counts, q
  uint64_t* qcursor = nullptr;   // per-query write cursors, q
  uint64_t* offsets = nullptr;   // q + 1, from the index's pool
  size_t offsets_cap = 0;
  size_t q_cap = 0;
  int32_t* out_ids = nullptr;    // unsorted then sorted ids
  int32_t* tmp_ids = nullptr;    // segmented-sort ping-pong buffer
  size_t out_cap = 0;            // ids
  // segmented sort job lists
  uint4* jobs[2] = {nullptr, nullptr};
  size_t jobs_cap = 0;
  uint32_t* seg_hist = nullptr;  // MSD tile -> job map
  size_t seg_hist_cap = 0;
  uint32_t* ctr = nullptr;       // device counters (see kCtr*)
  uint32_t* h_ctr = nullptr;     // pinned mirror of ctr
  uint64_t* h_total = nullptr;   // pinned total-hits readback
  // work counters (kStat* slots) and phase events of the current call
  unsigned long long* d_stats = nullptr;
  unsigned long long* h_stats = nullptr;
  cudaEvent_t ev[kEvCountSlots] = {};
  bool timing = false;
  bool sort_part_marked = false;
  // per-(query, window) id counts of the sorted path, gathered by the write
  // pass (hist_G == 0: not gathered, the sort counts them itself)
  uint32_t* qwhist = nullptr;
  size_t qwhist_cap = 0;
  void* scan_tmp = nullptr;  // scan chunk sums of the captured pipeline (plans)
  size_t scan_tmp_cap = 0;
  uint32_t hist_G = 0, hist_bits = 0;
  uint32_t blocks_per_sm = 8;    // traversal grid = SMs x this, this call
  uint32_t win_bits = 18;        // sort window, this call
  uint32_t leaf_ring = 2;        // leaf prefetch buffers per warp, this call (< 2: none)
  // hit cache of the count pass for the write pass: per item and 32-leaf
  // group {overlap mask, covered mask, word offset of the group's partial
  // leaves' hit masks in hmask}; per partially covered leaf its hit bits
  uint32_t* item_grp = nullptr;
  size_t item_grp_cap = 0;       // items
  uint32_t* hmask = nullptr;
  size_t hmask_cap = 0;          // words
  bool use_hit_cache = false;    // this call's count pass fills the cache
  bool hit_cache_on = true;      // qcp_query_opts.hit_cache of this call
  uint32_t lanes_per_item = 32;  // lanes of k_expand per (query, node) item, this call
  // CPU + GPU co-processing (QCP_ALGO_HYBRID) of this call
  bool hybrid = false;
  uint32_t cpu_threads = 0, handoff_level = 1;
  const float* h_boxes = nullptr;    // the call's boxes in host memory
  std::vector<float> h_boxes_copy;   // when the caller's boxes are on the device
  std::vector<uint2> h_items;        // host-walked frontier
  uint32_t h_nitems = 0;
  uint32_t sort_small_jobs = 0, sort_msd_jobs = 0;
};

// Slots of Workspace::d_stats.
enum StatSlot : uint32_t {
  kStatCovered = 0,     // covered leaves
  kStatPartial = 1,     // partially covered leaves (objects tested)
  kStatObjCovered = 2,  // objects in covered leaves
  kStatWindowIds = 3,   // ids of the slices sorted through windows
  kStatBitmapIds = 4,   // ids of the windows listed for the bitmap sort
  kStatLevel0 = 8,      // frontier items of level l at kStatLevel0 + l
  kStatCount = 24
};


inline void mark(Workspace* ws, int slot, cudaStream_t s) {
  if (ws->timing) cudaEventRecord(ws->ev[slot], s);
}

// Slots of Workspace::ctr.
enum CtrSlot : uint32_t {
  kCtrFrontier0 = 0,  // items in items[0]
  kCtrFrontier1 = 1,  // items in items[1]
  kCtrWork = 2,       // dynamic work fetch counter
  kCtrOverflow = 3,   // nonzero: a capacity was exceeded
  kCtrNeedItems = 4,  // items needed when the frontier overflowed
  kCtrJobs0 = 5,      // segmented-sort job list sizes
  kCtrJobs1 = 6,
  kCtrSmall = 7,      // small-segment job count
  kCtrWork2 = 8,
  kCtrTimeout = 9,    // nonzero: a bounded device wait ran out (results invalid)
  kCtrMaskWords = 10, // hit-cache words the count pass asked for (may exceed the capacity)
  kCtrWinBig = 11,    // windows listed for the bitmap sort
  kCtrWinSmall = 12,  // windows listed for the one-warp sort
  kCtrCount = 16
};

}  // namespace qcp

struct qcp_index {
  int device = 0;
  uint64_t n = 0;
  uint32_t dims = 0, is_rect = 0, fanout = 128, levels = 0;
  uint32_t key_mode = 0, key_bits = 0;
  uint32_t ncoord = 0;                // dims (points) or 2*dims (rects)
  uint64_t npad = 0;                  // n rounded up to a multiple of fanout
  uint64_t level_nodes[qcp::kMaxLevels] = {0};
  uint64_t level_pad[qcp::kMaxLevels] = {0};
  float* coords = nullptr;            // [ncoord][npad], sorted order
  int32_t* ids = nullptr;             // [npad] input id of each sorted position
  uint64_t* keys = nullptr;           // [n] sorted keys
  float* mbr[qcp::kMaxLevels] = {nullptr};  // per level [2*dims][level_pad]
  // host copies of the internal levels' MBRs (levels >= 1), made on the first
  // CPU + GPU co-processing query
  std::mutex host_mbr_mu;
  std::vector<float> host_mbr[qcp::kMaxLevels];
  bool host_mbr_ready = false;
  uint64_t device_bytes = 0;

  qcp::DevPool pool;
  std::mutex ws_mu;
  std::vector<qcp::Workspace*> ws_free;
  std::vector<qcp::Workspace*> ws_all;
};

namespace qcp {

// ---------------------------------------------------------------------------
// Device helpers
// ---------------------------------------------------------------------------

// Overlap of a query box with an entry [lo, hi] in every dimension:
// !(q.lo > e.hi || q.hi < e.lo), the predicate of src/node/node_soa.cpp:94-113.
__host__ __device__ __forceinline__ bool overlaps1(float qlo, float qhi, float lo, float hi) {
  return !(qlo > hi || qhi < lo);
}
// Entry [lo, hi] lies inside the query box in one dimension.  Only used to
// skip the per-entry test of leaves whose MBR is covered by the query: every
// finite entry inside such an MBR passes overlaps1.
__host__ __device__ __forceinline__ bool inside1(float qlo, float qhi, float lo, float hi) {
  return qlo <= lo && hi <= qhi;
}

__host__ __device__ __forceinline__ uint64_t low_ones64(uint32_t k) {
  return k >= 64 ? ~0ull : ((1ull << k) - 1ull);
}

__host__ __device__ __forceinline__ uint32_t clz64(uint64_t x) {
#ifdef __CUDA_ARCH__
  return (uint32_t)__clzll((long long)x);
#else
  return x ? (uint32_t)__builtin_clzll(x) : 64u;
#endif
}

// Bit b of x moved to bit D*b (b < 64/D): "dilation" by the binary magic
// numbers method (shift-or-mask rounds, as in S. E. Anderson's Bit
// Twiddling Hacks, "Interleave bits by Binary Magic Numbers"; R. Raman and
// D. S. Wise, "Converting to and from Dilated Integers", IEEE TC 2008) for
// D = 2 and 3, a plain loop otherwise.
template <int D>
__host__ __device__ __forceinline__ uint64_t dilate(uint64_t x, uint32_t bits) {
  if (D == 2) {
    x &= 0xffffffffull;
    x = (x | (x << 16)) & 0x0000ffff0000ffffull;
    x = (x | (x << 8)) & 0x00ff00ff00ff00ffull;
    x = (x | (x << 4)) & 0x0f0f0f0f0f0f0f0full;
    x = (x | (x << 2)) & 0x3333333333333333ull;
    x = (x | (x << 1)) & 0x5555555555555555ull;
    return x;
  } else if (D == 3) {
    x &= 0x1fffffull;
    x = (x | (x << 32)) & 0x001f00000000ffffull;
    x = (x | (x << 16)) & 0x001f0000ff0000ffull;
    x = (x | (x << 8)) & 0x100f00f00f00f00full;
    x = (x | (x << 4)) & 0x10c30c30c30c30c3ull;
    x = (x | (x << 2)) & 0x1249249249249249ull;
    return x;
  } else {
    uint64_t t = 0;
    for (uint32_t b = 0; b < bits; ++b) t |= ((x >> b) & 1ull) << (b * D);
    return t;
  }
}

// Hilbert index of integer coordinates, the algorithm of
// HilbertMapper::MappingIntoSingle (src/mapper/hilbert_mapper.cpp:25-64) and
// hilbert_macro.h:4-22, written in unsigned 64-bit arithmetic in three
// parts: the coordinates are packed (coordinate d at bits [d*bits,
// (d+1)*bits), wider values spilling into the next field as in the
// reference's shifts) and transposed into bit levels (level b holds bit b of
// every coordinate, coordinate d at bit d), the levels are Gray-coded from
// the top with the entry-point rotation (one hilbert_step per level), and
// the result is prefix-XORed.
template <int D>
__host__ __device__ __forceinline__ uint64_t hilbert_transpose(uint32_t bits, const int64_t* coord) {
  uint64_t packed = 0;
  for (int d = D - 1; d >= 0; --d) packed = (packed << bits) | (uint64_t)coord[d];
  uint64_t t = 0;
  const uint64_t field = low_ones64(bits);
  for (uint32_t d = 0; d < (uint32_t)D; ++d) t |= dilate<D>((packed >> (d * bits)) & field, bits) << d;
  return t;
}

// One level: gin = the level's D transposed bits; (rot, flip) the rotation
// state carried from the level above (0, 0 at the top).  Returns the level's
// D index bits.
template <int D>
__host__ __device__ __forceinline__ uint64_t hilbert_step(uint64_t gin, uint32_t& rot, uint64_t& flip) {
  constexpr uint64_t nd_ones = (1ull << D) - 1ull;
  constexpr uint64_t nd1_ones = nd_ones >> 1;
  uint64_t g = gin ^ flip;
  if (rot) g = ((g >> rot) | (g << (D - rot))) & nd_ones;
  flip = 1ull << rot;
  // the rotation advances past the lowest set bit of g below the top one
  const uint64_t low = g & (0ull - g) & nd1_ones;
  if (low) rot += 64u - clz64(low);
  if (++rot >= (uint32_t)D) rot -= D;
  return g;
}

template <int D>
__host__ __device__ __forceinline__ uint64_t hilbert_finish(uint64_t index, uint32_t bits) {
  const uint32_t total = (uint32_t)D * bits;
  if (bits > 1) index ^= dilate<D>(low_ones64(bits), bits) >> 1;  // bit 0 of every level, shifted
  for (uint32_t s = 1; s < total; s *= 2) index ^= index >> s;
  return index & low_ones64(total);
}

template <int D>
__host__ __device__ inline uint64_t hilbert_index_t(uint32_t bits, const int64_t* coord) {
  if (D <= 1) return (uint64_t)coord[0];
  uint64_t t = hilbert_transpose<D>(bits, coord);
  uint64_t index;
  if (bits > 1) {
    t ^= t >> D;
    index = 0;
    uint32_t rot = 0;
    uint64_t flip = 0;
    for (int lvl = (int)bits - 1; lvl >= 0; --lvl)
      index = (index << D) | hilbert_step<D>((t >> (lvl * D)) & ((1ull << D) - 1ull), rot, flip);
  } else {
    index = t;
  }
  return hilbert_finish<D>(index, bits);
}

// Table-driven levels for D = 2 and 3: kHilbertLevels<D> levels per lookup.
// A rotation state (rot, flip) is encoded as rot * (D + 1) + f, f = 0 for
// flip == 0 and 1 + log2(flip) otherwise.  Entry [state << (L*D) | input]
// holds the L*D index bits of the L levels in its low byte and the state
// after them in bits 8..15; it is filled from hilbert_step, so a lookup is
// exactly L steps.
template <int D> struct HilbertTab;
template <> struct HilbertTab<2> { static constexpr uint32_t L = 4, kStates = 6; };
template <> struct HilbertTab<3> { static constexpr uint32_t L = 2, kStates = 12; };

template <int D>
__host__ __device__ __forceinline__ uint16_t hilbert_tab_entry(uint32_t e) {
  constexpr uint32_t L = HilbertTab<D>::L, IB = L * D;
  const uint32_t state = e >> IB, in = e & ((1u << IB) - 1u);
  uint32_t rot = state / (D + 1), f = state % (D + 1);
  uint64_t flip = f ? (1ull << (f - 1)) : 0ull;
  uint32_t out = 0;
  for (uint32_t j = 0; j < L; ++j) {
    const uint64_t gin = (in >> ((L - 1 - j) * D)) & ((1u << D) - 1u);
    out = (out << D) | (uint32_t)hilbert_step<D>(gin, rot, flip);
  }
  const uint32_t nf = flip ? (uint32_t)(63u - clz64(flip)) + 1u : 0u;
  return (uint16_t)(out | ((rot * (D + 1) + nf) << 8));
}

// hilbert_index_t through a filled table (HilbertTab<D>::kStates << (L*D)
// entries of hilbert_tab_entry), then plain steps for the bits % L lowest
// levels.
template <int D>
__host__ __device__ __forceinline__ uint64_t hilbert_index_tab(uint32_t bits, const int64_t* coord,
                                                             const uint16_t* tab) {
  constexpr uint32_t L = HilbertTab<D>::L, IB = L * D;
  uint64_t t = hilbert_transpose<D>(bits, coord);
  if (bits <= 1) return hilbert_finish<D>(t, bits);
  t ^= t >> D;
  uint64_t index = 0;
  uint32_t state = 0;
  int lvl = (int)bits - 1;
  for (; lvl + 1 >= (int)L; lvl -= (int)L) {
    const uint32_t in = (uint32_t)(t >> ((lvl + 1 - (int)L) * D)) & ((1u << IB) - 1u);
    const uint32_t e = tab[(state << IB) | in];
    index = (index << IB) | (e & 0xffu);
    state = e >> 8;
  }
  uint32_t rot = state / (D + 1), f = state % (D + 1);
  uint64_t flip = f ? (1ull << (f - 1)) : 0ull;
  for (; lvl >= 0; --lvl)
    index = (index << D) | hilbert_step<D>((t >> (lvl * D)) & ((1ull << D) - 1ull), rot, flip);
  return hilbert_finish<D>(index, bits);
}

__host__ __device__ inline uint64_t hilbert_index(uint32_t dims, uint32_t bits, const int64_t* coord) {
  switch (dims) {
    case 1: return hilbert_index_t<1>(bits, coord);
    case 2: return hilbert_index_t<2>(bits, coord);
    case 3: return hilbert_index_t<3>(bits, coord);
    case 4: return hilbert_index_t<4>(bits, coord);
    case 5: return hilbert_index_t<5>(bits, coord);
    case 6: return hilbert_index_t<6>(bits, coord);
    case 7: return hilbert_index_t<7>(bits, coord);
    default: return hilbert_index_t<8>(bits, coord);
  }
}

// One per-query slice handed to the sort kernels: output offset, size and
// query index.
struct SortJob {
  unsigned long long off;
  uint32_t size;
  uint32_t q;
};

// Slices of at most this many ids are sorted whole in shared memory.
constexpr uint32_t kSmallSliceCap = 8192;
// Ids per tile of the window partition (a tile map holds one entry per tile
// of the larger slices: at most hits / kSortTile + slices).
constexpr uint32_t kSortTile = 2048;

// ---------------------------------------------------------------------------
// Kernel launchers (defined in the .cu files)
// ---------------------------------------------------------------------------
int num_sms();

// Build
qcp_status build_keys(const float* objs, uint64_t n, uint32_t dims, uint32_t is_rect,
                      uint32_t key_mode, uint32_t key_bits, uint64_t* keys, uint32_t* vals,
                      cudaStream_t s);
// With `scratch` (at least radix_scratch_bytes(n)) nothing is allocated, so
// the sort can be captured into a graph.
qcp_status radix_sort_pairs(uint64_t* keys, uint32_t* vals, uint64_t* keys_tmp, uint32_t* vals_tmp,
                            uint64_t n, uint32_t key_bits, DevPool& pool, cudaStream_t s,
                            bool* result_in_tmp, void* scratch = nullptr, size_t scratch_bytes = 0);
size_t radix_scratch_bytes(uint64_t n);
qcp_status build_keys_kmeans(const float* objs, uint64_t n, uint32_t dims, uint32_t is_rect, uint32_t bits,
                             uint32_t K, uint32_t max_iters, uint64_t* keys, uint32_t* vals, cudaStream_t s);
uint32_t kmeans_rank_bits(uint32_t K);
qcp_status build_pack(qcp_index* ix, const float* objs, const uint32_t* perm, cudaStream_t s,
                      uint32_t* d_bad);
qcp_status build_levels(qcp_index* ix, cudaStream_t s);

// Query
qcp_status run_batched(qcp_index* ix, Workspace* ws, uint32_t q, bool counts_only, bool sort,
                       cudaStream_t s);
qcp_status run_plain(qcp_index* ix, Workspace* ws, uint32_t q, bool counts_only, bool sort,
                     cudaStream_t s);
// Steps of the batched pipeline (qcp_search.cu): root items of every query
// into items[0]; (query, node) items of level l in items[cur] -> items of
// level l - 1 in items[cur ^ 1]; unsorted write of the level-1 items in
// items[cur] whose item_hits are nonzero.
qcp_status init_items(Workspace* ws, uint32_t q, cudaStream_t s);
qcp_status expand_level(qcp_index* ix, Workspace* ws, uint32_t l, int cur, cudaStream_t s);
qcp_status write_items(qcp_index* ix, Workspace* ws, int cur, cudaStream_t s);
// Host walk of the internal levels for QCP_ALGO_HYBRID: the (query, node)
// items of `level` for every query into items[0] and its counter.
qcp_status host_frontier(qcp_index* ix, Workspace* ws, uint32_t q, uint32_t level, cudaStream_t s);
// Fixed-capacity, readback-free variants for captured pipelines (qcp_plan).
qcp_status run_batched_device(qcp_index* ix, Workspace* ws, uint32_t q, uint64_t ids_cap, bool sort,
                              void* sort_tables, cudaStream_t s);
qcp_status segmented_sort_device(qcp_index* ix, Workspace* ws, uint32_t q, void* tables, cudaStream_t s);
size_t sort_tables_bytes(const qcp_index* ix, const Workspace* ws, uint32_t q);
// Window bits and window count of the per-query sort for this call.
void sort_window_shape(const qcp_index* ix, const Workspace* ws, uint32_t* wbits, uint32_t* G);
// Leaf prefetch buffers per warp of the traversal's leaf passes for a
// qcp_query_opts.leaf_prefetch value: 0 = the default (2), 1 = none (direct
// loads), 2..4 = that many.
constexpr uint32_t kDefaultLeafRing = 2;
inline uint32_t leaf_ring_of(uint32_t knob) {
  if (knob == 0) return kDefaultLeafRing;
  if (knob == 1) return 0;
  return knob > 4 ? 4u : knob;
}
// Lanes per (query, node) item of the level expansion for a
// qcp_query_opts.lanes_per_item value (0 = 32; 8, 16 or 32).
inline uint32_t lanes_per_item_of(uint32_t knob) { return (knob == 8 || knob == 16) ? knob : 32u; }
// Largest window count whose per-window counts the write pass gathers.
constexpr uint32_t kHistMaxG = 256;
// Default log2 of the per-query sort's id windows (qcp_query_opts.win_bits).
constexpr uint32_t kDefaultWinBits = 17;
qcp_status ws_reserve_qwhist(Workspace* ws, size_t n);
// Words per (item, group) record of the hit cache and groups per item.
constexpr uint32_t kGrpWords = 3;
constexpr uint32_t kMaxGroups = 8;                    // fan-out <= 256
constexpr uint32_t kNoMask = 0xffffffffu;            // group without cached hit masks
qcp_status ws_reserve_hitcache(Workspace* ws, size_t items, size_t mask_words);
// Workspace construction and buffer reservation (qcp_capi.cu).
qcp_status ws_reserve_queries(qcp_index* ix, Workspace* ws, uint32_t q);
qcp_status ws_reserve_items(qcp_index* ix, Workspace* ws, size_t items);
qcp_status ws_reserve_out(qcp_index* ix, Workspace* ws, size_t ids);
qcp_status ws_reserve_sort(qcp_index* ix, Workspace* ws, size_t jobs, size_t tiles);
void ws_destroy(Workspace* ws, qcp_index* ix);
qcp_status segmented_sort(qcp_index* ix, Workspace* ws, uint32_t q, cudaStream_t s);
// Sorts the slices of <= kSmallSliceCap ids; the larger slices are returned
// as a device job list (big, *nbig entries) for the caller.
qcp_status sort_small_slices(qcp_index* ix, Workspace* ws, uint32_t q, cudaStream_t s,
                             const SortJob** big, uint32_t* nbig);

qcp_status run_batched_counts_into(qcp_index* ix, const float* boxes, uint32_t q, uint64_t* counts,
                                   uint2* items0, uint2* items1, uint32_t* item_hits, size_t item_cap,
                                   uint32_t* ctr, unsigned long long* stats, cudaStream_t s);
qcp_status exclusive_scan_counts(const uint64_t* counts, uint64_t* offsets, uint32_t q,
                                 DevPool& pool, cudaStream_t s, void* scratch = nullptr,
                                 size_t scratch_bytes = 0);
template <class T>
qcp_status exclusive_scan(const T* in, T* out, uint64_t n, T* grand_total, DevPool& pool,
                          cudaStream_t s, void* scratch = nullptr, size_t scratch_bytes = 0);
// Bytes of caller-owned scratch an exclusive scan of n values needs.
size_t scan_scratch_bytes(uint64_t n);

}  // namespace qcp
