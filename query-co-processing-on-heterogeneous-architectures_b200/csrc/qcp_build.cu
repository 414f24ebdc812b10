// Device bulk load: Hilbert keys -> LSD radix sort of (key, id) -> packing
// into sorted SoA coordinate arrays -> bottom-up MBR levels.
//
// Replaces the host-threaded steps of the reference build
// (src/tree/tree.cpp:544-639 branch creation and key mapping,
// src/sort/thrust_sorter.cpp:12-47 sort and rank reassignment,
// src/tree/tree.cpp:683-745 packing, :410-495 and :1025-1133 bottom-up
// build, src/transformer/transformer.cpp:52-88 AoS->SoA transform): every
// step runs on the device and nothing crosses PCIe between them.
//
// Layout in HBM (see qcp_index):
//   coords[c * npad + i]   coordinate c of the i-th object in key order
//   ids[i]                 input id of the i-th object in key order
//   mbr[l][c * pad_l + k]  MBR component c ([lo0..lo(D-1), hi0..hi(D-1)]) of
//                          node k of level l (level 0 = leaves)
// Node k of level l covers children [k*F, (k+1)*F) of level l-1; leaf j
// covers objects [j*F, (j+1)*F).  No child pointers are stored.
#include <cfloat>
#include <cmath>

#include <mutex>

#include "qcp_internal.cuh"
#include "qcp_tree.cuh"

namespace qcp {

namespace {

__device__ __forceinline__ int64_t quantise(float p, uint32_t bits, uint32_t mode) {
  if (mode == QCP_KEY_REF) {
    // (long long)(1000000 * p): single-precision multiply then truncation
    // (src/mapper/hilbert_mapper.cpp:21-23)
    return (int64_t)__fmul_rn(1000000.0f, p);
  }
  float v = (p > 0.0f) ? p : 0.0f;  // negatives and NaN -> 0
  uint64_t maxq = low_ones64(bits);
  if (v >= 1.0f) return (int64_t)maxq;
  uint64_t q = (uint64_t)__fmul_rn(v, (float)(1ull << bits));  // exact scaling
  return (int64_t)(q > maxq ? maxq : q);
}

// One thread per object, the dimension count a template parameter so that
// the coordinates and the key's bit levels stay in registers.  For D = 2 and
// 3 each block first fills a shared-memory table of HilbertTab<D>::L levels
// per lookup (3 KB, 1.5 KB), so a 2-D key takes 8 lookups instead of 32
// level steps.
template <int D>
__global__ void k_keys(const float* __restrict__ objs, uint64_t n, uint32_t is_rect, uint32_t mode,
                       uint32_t bits, uint64_t* __restrict__ keys, uint32_t* __restrict__ vals) {
  constexpr bool kTab = D == 2 || D == 3;
  constexpr uint32_t kTabSize = kTab ? (HilbertTab<(D == 2 || D == 3) ? D : 2>::kStates
                                        << (HilbertTab<(D == 2 || D == 3) ? D : 2>::L * D))
                                     : 1u;
  __shared__ uint16_t tab[kTabSize];
  if constexpr (kTab) {
    for (uint32_t e = threadIdx.x; e < kTabSize; e += blockDim.x) tab[e] = hilbert_tab_entry<D>(e);
    __syncthreads();
  }
  const uint32_t stride = is_rect ? 2 * D : D;
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n;
       i += (uint64_t)gridDim.x * blockDim.x) {
    int64_t c[D];
    const float* o = objs + i * stride;
#pragma unroll
    for (int d = 0; d < D; ++d) {
      float p = is_rect ? __fmul_rn(0.5f, __fadd_rn(__ldg(o + d), __ldg(o + D + d))) : __ldg(o + d);
      c[d] = quantise(p, bits, mode);
    }
    if constexpr (kTab) keys[i] = hilbert_index_tab<D>(bits, c, tab);
    else keys[i] = hilbert_index_t<D>(bits, c);
    vals[i] = (uint32_t)i;
  }
}

// ---------------------------------------------------------------------------
// LSD radix sort, 8-bit digits.  Per pass: upsweep (tile histograms), an
// exclusive scan of the digit-major [256][tiles] table, and a downsweep that
// ranks each tile stably (the lanes of a warp with the same digit found by 8
// ballots, one per digit bit, + per-warp digit counters), regroups the tile
// by digit in shared memory and writes each digit run contiguously.
// ---------------------------------------------------------------------------
constexpr int RS_THREADS = 256;
constexpr int RS_WARPS = RS_THREADS / 32;
constexpr int RS_ITEMS = 8;
constexpr int RS_TILE = RS_THREADS * RS_ITEMS;  // 2048
constexpr int RS_PER_WARP = RS_TILE / RS_WARPS; // 256

__global__ void __launch_bounds__(RS_THREADS) k_rs_upsweep(const uint64_t* __restrict__ keys,
                                                           uint64_t n, uint32_t shift,
                                                           uint32_t* __restrict__ hist,
                                                           uint32_t ntiles) {
  __shared__ uint32_t h[RS_WARPS][256];
  const uint32_t tid = threadIdx.x, w = tid >> 5;
  for (uint32_t i = tid; i < RS_WARPS * 256; i += RS_THREADS) (&h[0][0])[i] = 0;
  __syncthreads();
  const uint64_t base = (uint64_t)blockIdx.x * RS_TILE;
  const uint64_t end = (base + RS_TILE < n) ? base + RS_TILE : n;
  for (uint64_t i = base + tid; i < end; i += RS_THREADS) {
    uint32_t d = (uint32_t)(keys[i] >> shift) & 255u;
    atomicAdd(&h[w][d], 1u);
  }
  __syncthreads();
  uint32_t s = 0;
  for (int k = 0; k < RS_WARPS; ++k) s += h[k][tid];
  hist[(uint64_t)tid * ntiles + blockIdx.x] = s;
}

__device__ __forceinline__ uint32_t lanemask_lt() {
  uint32_t m;
  asm("mov.u32 %0, %%lanemask_lt;" : "=r"(m));
  return m;
}

// Exclusive scan of one value per thread over a 256-thread block.
__device__ __forceinline__ uint32_t block_excl_scan256(uint32_t v, uint32_t* warp_tot) {
  const uint32_t lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  uint32_t x = v;
  for (int o = 1; o < 32; o <<= 1) {
    uint32_t y = __shfl_up_sync(0xffffffffu, x, o);
    if (lane >= (uint32_t)o) x += y;
  }
  if (lane == 31) warp_tot[w] = x;
  __syncthreads();
  if (w == 0) {
    uint32_t t = (lane < RS_WARPS) ? warp_tot[lane] : 0;
    for (int o = 1; o < RS_WARPS; o <<= 1) {
      uint32_t y = __shfl_up_sync(0xffffffffu, t, o);
      if (lane >= (uint32_t)o) t += y;
    }
    if (lane < RS_WARPS) warp_tot[lane] = t;  // inclusive
  }
  __syncthreads();
  uint32_t before = (w > 0) ? warp_tot[w - 1] : 0;
  uint32_t r = before + x - v;
  __syncthreads();
  return r;
}

__global__ void __launch_bounds__(RS_THREADS, 5) k_rs_downsweep(
    const uint64_t* __restrict__ keys_in, const uint32_t* __restrict__ vals_in,
    uint64_t* __restrict__ keys_out, uint32_t* __restrict__ vals_out, uint64_t n, uint32_t shift,
    const uint32_t* __restrict__ offs, uint32_t ntiles) {
  __shared__ uint32_t wcnt[RS_WARPS][256];
  __shared__ uint32_t tile_excl[256];
  __shared__ uint32_t gbase[256];
  __shared__ uint32_t warp_tot[RS_WARPS];
  __shared__ uint64_t skeys[RS_TILE];
  __shared__ uint32_t svals[RS_TILE];

  const uint32_t tid = threadIdx.x, lane = tid & 31, w = tid >> 5;
  for (uint32_t i = tid; i < RS_WARPS * 256; i += RS_THREADS) (&wcnt[0][0])[i] = 0;
  gbase[tid] = offs[(uint64_t)tid * ntiles + blockIdx.x];
  __syncthreads();

  const uint64_t base = (uint64_t)blockIdx.x * RS_TILE;
  const uint32_t tile_n = (uint32_t)((n - base) < (uint64_t)RS_TILE ? (n - base) : RS_TILE);
  uint64_t k[RS_ITEMS];
  uint32_t v[RS_ITEMS];
  uint32_t rank[RS_ITEMS];
  // every load of the tile in flight before the first ranking step
#pragma unroll
  for (int r = 0; r < RS_ITEMS; ++r) {
    const uint32_t li = w * RS_PER_WARP + r * 32 + lane;
    const bool valid = li < tile_n;
    k[r] = valid ? __ldcs(keys_in + base + li) : 0ull;
    v[r] = valid ? __ldcs(vals_in + base + li) : 0u;
  }
#pragma unroll
  for (int r = 0; r < RS_ITEMS; ++r) {
    const uint32_t li = w * RS_PER_WARP + r * 32 + lane;
    const bool valid = li < tile_n;
    rank[r] = 0;
    const uint32_t active = __ballot_sync(0xffffffffu, valid);
    if (valid) {
      const uint32_t d = (uint32_t)(k[r] >> shift) & 255u;
      uint32_t peers = active;
#pragma unroll
      for (int bb = 0; bb < 8; ++bb) {
        const uint32_t bit = (d >> bb) & 1u;
        const uint32_t bal = __ballot_sync(active, bit);
        peers &= bit ? bal : ~bal;
      }
      const uint32_t prev = wcnt[w][d];
      rank[r] = prev + __popc(peers & lanemask_lt());
      __syncwarp(active);
      if (lane == (uint32_t)(__ffs(peers) - 1)) wcnt[w][d] = prev + __popc(peers);
      __syncwarp(active);
    }
  }
  __syncthreads();
  // per digit: exclusive prefix across warps, then across digits
  uint32_t run = 0;
  for (int ww = 0; ww < RS_WARPS; ++ww) {
    uint32_t c = wcnt[ww][tid];
    wcnt[ww][tid] = run;
    run += c;
  }
  uint32_t ex = block_excl_scan256(run, warp_tot);
  tile_excl[tid] = ex;
  __syncthreads();
#pragma unroll
  for (int r = 0; r < RS_ITEMS; ++r) {
    const uint32_t li = w * RS_PER_WARP + r * 32 + lane;
    if (li < tile_n) {
      const uint32_t d = (uint32_t)(k[r] >> shift) & 255u;
      const uint32_t lp = tile_excl[d] + wcnt[w][d] + rank[r];
      skeys[lp] = k[r];
      svals[lp] = v[r];
    }
  }
  __syncthreads();
  for (uint32_t i = tid; i < tile_n; i += RS_THREADS) {
    const uint64_t key = skeys[i];
    const uint32_t d = (uint32_t)(key >> shift) & 255u;
    const uint64_t dst = (uint64_t)gbase[d] + (i - tile_excl[d]);
    keys_out[dst] = key;
    vals_out[dst] = svals[i];
  }
}

// Generic exclusive scan of uint32 (3 kernels: chunk sums, scan of sums, apply).
constexpr int SC_THREADS = 256;
constexpr int SC_ITEMS = 16;
constexpr int SC_CHUNK = SC_THREADS * SC_ITEMS;

template <class T>
__device__ __forceinline__ T warp_incl_scan(T x) {
  const uint32_t lane = threadIdx.x & 31;
  for (int o = 1; o < 32; o <<= 1) {
    T y = __shfl_up_sync(0xffffffffu, x, o);
    if (lane >= (uint32_t)o) x += y;
  }
  return x;
}

template <class T>
__device__ T block_excl_scan(T v, T* warp_tot, T* total) {
  const uint32_t lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  const uint32_t nw = blockDim.x >> 5;
  T x = warp_incl_scan(v);
  if (lane == 31) warp_tot[w] = x;
  __syncthreads();
  if (w == 0) {
    T t = (lane < nw) ? warp_tot[lane] : (T)0;
    t = warp_incl_scan(t);
    if (lane < nw) warp_tot[lane] = t;
  }
  __syncthreads();
  T before = (w > 0) ? warp_tot[w - 1] : (T)0;
  if (total) *total = warp_tot[nw - 1];
  __syncthreads();
  return before + x - v;
}

template <class T>
__global__ void k_scan_sums(const T* __restrict__ in, uint64_t n, T* __restrict__ sums) {
  __shared__ T wt[32];
  const uint64_t base = (uint64_t)blockIdx.x * SC_CHUNK;
  T s = 0;
  for (int r = 0; r < SC_ITEMS; ++r) {
    uint64_t i = base + (uint64_t)r * SC_THREADS + threadIdx.x;
    if (i < n) s += in[i];
  }
  T total;
  block_excl_scan(s, wt, &total);
  if (threadIdx.x == 0) sums[blockIdx.x] = total;
}

template <class T>
__global__ void k_scan_partials(T* sums, uint32_t m, T* grand_total) {
  __shared__ T wt[32];
  __shared__ T carry;
  if (threadIdx.x == 0) carry = 0;
  __syncthreads();
  for (uint32_t b = 0; b < m; b += blockDim.x) {
    uint32_t i = b + threadIdx.x;
    T v = (i < m) ? sums[i] : (T)0;
    T tot;
    T ex = block_excl_scan(v, wt, &tot);
    if (i < m) sums[i] = carry + ex;
    __syncthreads();
    if (threadIdx.x == 0) carry += tot;
    __syncthreads();
  }
  if (threadIdx.x == 0 && grand_total) *grand_total = carry;
}

template <class T>
__global__ void k_scan_apply(const T* __restrict__ in, T* __restrict__ out, uint64_t n,
                             const T* __restrict__ sums) {
  __shared__ T wt[32];
  const uint64_t base = (uint64_t)blockIdx.x * SC_CHUNK + (uint64_t)threadIdx.x * SC_ITEMS;
  T vals[SC_ITEMS];
  T s = 0;
#pragma unroll
  for (int r = 0; r < SC_ITEMS; ++r) {
    uint64_t i = base + r;
    vals[r] = (i < n) ? in[i] : (T)0;
    s += vals[r];
  }
  T ex = block_excl_scan(s, wt, (T*)nullptr) + sums[blockIdx.x];
#pragma unroll
  for (int r = 0; r < SC_ITEMS; ++r) {
    uint64_t i = base + r;
    if (i < n) out[i] = ex;
    ex += vals[r];
  }
}

// objs -> sorted SoA arrays; flags non-finite coordinates in *bad.
__global__ void k_pack(const float* __restrict__ objs, const uint32_t* __restrict__ perm, uint64_t n,
                       uint64_t npad, uint32_t ncoord, float* __restrict__ coords,
                       int32_t* __restrict__ ids, uint32_t* bad) {
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < npad;
       i += (uint64_t)gridDim.x * blockDim.x) {
    if (i < n) {
      const uint32_t id = perm[i];
      const float* o = objs + (uint64_t)id * ncoord;
      bool finite = true;
      for (uint32_t c = 0; c < ncoord; ++c) {
        float x = o[c];
        finite &= isfinite(x);
        coords[(uint64_t)c * npad + i] = x;
      }
      ids[i] = (int32_t)id;
      if (!finite) atomicOr(bad, 1u);
    } else {
      for (uint32_t c = 0; c < ncoord; ++c) coords[(uint64_t)c * npad + i] = __int_as_float(0x7fc00000);
      ids[i] = -1;
    }
  }
}

__device__ __forceinline__ float warp_min(float x) {
  for (int o = 16; o > 0; o >>= 1) x = fminf(x, __shfl_xor_sync(0xffffffffu, x, o));
  return x;
}
__device__ __forceinline__ float warp_max(float x) {
  for (int o = 16; o > 0; o >>= 1) x = fmaxf(x, __shfl_xor_sync(0xffffffffu, x, o));
  return x;
}

// One warp per leaf: MBR = per-dim min of lo / max of hi over its objects.
__global__ void k_leaf_mbr(const float* __restrict__ coords, uint64_t n, uint64_t npad, uint32_t dims,
                           uint32_t is_rect, uint32_t fanout, uint64_t nleaves, uint64_t pad0,
                           float* __restrict__ mbr) {
  const uint32_t lane = threadIdx.x & 31;
  const uint64_t warps = ((uint64_t)gridDim.x * blockDim.x) >> 5;
  for (uint64_t j = (blockIdx.x * (uint64_t)blockDim.x + threadIdx.x) >> 5; j < pad0; j += warps) {
    if (j >= nleaves) {
      if (lane < dims) {
        mbr[(uint64_t)lane * pad0 + j] = INFINITY;
        mbr[(uint64_t)(dims + lane) * pad0 + j] = -INFINITY;
      }
      continue;
    }
    const uint64_t e0 = j * fanout;
    const uint64_t e1 = (e0 + fanout < n) ? e0 + fanout : n;
    for (uint32_t d = 0; d < dims; ++d) {
      const float* lo_arr = coords + (uint64_t)d * npad;
      const float* hi_arr = coords + (uint64_t)(is_rect ? dims + d : d) * npad;
      float lo = INFINITY, hi = -INFINITY;
      for (uint64_t e = e0 + lane; e < e1; e += 32) {
        lo = fminf(lo, lo_arr[e]);
        hi = fmaxf(hi, hi_arr[e]);
      }
      lo = warp_min(lo);
      hi = warp_max(hi);
      if (lane == 0) {
        mbr[(uint64_t)d * pad0 + j] = lo;
        mbr[(uint64_t)(dims + d) * pad0 + j] = hi;
      }
    }
  }
}

// One warp per node of level l: MBR over the children's MBRs (level l-1).
__global__ void k_level_mbr(const float* __restrict__ child, uint64_t nchild, uint64_t child_pad,
                            uint32_t dims, uint32_t fanout, uint64_t nnodes, uint64_t pad,
                            float* __restrict__ mbr) {
  const uint32_t lane = threadIdx.x & 31;
  const uint64_t warps = ((uint64_t)gridDim.x * blockDim.x) >> 5;
  for (uint64_t k = (blockIdx.x * (uint64_t)blockDim.x + threadIdx.x) >> 5; k < pad; k += warps) {
    if (k >= nnodes) {
      if (lane < dims) {
        mbr[(uint64_t)lane * pad + k] = INFINITY;
        mbr[(uint64_t)(dims + lane) * pad + k] = -INFINITY;
      }
      continue;
    }
    const uint64_t c0 = k * fanout;
    const uint64_t c1 = (c0 + fanout < nchild) ? c0 + fanout : nchild;
    for (uint32_t d = 0; d < dims; ++d) {
      float lo = INFINITY, hi = -INFINITY;
      for (uint64_t c = c0 + lane; c < c1; c += 32) {
        lo = fminf(lo, child[(uint64_t)d * child_pad + c]);
        hi = fmaxf(hi, child[(uint64_t)(dims + d) * child_pad + c]);
      }
      lo = warp_min(lo);
      hi = warp_max(hi);
      if (lane == 0) {
        mbr[(uint64_t)d * pad + k] = lo;
        mbr[(uint64_t)(dims + d) * pad + k] = hi;
      }
    }
  }
}

uint32_t grid_for(uint64_t work, uint32_t per_block, uint32_t cap_blocks) {
  uint64_t g = (work + per_block - 1) / per_block;
  if (g < 1) g = 1;
  if (g > cap_blocks) g = cap_blocks;
  return (uint32_t)g;
}

}  // namespace

int num_sms() {
  static int sms = 0;
  if (!sms) {
    int dev = 0;
    cudaGetDevice(&dev);
    if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess || sms <= 0)
      sms = 148;
  }
  return sms;
}

// Temporaries freed before the work that uses them has run are taken from
// the device's stream-ordered pool (cudaMallocAsync / cudaFreeAsync): a
// buffer freed on one stream is handed to another stream only after the
// freeing stream has reached the free, so calls that run concurrently on
// different streams never share one.  The pool keeps what it caches.
qcp_status temp_alloc(size_t bytes, cudaStream_t s, void** out) {
  int dev = 0;
  QCP_CUDA(cudaGetDevice(&dev));
  static std::mutex mu;
  static bool kept[64] = {};
  if (dev >= 0 && dev < 64) {
    std::lock_guard<std::mutex> g(mu);
    if (!kept[dev]) {
      cudaMemPool_t mp;
      if (cudaDeviceGetDefaultMemPool(&mp, dev) == cudaSuccess) {
        uint64_t keep = UINT64_MAX;
        cudaMemPoolSetAttribute(mp, cudaMemPoolAttrReleaseThreshold, &keep);
      }
      kept[dev] = true;
    }
  }
  QCP_CUDA(cudaMallocAsync(out, bytes ? bytes : 1, s));
  return QCP_OK;
}

void temp_free(void* p, cudaStream_t s) {
  if (p) cudaFreeAsync(p, s);
}

size_t scan_scratch_bytes(uint64_t n) {
  return sizeof(uint64_t) * (size_t)((n + SC_CHUNK - 1) / SC_CHUNK + 1);
}

// The chunk sums live in `scratch` when the caller passes one (at least
// scan_scratch_bytes(n) bytes), else in a stream-ordered temporary.  Captured
// pipelines pass scratch: a temporary would become a graph memory node,
// whose physical memory the driver maps at a launch that needs more of it
// than the graphs already running hold.
template <class T>
qcp_status exclusive_scan(const T* in, T* out, uint64_t n, T* grand_total, DevPool& pool,
                          cudaStream_t s, void* scratch, size_t scratch_bytes) {
  (void)pool;
  const uint32_t nblk = (uint32_t)((n + SC_CHUNK - 1) / SC_CHUNK);
  void* sums = scratch;
  if (scratch) {
    if (scratch_bytes < sizeof(T) * (nblk ? nblk : 1)) {
      set_error("exclusive_scan: scratch too small");
      return QCP_ERR_BAD_ARG;
    }
  } else {
    QCP_TRY(temp_alloc(sizeof(T) * (nblk ? nblk : 1), s, &sums));
  }
  if (n) {
    k_scan_sums<T><<<nblk, SC_THREADS, 0, s>>>(in, n, (T*)sums);
    k_scan_partials<T><<<1, 1024, 0, s>>>((T*)sums, nblk, grand_total);
    k_scan_apply<T><<<nblk, SC_THREADS, 0, s>>>(in, out, n, (T*)sums);
    note_launch(3);
  }
  qcp_status st = check_launch("exclusive_scan");
  if (!scratch) temp_free(sums, s);
  return st;
}

template qcp_status exclusive_scan<uint32_t>(const uint32_t*, uint32_t*, uint64_t, uint32_t*,
                                             DevPool&, cudaStream_t, void*, size_t);
template qcp_status exclusive_scan<uint64_t>(const uint64_t*, uint64_t*, uint64_t, uint64_t*,
                                             DevPool&, cudaStream_t, void*, size_t);

qcp_status build_keys(const float* objs, uint64_t n, uint32_t dims, uint32_t is_rect,
                      uint32_t key_mode, uint32_t key_bits, uint64_t* keys, uint32_t* vals,
                      cudaStream_t s) {
  const uint32_t grid = grid_for(n, 256, num_sms() * 16);
  QCP_DISPATCH_D(dims, (k_keys<DD><<<grid, 256, 0, s>>>(objs, n, is_rect, key_mode, key_bits, keys, vals)));
  note_launch();
  return check_launch("k_keys");
}

size_t radix_scratch_bytes(uint64_t n) {
  const uint64_t ntiles = (n + RS_TILE - 1) / RS_TILE;
  const uint64_t hn = 256ull * ntiles;
  return 2 * ((sizeof(uint32_t) * hn + 255) & ~(size_t)255) + scan_scratch_bytes(hn);
}

qcp_status radix_sort_pairs(uint64_t* keys, uint32_t* vals, uint64_t* keys_tmp, uint32_t* vals_tmp,
                            uint64_t n, uint32_t key_bits, DevPool& pool, cudaStream_t s,
                            bool* result_in_tmp, void* scratch, size_t scratch_bytes) {
  *result_in_tmp = false;
  if (n <= 1) return QCP_OK;
  const uint32_t ntiles = (uint32_t)((n + RS_TILE - 1) / RS_TILE);
  const uint64_t hn = 256ull * ntiles;
  void* hist = nullptr;
  void* offs = nullptr;
  void* sums = nullptr;  // the scan's chunk sums (caller scratch), else its own temporary
  size_t sums_bytes = 0;
  qcp_status st = QCP_OK;
  if (scratch) {
    // caller-owned scratch (a captured build): no allocation on the stream
    if (scratch_bytes < radix_scratch_bytes(n)) {
      set_error("radix_sort_pairs: scratch too small");
      return QCP_ERR_BAD_ARG;
    }
    const size_t hb = (sizeof(uint32_t) * hn + 255) & ~(size_t)255;
    hist = scratch;
    offs = static_cast<char*>(scratch) + hb;
    sums = static_cast<char*>(scratch) + 2 * hb;
    sums_bytes = scan_scratch_bytes(hn);
  } else {
    QCP_TRY(temp_alloc(sizeof(uint32_t) * hn, s, &hist));
    st = temp_alloc(sizeof(uint32_t) * hn, s, &offs);
    if (st != QCP_OK) {
      temp_free(hist, s);
      return st;
    }
  }
  uint64_t* kin = keys;
  uint32_t* vin = vals;
  uint64_t* kout = keys_tmp;
  uint32_t* vout = vals_tmp;
  const uint32_t passes = (key_bits + 7) / 8;
  for (uint32_t p = 0; p < passes && st == QCP_OK; ++p) {
    const uint32_t shift = 8 * p;
    k_rs_upsweep<<<ntiles, RS_THREADS, 0, s>>>(kin, n, shift, (uint32_t*)hist, ntiles);
    note_launch();
    st = exclusive_scan<uint32_t>((uint32_t*)hist, (uint32_t*)offs, hn, nullptr, pool, s, sums, sums_bytes);
    if (st != QCP_OK) break;
    k_rs_downsweep<<<ntiles, RS_THREADS, 0, s>>>(kin, vin, kout, vout, n, shift, (uint32_t*)offs,
                                                 ntiles);
    note_launch();
    st = check_launch("radix_sort_pairs");
    std::swap(kin, kout);
    std::swap(vin, vout);
    *result_in_tmp = !*result_in_tmp;
  }
  if (!scratch) {
    temp_free(hist, s);
    temp_free(offs, s);
  }
  return st;
}

qcp_status build_pack(qcp_index* ix, const float* objs, const uint32_t* perm, cudaStream_t s,
                      uint32_t* d_bad) {
  k_pack<<<grid_for(ix->npad, 256, num_sms() * 16), 256, 0, s>>>(objs, perm, ix->n, ix->npad,
                                                                 ix->ncoord, ix->coords, ix->ids,
                                                                 d_bad);
  note_launch();
  return check_launch("k_pack");
}

qcp_status build_levels(qcp_index* ix, cudaStream_t s) {
  const uint32_t threads = 256, wpb = threads / 32;
  k_leaf_mbr<<<grid_for(ix->level_pad[0], wpb, num_sms() * 32), threads, 0, s>>>(
      ix->coords, ix->n, ix->npad, ix->dims, ix->is_rect, ix->fanout, ix->level_nodes[0],
      ix->level_pad[0], ix->mbr[0]);
  note_launch();
  QCP_TRY(check_launch("k_leaf_mbr"));
  for (uint32_t l = 1; l < ix->levels; ++l) {
    k_level_mbr<<<grid_for(ix->level_pad[l], wpb, num_sms() * 32), threads, 0, s>>>(
        ix->mbr[l - 1], ix->level_nodes[l - 1], ix->level_pad[l - 1], ix->dims, ix->fanout,
        ix->level_nodes[l], ix->level_pad[l], ix->mbr[l]);
    note_launch();
    QCP_TRY(check_launch("k_level_mbr"));
  }
  return QCP_OK;
}

qcp_status exclusive_scan_counts(const uint64_t* counts, uint64_t* offsets, uint32_t q,
                                 DevPool& pool, cudaStream_t s, void* scratch, size_t scratch_bytes) {
  // offsets has q+1 entries; offsets[q] receives the total.
  if (q == 0) {
    QCP_CUDA(cudaMemsetAsync(offsets, 0, sizeof(uint64_t), s));
    return QCP_OK;
  }
  return exclusive_scan<uint64_t>(counts, offsets, q, offsets + q, pool, s, scratch, scratch_bytes);
}

}  // namespace qcp
