// Per-query sort of the output ids.
//
// The reference returns hit counts only; this library returns every query's
// hits as ascending input ids.  The traversal writes each query's ids in
// arbitrary order into its CSR slice; this file sorts every slice in place.
// The ids of one slice are distinct and lie in [0, n), so only the low
// `idbits` = ceil(log2 n) bits carry order.
//
// Every slice of more than one id is a job.  A job of at most kRegionCap ids
// is one region, sorted in place.  A larger job is first split into
// G = 2^g id windows (window = id >> (idbits - g), g chosen so that a window
// holds about kTargetRegion ids): tile histograms -> per-window bases ->
// every tile regrouped by window in shared memory and written as contiguous
// runs into the scratch buffer.  Each window is then one region.
//
// A region is sorted by one CTA.  Windows at most 2^kSpanBits ids wide are
// ranked through a bitmap: every id sets its bit, an exclusive popcount
// prefix over the bitmap words gives each id its rank, ids are placed at
// their rank in shared memory and leave in coalesced stores (no comparisons,
// no divergence).  Wider spans (small slices of large id ranges) are counted
// into 2048 buckets by their top bits (the atomic's return value is the id's
// slot in its bucket), a block scan gives bucket bases, each bucket (a few
// ids) is insertion-sorted.  A region holding more than kRegionCap ids (ids
// clustered in id space) is subdivided: its span is halved until each part
// fits, the parts are sorted by buckets and written in span order.
#include "qcp_internal.cuh"

namespace qcp {

namespace {

constexpr uint32_t kRegionCap = 8192;      // ids one CTA sorts at once
constexpr uint32_t kTargetRegion = 6144;   // ids per window aimed at
constexpr uint32_t kRegThreads = 256;
constexpr uint32_t kRegWarps = kRegThreads / 32;
constexpr uint32_t kBucketBits = 11;
constexpr uint32_t kBuckets = 1u << kBucketBits;
constexpr uint32_t kSpanBits = 17;         // widest window the bitmap path takes
constexpr uint32_t kBmWords = (1u << kSpanBits) / 32;  // 4096
constexpr uint32_t kMaxG = 10;             // at most 2^10 windows per job
constexpr uint32_t kTile = 4096;           // ids per partition tile
constexpr uint32_t kTileThreads = 256;
constexpr uint32_t kTileWarps = kTileThreads / 32;

struct Job {
  unsigned long long off;
  uint32_t size;
  uint32_t g;  // log2 of the window count
};

struct Region {
  unsigned long long off;
  uint32_t size;
  uint32_t info;  // bit 0: ids in the scratch buffer; bits 1..5: span bits; bits 8..: window
};

// ---------------------------------------------------------------------------
// Region sort
// ---------------------------------------------------------------------------
struct RegionSmem {
  uint32_t stage[kRegionCap];  // sorted ids on their way out
  union {
    struct {  // bucket path
      uint32_t cnt[kBuckets];
      uint32_t base[kBuckets];
      uint16_t slot[kRegionCap];
    } bk;
    struct {  // bitmap path
      uint32_t bm[kBmWords];
      uint32_t pre[kBmWords];  // exclusive popcount prefix per word
    } bmp;
  };
  uint32_t wtot[kRegWarps];
  uint32_t stack_lo[40];
  uint32_t stack_bits[40];
  uint32_t sp, count, pos;
};

// Block-wide exclusive scan of the bucket counts into base[] (kBuckets /
// kRegThreads consecutive buckets per thread).
__device__ __forceinline__ void scan_buckets(RegionSmem& s) {
  constexpr uint32_t kPer = kBuckets / kRegThreads;
  const uint32_t tid = threadIdx.x, lane = tid & 31, wp = tid >> 5;
  uint32_t c[kPer];
  uint32_t t = 0;
#pragma unroll
  for (uint32_t k = 0; k < kPer; ++k) {
    c[k] = s.bk.cnt[tid * kPer + k];
    t += c[k];
  }
  uint32_t x = t;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const uint32_t y = __shfl_up_sync(0xffffffffu, x, o);
    if (lane >= (uint32_t)o) x += y;
  }
  if (lane == 31) s.wtot[wp] = x;
  __syncthreads();
  uint32_t run = x - t;
  for (uint32_t k = 0; k < wp; ++k) run += s.wtot[k];
#pragma unroll
  for (uint32_t k = 0; k < kPer; ++k) {
    s.bk.base[tid * kPer + k] = run;
    run += c[k];
  }
  __syncthreads();
}

// Sorts the ids of src[off..off+size) that lie in [slo, slo + 2^sbits) --
// exactly `count` (<= kRegionCap) of them -- into out[dst..dst+count).  With
// filter == false every id of the range lies in the span (count == size).
// s.cnt must be zero on entry; it is zero again on exit.
__device__ void sort_span(const int32_t* src, unsigned long long off, uint32_t size, uint32_t slo,
                          uint32_t sbits, bool filter, uint32_t count, int32_t* out,
                          unsigned long long dst, RegionSmem& s) {
  const uint32_t tid = threadIdx.x;
  const uint32_t bshift = sbits > kBucketBits ? sbits - kBucketBits : 0;
  const uint64_t span = 1ull << sbits;
  if (!filter) {
    // 1. count into buckets; each id's slot in its bucket is kept by index
    for (uint32_t i0 = 0; i0 < size; i0 += kRegThreads * 8) {
      uint32_t v[8];
#pragma unroll
      for (int k = 0; k < 8; ++k) {
        const uint32_t i = i0 + k * kRegThreads + tid;
        v[k] = (i < size) ? (uint32_t)src[off + i] - slo : 0xffffffffu;
      }
#pragma unroll
      for (int k = 0; k < 8; ++k) {
        const uint32_t i = i0 + k * kRegThreads + tid;
        if (v[k] != 0xffffffffu) s.bk.slot[i] = (uint16_t)atomicAdd(&s.bk.cnt[v[k] >> bshift], 1u);
      }
    }
    __syncthreads();
    scan_buckets(s);
    // 2. place (the ids are read again, from L2)
    for (uint32_t i0 = 0; i0 < size; i0 += kRegThreads * 8) {
      uint32_t v[8];
#pragma unroll
      for (int k = 0; k < 8; ++k) {
        const uint32_t i = i0 + k * kRegThreads + tid;
        v[k] = (i < size) ? (uint32_t)src[off + i] - slo : 0xffffffffu;
      }
#pragma unroll
      for (int k = 0; k < 8; ++k) {
        const uint32_t i = i0 + k * kRegThreads + tid;
        if (v[k] != 0xffffffffu) s.stage[s.bk.base[v[k] >> bshift] + s.bk.slot[i]] = v[k];
      }
    }
  } else {
    // only the ids inside the span take part: count, scan, then place with
    // a second round of atomics for the slots
    for (uint32_t i = tid; i < size; i += kRegThreads) {
      const uint32_t r = (uint32_t)src[off + i] - slo;
      if ((uint64_t)r < span) atomicAdd(&s.bk.cnt[r >> bshift], 1u);
    }
    __syncthreads();
    scan_buckets(s);
    for (uint32_t i = tid; i < kBuckets; i += kRegThreads) s.bk.cnt[i] = 0;
    __syncthreads();
    for (uint32_t i = tid; i < size; i += kRegThreads) {
      const uint32_t r = (uint32_t)src[off + i] - slo;
      if ((uint64_t)r < span) {
        const uint32_t b = r >> bshift;
        s.stage[s.bk.base[b] + atomicAdd(&s.bk.cnt[b], 1u)] = r;
      }
    }
  }
  __syncthreads();
  // 3. insertion sort inside each bucket, clear the counts
  constexpr uint32_t kPer = kBuckets / kRegThreads;
#pragma unroll
  for (uint32_t k = 0; k < kPer; ++k) {
    const uint32_t b = tid * kPer + k;
    const uint32_t b0 = s.bk.base[b];
    const uint32_t n = s.bk.cnt[b];
    for (uint32_t i = 1; i < n; ++i) {
      const uint32_t key = s.stage[b0 + i];
      uint32_t j = i;
      while (j > 0 && s.stage[b0 + j - 1] > key) {
        s.stage[b0 + j] = s.stage[b0 + j - 1];
        --j;
      }
      s.stage[b0 + j] = key;
    }
    s.bk.cnt[b] = 0;
  }
  __syncthreads();
  // 4. coalesced copy out
  for (uint32_t i = tid; i < count; i += kRegThreads) __stcs(out + dst + i, (int32_t)(s.stage[i] + slo));
  __syncthreads();
}

// Sorts the `size` (<= kRegionCap) distinct ids of src[off..) -- all in
// [lo, lo + 2^sbits), sbits <= kSpanBits -- into out[off..) by rank: every id
// sets its bit in a bitmap of the span, an exclusive popcount prefix over the
// bitmap words gives the number of smaller ids before each word, so an id's
// rank is pre[word] + popc(word & bits below it).  No id is compared and no
// thread diverges.  The bucket counters (which share this memory) are zero
// on entry and zero again on exit.
__device__ void sort_span_bitmap(const int32_t* src, unsigned long long off, uint32_t size, uint32_t lo,
                                 uint32_t sbits, int32_t* out, RegionSmem& s) {
  const uint32_t tid = threadIdx.x, lane = tid & 31, wp = tid >> 5;
  const uint32_t nwords = ((1u << sbits) + 31) >> 5;           // <= kBmWords
  constexpr uint32_t kPer = kBmWords / kRegThreads;            // 16 words per thread
  uint4* bm4 = reinterpret_cast<uint4*>(s.bmp.bm);
  for (uint32_t i = tid; i < kBmWords / 4; i += kRegThreads) bm4[i] = make_uint4(0, 0, 0, 0);
  __syncthreads();
  for (uint32_t i0 = 0; i0 < size; i0 += kRegThreads * 8) {
    uint32_t v[8];
#pragma unroll
    for (int k = 0; k < 8; ++k) {
      const uint32_t i = i0 + k * kRegThreads + tid;
      v[k] = (i < size) ? (uint32_t)src[off + i] - lo : 0xffffffffu;
    }
#pragma unroll
    for (int k = 0; k < 8; ++k)
      if (v[k] != 0xffffffffu) atomicOr(&s.bmp.bm[v[k] >> 5], 1u << (v[k] & 31));
  }
  __syncthreads();
  // exclusive popcount prefix: each thread owns kPer consecutive words
  uint32_t c[kPer];
  uint32_t t = 0;
  const uint32_t w0 = tid * kPer;
#pragma unroll
  for (uint32_t k = 0; k < kPer; k += 4) {
    const uint4 q = (w0 + k < nwords) ? bm4[(w0 + k) / 4] : make_uint4(0, 0, 0, 0);
    c[k] = __popc(q.x);
    c[k + 1] = __popc(q.y);
    c[k + 2] = __popc(q.z);
    c[k + 3] = __popc(q.w);
    t += c[k] + c[k + 1] + c[k + 2] + c[k + 3];
  }
  uint32_t x = t;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const uint32_t y = __shfl_up_sync(0xffffffffu, x, o);
    if (lane >= (uint32_t)o) x += y;
  }
  if (lane == 31) s.wtot[wp] = x;
  __syncthreads();
  uint32_t run = x - t;
  for (uint32_t k = 0; k < wp; ++k) run += s.wtot[k];
  uint4* pre4 = reinterpret_cast<uint4*>(s.bmp.pre);
#pragma unroll
  for (uint32_t k = 0; k < kPer; k += 4) {
    uint4 q;
    q.x = run;
    q.y = q.x + c[k];
    q.z = q.y + c[k + 1];
    q.w = q.z + c[k + 2];
    run = q.w + c[k + 3];
    pre4[(w0 + k) / 4] = q;
  }
  __syncthreads();
  // rank and place (ids read again, from L2)
  for (uint32_t i0 = 0; i0 < size; i0 += kRegThreads * 8) {
    uint32_t v[8];
#pragma unroll
    for (int k = 0; k < 8; ++k) {
      const uint32_t i = i0 + k * kRegThreads + tid;
      v[k] = (i < size) ? (uint32_t)src[off + i] - lo : 0xffffffffu;
    }
#pragma unroll
    for (int k = 0; k < 8; ++k) {
      if (v[k] == 0xffffffffu) continue;
      const uint32_t w = v[k] >> 5;
      const uint32_t below = s.bmp.bm[w] & ((1u << (v[k] & 31)) - 1u);
      s.stage[s.bmp.pre[w] + __popc(below)] = v[k];
    }
  }
  __syncthreads();
  for (uint32_t i = tid; i < size; i += kRegThreads) __stcs(out + off + i, (int32_t)(s.stage[i] + lo));
  // restore the zero bucket counters that alias the bitmap
  for (uint32_t i = tid; i < kBuckets; i += kRegThreads) s.bk.cnt[i] = 0;
  __syncthreads();
}

// Persistent CTAs over the regions.
__global__ void __launch_bounds__(kRegThreads) k_region_sort(const Region* __restrict__ regions, uint32_t nreg,
                                                             const int32_t* out_src, const int32_t* tmp_src,
                                                             int32_t* out) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  RegionSmem& s = *reinterpret_cast<RegionSmem*>(smem_raw);
  const uint32_t tid = threadIdx.x;
  for (uint32_t i = tid; i < kBuckets; i += kRegThreads) s.bk.cnt[i] = 0;
  __syncthreads();
  for (uint32_t r = blockIdx.x; r < nreg; r += gridDim.x) {
    const Region rg = regions[r];
    const int32_t* src = (rg.info & 1u) ? tmp_src : out_src;
    const uint32_t sbits = (rg.info >> 1) & 31u;
    const uint32_t lo = (rg.info >> 8) << sbits;
    if (rg.size == 0) continue;
    if (rg.size == 1) {
      if (tid == 0) out[rg.off] = src[rg.off];
      continue;
    }
    if (rg.size <= kRegionCap) {
      if (sbits <= kSpanBits)
        sort_span_bitmap(src, rg.off, rg.size, lo, sbits, out, s);
      else
        sort_span(src, rg.off, rg.size, lo, sbits, false, rg.size, out, rg.off, s);
      continue;
    }
    // more ids than one pass holds: halve the span until every part fits,
    // emitting the parts in span order (only windows of split jobs get here,
    // so src is the scratch buffer and out can be written while src is read)
    if (tid == 0) {
      s.sp = 1;
      s.stack_lo[0] = lo;
      s.stack_bits[0] = sbits;
      s.pos = 0;
    }
    __syncthreads();
    while (s.sp > 0) {
      const uint32_t top = s.sp - 1;
      const uint32_t slo = s.stack_lo[top], sb = s.stack_bits[top];
      __syncthreads();
      if (tid == 0) {
        s.sp = top;
        s.count = 0;
      }
      __syncthreads();
      uint32_t c = 0;
      const uint64_t span = 1ull << sb;
      for (uint32_t i = tid; i < rg.size; i += kRegThreads)
        c += ((uint64_t)((uint32_t)src[rg.off + i] - slo) < span) ? 1u : 0u;
      for (int o = 16; o > 0; o >>= 1) c += __shfl_xor_sync(0xffffffffu, c, o);
      if ((tid & 31) == 0 && c) atomicAdd(&s.count, c);
      __syncthreads();
      const uint32_t count = s.count;
      if (count > kRegionCap) {
        if (tid == 0) {  // the upper half goes below the lower half on the stack
          const uint32_t h = sb - 1;
          s.stack_lo[s.sp] = slo + (1u << h);
          s.stack_bits[s.sp] = h;
          s.stack_lo[s.sp + 1] = slo;
          s.stack_bits[s.sp + 1] = h;
          s.sp += 2;
        }
      } else if (count > 0) {
        sort_span(src, rg.off, rg.size, slo, sb, true, count, out, rg.off + s.pos, s);
        if (tid == 0) s.pos += count;
      }
      __syncthreads();
    }
  }
}

// ---------------------------------------------------------------------------
// Jobs and window partition
// ---------------------------------------------------------------------------
__device__ __forceinline__ uint32_t ceil_log2(uint32_t x) { return x <= 1 ? 0 : 32 - __clz(x - 1); }

__global__ void k_classify(const unsigned long long* __restrict__ offsets, uint32_t q, uint32_t idbits,
                           Job* jobs, uint32_t* njobs) {
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < q; i += gridDim.x * blockDim.x) {
    const unsigned long long off = offsets[i];
    const unsigned long long sz = offsets[i + 1] - off;
    if (sz <= 1) continue;
    Job j;
    j.off = off;
    j.size = (uint32_t)sz;
    uint32_t g = 0;
    if (sz > kRegionCap) {
      // windows narrow enough for the bitmap path and small enough to fit
      g = ceil_log2((uint32_t)((sz + kTargetRegion - 1) / kTargetRegion));
      if (idbits > kSpanBits) g = max(g, idbits - kSpanBits);
      g = min(g, min(kMaxG, idbits));
    }
    j.g = g;
    jobs[atomicAdd(njobs, 1u)] = j;
  }
}

// Per job: windows (1 for g == 0) and partition tiles (0 for g == 0).
__global__ void k_job_counts(const Job* __restrict__ jobs, uint32_t njobs, uint32_t* nwin, uint32_t* ntile) {
  for (uint32_t j = blockIdx.x * blockDim.x + threadIdx.x; j < njobs; j += gridDim.x * blockDim.x) {
    const Job jb = jobs[j];
    nwin[j] = 1u << jb.g;
    ntile[j] = jb.g ? (jb.size + kTile - 1) / kTile : 0u;
  }
}

__global__ void k_tile_map(const uint32_t* __restrict__ tiles, const uint32_t* __restrict__ tile_off,
                           uint32_t njobs, uint32_t* map) {
  for (uint32_t j = blockIdx.x; j < njobs; j += gridDim.x) {
    const uint32_t t0 = tile_off[j], nt = tiles[j];
    for (uint32_t k = threadIdx.x; k < nt; k += blockDim.x) map[t0 + k] = j;
  }
}

// Window histogram of every tile -> whist[woff[job] + window].  Each warp
// counts into its own shared counters (no contention across warps).
__global__ void __launch_bounds__(kTileThreads) k_win_hist(const Job* __restrict__ jobs,
                                                           const uint32_t* __restrict__ map,
                                                           const uint32_t* __restrict__ tile_off,
                                                           uint32_t ntiles, const int32_t* __restrict__ src,
                                                           uint32_t idbits, const uint32_t* __restrict__ woff,
                                                           uint32_t* whist) {
  extern __shared__ uint32_t h[];  // [kTileWarps][G]
  const uint32_t wp = threadIdx.x >> 5;
  for (uint32_t t = blockIdx.x; t < ntiles; t += gridDim.x) {
    const uint32_t j = map[t];
    const Job jb = jobs[j];
    const uint32_t G = 1u << jb.g;
    const uint32_t shift = idbits - jb.g;
    for (uint32_t w = threadIdx.x; w < G * kTileWarps; w += kTileThreads) h[w] = 0;
    __syncthreads();
    const uint32_t b0 = (t - tile_off[j]) * kTile;
    const uint32_t b1 = min(b0 + kTile, jb.size);
    uint32_t v[kTile / kTileThreads];
#pragma unroll
    for (uint32_t k = 0; k < kTile / kTileThreads; ++k) {
      const uint32_t i = b0 + k * kTileThreads + threadIdx.x;
      v[k] = (i < b1) ? (uint32_t)__ldcs(src + jb.off + i) : 0xffffffffu;
    }
    uint32_t* hw = h + wp * G;
#pragma unroll
    for (uint32_t k = 0; k < kTile / kTileThreads; ++k)
      if (v[k] != 0xffffffffu) atomicAdd(&hw[v[k] >> shift], 1u);
    __syncthreads();
    for (uint32_t w = threadIdx.x; w < G; w += kTileThreads) {
      uint32_t c = 0;
      for (uint32_t k = 0; k < kTileWarps; ++k) c += h[k * G + w];
      if (c) atomicAdd(&whist[woff[j] + w], c);
    }
    __syncthreads();
  }
}

// Per job: exclusive scan over its window counts -> write cursors, and the
// job's regions (one per window, or the whole slice for g == 0).
__global__ void __launch_bounds__(kTileThreads) k_win_scan(const Job* __restrict__ jobs, uint32_t njobs,
                                                           uint32_t idbits, const uint32_t* __restrict__ woff,
                                                           const uint32_t* __restrict__ whist,
                                                           unsigned long long* wcur, Region* regions) {
  __shared__ uint32_t wt[kTileThreads / 32];
  const uint32_t lane = threadIdx.x & 31, wp = threadIdx.x >> 5;
  for (uint32_t j = blockIdx.x; j < njobs; j += gridDim.x) {
    const Job jb = jobs[j];
    const uint32_t base = woff[j];
    if (jb.g == 0) {
      if (threadIdx.x == 0) {
        Region r;
        r.off = jb.off;
        r.size = jb.size;
        r.info = (idbits << 1);  // ids in out, window 0, span = all ids
        regions[base] = r;
      }
      continue;
    }
    const uint32_t G = 1u << jb.g;
    const uint32_t sbits = idbits - jb.g;
    const uint32_t per = (G + kTileThreads - 1) / kTileThreads;
    const uint32_t w0 = threadIdx.x * per;
    uint32_t s = 0;
    for (uint32_t k = 0; k < per; ++k)
      if (w0 + k < G) s += whist[base + w0 + k];
    uint32_t x = s;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const uint32_t y = __shfl_up_sync(0xffffffffu, x, o);
      if (lane >= (uint32_t)o) x += y;
    }
    if (lane == 31) wt[wp] = x;
    __syncthreads();
    uint32_t before = 0;
    for (uint32_t k = 0; k < wp; ++k) before += wt[k];
    unsigned long long run = jb.off + before + x - s;
    for (uint32_t k = 0; k < per; ++k) {
      const uint32_t w = w0 + k;
      if (w < G) {
        const uint32_t c = whist[base + w];
        wcur[base + w] = run;
        Region r;
        r.off = run;
        r.size = c;
        r.info = (w << 8) | (sbits << 1) | 1u;  // ids in the scratch buffer
        regions[base + w] = r;
        run += c;
      }
    }
    __syncthreads();
  }
}

// Each tile: regroup its ids by window in shared memory, reserve the window
// ranges with one atomic per nonempty window, write contiguous runs.  Each
// warp counts into its own shared counters; the counter's old value is the
// id's slot among its warp's ids of that window (the order inside a window
// does not matter, the region sort orders it).
__global__ void __launch_bounds__(kTileThreads) k_win_scatter(const Job* __restrict__ jobs,
                                                              const uint32_t* __restrict__ map,
                                                              const uint32_t* __restrict__ tile_off,
                                                              uint32_t ntiles, const int32_t* __restrict__ src,
                                                              int32_t* __restrict__ dst, uint32_t idbits,
                                                              const uint32_t* __restrict__ woff,
                                                              unsigned long long* wcur) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  unsigned long long* gstart = reinterpret_cast<unsigned long long*>(smem_raw);  // [G]
  uint32_t* lbase = reinterpret_cast<uint32_t*>(gstart + (1u << kMaxG));       // [G]
  uint32_t* cnt = lbase + (1u << kMaxG);                                        // [kTileWarps][G]
  __shared__ uint32_t stage[kTile];
  __shared__ uint32_t wt[kTileThreads / 32];
  const uint32_t lane = threadIdx.x & 31, wp = threadIdx.x >> 5;
  for (uint32_t t = blockIdx.x; t < ntiles; t += gridDim.x) {
    const uint32_t j = map[t];
    const Job jb = jobs[j];
    const uint32_t G = 1u << jb.g;
    const uint32_t shift = idbits - jb.g;
    for (uint32_t w = threadIdx.x; w < G * kTileWarps; w += kTileThreads) cnt[w] = 0;
    __syncthreads();
    const uint32_t b0 = (t - tile_off[j]) * kTile;
    const uint32_t n = min(b0 + kTile, jb.size) - b0;
    uint32_t v[kTile / kTileThreads];
    uint32_t slot[kTile / kTileThreads];
#pragma unroll
    for (uint32_t k = 0; k < kTile / kTileThreads; ++k) {
      const uint32_t i = k * kTileThreads + threadIdx.x;
      v[k] = (i < n) ? (uint32_t)__ldcs(src + jb.off + b0 + i) : 0xffffffffu;
    }
    uint32_t* cw = cnt + wp * G;
#pragma unroll
    for (uint32_t k = 0; k < kTile / kTileThreads; ++k)
      slot[k] = (v[k] != 0xffffffffu) ? atomicAdd(&cw[v[k] >> shift], 1u) : 0u;
    __syncthreads();
    // per window: exclusive scan over (window, warp) -> each warp's base in
    // the tile's window-grouped order; window totals reserve global ranges
    const uint32_t per = (G + kTileThreads - 1) / kTileThreads;
    const uint32_t w0 = threadIdx.x * per;
    uint32_t s = 0;
    for (uint32_t k = 0; k < per; ++k) {
      const uint32_t w = w0 + k;
      if (w < G)
        for (uint32_t q = 0; q < kTileWarps; ++q) s += cnt[q * G + w];
    }
    uint32_t x = s;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const uint32_t y = __shfl_up_sync(0xffffffffu, x, o);
      if (lane >= (uint32_t)o) x += y;
    }
    if (lane == 31) wt[wp] = x;
    __syncthreads();
    uint32_t run = x - s;
    for (uint32_t k = 0; k < wp; ++k) run += wt[k];
    for (uint32_t k = 0; k < per; ++k) {
      const uint32_t w = w0 + k;
      if (w < G) {
        lbase[w] = run;
        uint32_t tot = 0;
        for (uint32_t q = 0; q < kTileWarps; ++q) {
          const uint32_t c = cnt[q * G + w];
          cnt[q * G + w] = run + tot;  // now: this warp's first slot in the tile
          tot += c;
        }
        if (tot) gstart[w] = atomicAdd(&wcur[woff[j] + w], (unsigned long long)tot);
        run += tot;
      }
    }
    __syncthreads();
#pragma unroll
    for (uint32_t k = 0; k < kTile / kTileThreads; ++k)
      if (v[k] != 0xffffffffu) stage[cw[v[k] >> shift] + slot[k]] = v[k];
    __syncthreads();
    for (uint32_t i = threadIdx.x; i < n; i += kTileThreads) {
      const uint32_t id = stage[i];
      const uint32_t w = id >> shift;
      dst[gstart[w] + (i - lbase[w])] = (int32_t)id;
    }
    __syncthreads();
  }
}

}  // namespace

qcp_status ws_reserve_sort(qcp_index* ix, Workspace* ws, size_t jobs, size_t tiles);

qcp_status segmented_sort(qcp_index* ix, Workspace* ws, uint32_t q, cudaStream_t s) {
  ws->sort_small_jobs = ws->sort_msd_jobs = 0;
  ws->sort_part_marked = false;
  if (q == 0) return QCP_OK;
  uint32_t idbits = 1;
  while (idbits < 31 && (1ull << idbits) < ix->n) ++idbits;
  const uint32_t sms = (uint32_t)num_sms();
  const size_t region_bytes = sizeof(RegionSmem);
  const size_t hist_bytes = sizeof(uint32_t) * kTileWarps * (1u << kMaxG);
  const size_t scatter_bytes = (sizeof(unsigned long long) + sizeof(uint32_t) * (1 + kTileWarps)) * (1u << kMaxG);
  static thread_local int attrs_device = -1;  // attributes are per device
  if (attrs_device != ix->device) {
    QCP_CUDA(cudaFuncSetAttribute(k_region_sort, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)region_bytes));
    QCP_CUDA(cudaFuncSetAttribute(k_win_hist, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)hist_bytes));
    QCP_CUDA(cudaFuncSetAttribute(k_win_scatter, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)scatter_bytes));
    attrs_device = ix->device;
  }
  QCP_TRY(ws_reserve_sort(ix, ws, (size_t)q + 256, 0));
  uint32_t* ctr = ws->ctr;
  QCP_CUDA(cudaMemsetAsync(ctr + kCtrJobs0, 0, sizeof(uint32_t), s));
  Job* jobs = reinterpret_cast<Job*>(ws->jobs[0]);
  k_classify<<<(q + 255) / 256, 256, 0, s>>>((const unsigned long long*)ws->offsets, q, idbits, jobs,
                                             ctr + kCtrJobs0);
  note_launch();
  QCP_CUDA(cudaMemcpyAsync(ws->h_ctr, ctr, sizeof(uint32_t) * kCtrCount, cudaMemcpyDeviceToHost, s));
  QCP_CUDA(cudaStreamSynchronize(s));
  const uint32_t njobs = ws->h_ctr[kCtrJobs0];
  if (njobs == 0) return QCP_OK;

  // per-job tables: windows, tiles and their offsets
  const size_t tbytes = (size_t)njobs * 16 + 64;
  void* tables = nullptr;
  QCP_TRY(ix->pool.get(tbytes, &tables));
  uint32_t* nwin = reinterpret_cast<uint32_t*>(tables);
  uint32_t* woff = nwin + njobs;
  uint32_t* ntile = woff + njobs;
  uint32_t* toff = ntile + njobs;
  void* wtables = nullptr;
  size_t wbytes = 0;
  qcp_status st = QCP_OK;
  do {
    k_job_counts<<<(njobs + 255) / 256, 256, 0, s>>>(jobs, njobs, nwin, ntile);
    note_launch();
    if ((st = exclusive_scan<uint32_t>(nwin, woff, njobs, ctr + kCtrWork, ix->pool, s)) != QCP_OK) break;
    if ((st = exclusive_scan<uint32_t>(ntile, toff, njobs, ctr + kCtrWork2, ix->pool, s)) != QCP_OK) break;
    if (cudaMemcpyAsync(ws->h_ctr, ctr, sizeof(uint32_t) * kCtrCount, cudaMemcpyDeviceToHost, s) != cudaSuccess ||
        cudaStreamSynchronize(s) != cudaSuccess) {
      st = cuda_status(cudaGetLastError(), "segmented sort tables");
      break;
    }
    const uint32_t nreg = ws->h_ctr[kCtrWork];
    const uint32_t ntiles = ws->h_ctr[kCtrWork2];
    ws->sort_small_jobs = njobs;
    ws->sort_msd_jobs = nreg;
    // per-window tables: regions (16 B), cursors (u64), counts (u32)
    wbytes = (size_t)nreg * (16 + 8 + 4) + 64;
    if ((st = ix->pool.get(wbytes, &wtables)) != QCP_OK) {
      wtables = nullptr;
      break;
    }
    Region* regions = reinterpret_cast<Region*>(wtables);
    unsigned long long* wcur = reinterpret_cast<unsigned long long*>(regions + nreg);
    uint32_t* whist = reinterpret_cast<uint32_t*>(wcur + nreg);
    if (cudaMemsetAsync(whist, 0, sizeof(uint32_t) * nreg, s) != cudaSuccess) {
      st = cuda_status(cudaGetLastError(), "memset");
      break;
    }
    mark(ws, kEvSortSmall, s);
    if (ntiles) {
      if ((st = ws_reserve_sort(ix, ws, 0, ntiles)) != QCP_OK) break;
      k_tile_map<<<min(njobs, sms * 8), 256, 0, s>>>(ntile, toff, njobs, ws->seg_hist);
      k_win_hist<<<min(ntiles, sms * 8), kTileThreads, hist_bytes, s>>>(jobs, ws->seg_hist, toff, ntiles,
                                                                       ws->out_ids, idbits, woff, whist);
      note_launch(2);
    }
    k_win_scan<<<min(njobs, sms * 16), kTileThreads, 0, s>>>(jobs, njobs, idbits, woff, whist, wcur, regions);
    note_launch();
    if (ntiles) {
      k_win_scatter<<<min(ntiles, sms * 4), kTileThreads, scatter_bytes, s>>>(
          jobs, ws->seg_hist, toff, ntiles, ws->out_ids, ws->tmp_ids, idbits, woff, wcur);
      note_launch();
    }
    mark(ws, kEvSortPart, s);
    ws->sort_part_marked = ws->timing;
    k_region_sort<<<min(nreg, sms * 4), kRegThreads, region_bytes, s>>>(regions, nreg, ws->out_ids,
                                                                       ws->tmp_ids, ws->out_ids);
    note_launch();
    st = check_launch("segmented sort");
    // the tables go back to the pool below: make sure the kernels are done
    if (st == QCP_OK && cudaStreamSynchronize(s) != cudaSuccess) st = cuda_status(cudaGetLastError(), "sort");
  } while (false);
  if (wtables) ix->pool.put(wbytes, wtables);
  ix->pool.put(tbytes, tables);
  return st;
}

}  // namespace qcp
