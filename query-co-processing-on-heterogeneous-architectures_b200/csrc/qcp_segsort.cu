// Per-query sort of the output ids.
//
// The reference returns hit counts only; this library returns every query's
// hits as ascending input ids.  The traversal writes each query's ids in
// arbitrary order into its CSR slice; this file sorts every slice in place.
// The ids of one slice are distinct and lie in [0, n), so only the low
// `idbits` = ceil(log2 n) bits carry order.
//
//   slice <= kTinyCap ids   one warp bucket-sorts it in shared memory (256
//                           buckets, a few ids each, insertion-sorted);
//   slice <= kSmallCap ids  one CTA bucket-sorts it in shared memory: ids
//                           are counted into 2048 buckets by their top bits
//                           (the atomic's return value is the id's slot in
//                           its bucket), a block scan gives bucket bases,
//                           each bucket (a few ids) is insertion-sorted and
//                           the order leaves in coalesced stores.
//   larger slices           1. window partition: ids are split by
//                              id >> wbits (wbits = min(idbits, 18)) into
//                              G = 2^(idbits - wbits) windows: tile
//                              histograms -> per-slice window bases -> every
//                              tile regrouped by window in shared memory and
//                              written as contiguous runs into the scratch
//                              buffer;
//                           2. each (slice, window) of more than
//                              kWinWarpMax ids is sorted through a bitmap of
//                              its 2^wbits possible ids: every id sets its
//                              bit, every thread counts the set bits of its
//                              words, and after a CTA prefix enumerates them
//                              in order -- no comparisons; the smaller
//                              windows are bucket-sorted by one warp each.
#include "qcp_internal.cuh"
#include "qcp_tree.cuh"

namespace qcp {

namespace {

// ---- tiny slices (one warp each) --------------------------------------------
constexpr uint32_t kTinyCap = 1024;                    // ids of a slice sorted by one warp
constexpr uint32_t kTinyBuckets = 256;                 // buckets of the warp's counting pass
constexpr uint32_t kTinyWarps = 8;                     // warps per CTA
constexpr uint32_t kWinWarpMax = 512;                  // windows of at most this many ids: one warp each
// ---- small slices ----------------------------------------------------------
constexpr uint32_t kSmallCap = kSmallSliceCap;
constexpr uint32_t kSmallThreads = 256;
constexpr uint32_t kSmallWarps = kSmallThreads / 32;
constexpr uint32_t kBucketBits = 11;
constexpr uint32_t kBuckets = 1u << kBucketBits;
// ---- window partition ------------------------------------------------------
constexpr uint32_t kWinBits = 18;
// 128 threads x 16 ids per tile, 10 CTAs per SM: the partition's per-tile
// chain (counts, scan, one global atomic per window, barriers) is latency-
// bound, and more, smaller CTAs keep more chains in flight per SM
constexpr uint32_t kTile = kSortTile;
constexpr uint32_t kTileThreads = 128;
constexpr uint32_t kTileBlocks = 10;  // launch bound of k_win_scatter (registers for 10 CTAs per SM)
constexpr uint32_t kTileWarps = kTileThreads / 32;
constexpr uint32_t kPerWarpMaxG = 256;  // per-warp window counters up to this G
// ---- window sort ------------------------------------------------------------
// One instantiation per window size 2^BITS ids (BITS = 16, 17, 18).  Each
// thread owns kLaneWords bitmap words (32 for 2^17- and 2^18-id windows, 16
// for 2^16): a window's per-window bookkeeping is paid per warp, so fewer
// warps per window cost fewer instructions per id, and more bits per thread
// even out the enumeration's lanes.  Shared memory sets the resident CTAs per
// SM (kBlocks: 3, 6, 10); the launch takes the occupancy API's count.
template <uint32_t BITS>
struct WinCfg {
  static constexpr uint32_t kWords = (1u << BITS) / 32;            // bitmap words
  static constexpr uint32_t kLaneWords = BITS >= 17 ? 32u : 16u;   // bitmap words per thread
  static constexpr uint32_t kThreads = kWords / kLaneWords;        // 256, 128, 128
  static constexpr uint32_t kWarps = kThreads / 32;
  static constexpr uint32_t kBlocks = BITS >= 18 ? 3u : (BITS == 17 ? 6u : 10u);  // resident CTAs per SM
  // the launch bound: registers for kBlocks CTAs per SM (shared memory allows
  // no more); tighter caps (~40 registers) measured 5 % slower
  static constexpr uint32_t kStage = BITS >= 18 ? 6144u : (BITS == 17 ? 3072u : 1408u);  // staged output ids
  static constexpr uint32_t kPrefetch = 4096u >> (18 - BITS);      // ids of the next window loaded ahead
};
constexpr uint32_t kBatch = 8;                         // ids per thread per load round
constexpr uint32_t kNone = 0xffffffffu;                // empty register slot

using Job = SortJob;

// ============================================================================
// Small slices: bucket sort
// ============================================================================
struct BucketSmem {
  uint32_t stage[kSmallCap];
  uint32_t cnt[kBuckets];
  uint32_t base[kBuckets];
  uint16_t slot[kSmallCap];
  uint32_t wtot[kSmallWarps];
};

// Slices of at most kTinyCap ids, one warp each (no CTA barriers): the ids
// are loaded into registers (32 per lane, all loads in flight together) and
// counted into kTinyBuckets buckets by their top bits, a warp scan gives the
// bucket bases, every id takes the next slot of its bucket, each lane insertion-sorts its 8 buckets (a few ids each) and the
// slice leaves in coalesced stores.  Jobs of more ids are k_sort_small's.
struct TinySmem {
  uint32_t stage[kTinyWarps][kTinyCap];
  uint32_t cnt[kTinyWarps][kTinyBuckets];
  uint32_t base[kTinyWarps][kTinyBuckets];
};

// One warp sorts the size <= CAP (<= kTinyCap) distinct ids at src into dst
// (src may equal dst): buckets by (id - lo) >> bshift (every id's bucket
// below kTinyBuckets), then the steps above.  The warp's counters are zero
// on entry and on return.
template <uint32_t CAP>
__device__ __forceinline__ void warp_bucket_sort(const int32_t* src, int32_t* dst, uint32_t size, uint32_t lo,
                                                 uint32_t bshift, uint32_t* stage, uint32_t* cnt, uint32_t* base,
                                                 uint32_t lane) {
  constexpr uint32_t kPer = kTinyBuckets / 32;  // buckets per lane
  // 1. the slice into registers (all loads in flight at once), bucket counts
  static_assert(CAP % 32 == 0 && CAP <= kTinyCap, "one warp's stage holds kTinyCap ids");
  constexpr uint32_t kPerLane = CAP / 32;
  uint32_t v[kPerLane];
#pragma unroll
  for (uint32_t k = 0; k < kPerLane; ++k) {
    const uint32_t i = lane + 32 * k;
    v[k] = (i < size) ? (uint32_t)__ldg(src + i) : kNone;
  }
#pragma unroll
  for (uint32_t k = 0; k < kPerLane; ++k)
    if (v[k] != kNone) atomicAdd(&cnt[(v[k] - lo) >> bshift], 1u);
  __syncwarp();
  // 2. bucket bases: each lane owns kPer consecutive buckets
  uint32_t c[kPer];
  uint32_t t = 0;
#pragma unroll
  for (uint32_t k = 0; k < kPer; ++k) {
    c[k] = cnt[lane * kPer + k];
    t += c[k];
  }
  uint32_t tot;
  uint32_t run = warp_excl_sum(t, &tot);
#pragma unroll
  for (uint32_t k = 0; k < kPer; ++k) {
    base[lane * kPer + k] = run;
    run += c[k];
  }
  __syncwarp();
  // 3. every id to the next slot of its bucket (order inside a bucket is
  //    settled below)
#pragma unroll
  for (uint32_t k = 0; k < kPerLane; ++k)
    if (v[k] != kNone) stage[atomicAdd(&base[(v[k] - lo) >> bshift], 1u)] = v[k];
  __syncwarp();
  // 4. insertion sort of each bucket [base - count, base); counts cleared
#pragma unroll
  for (uint32_t k = 0; k < kPer; ++k) {
    const uint32_t n = c[k];
    const uint32_t b0 = base[lane * kPer + k] - n;
    for (uint32_t i = 1; i < n; ++i) {
      const uint32_t key = stage[b0 + i];
      uint32_t jj = i;
      while (jj > 0 && stage[b0 + jj - 1] > key) {
        stage[b0 + jj] = stage[b0 + jj - 1];
        --jj;
      }
      stage[b0 + jj] = key;
    }
    cnt[lane * kPer + k] = 0;
  }
  __syncwarp();
  for (uint32_t i = lane; i < size; i += 32) __stcs(dst + i, (int32_t)stage[i]);
  __syncwarp();
}

__global__ void __launch_bounds__(kTinyWarps * 32, 3) k_sort_tiny(const Job* __restrict__ jobs,
                                                               const uint32_t* __restrict__ njobs_p,
                                                               int32_t* out, uint32_t idbits) {
  const uint32_t njobs = *njobs_p;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  TinySmem& sm = *reinterpret_cast<TinySmem*>(smem_raw);
  const uint32_t lane = threadIdx.x & 31, wp = threadIdx.x >> 5;
  constexpr uint32_t kPer = kTinyBuckets / 32;
  const uint32_t bshift = idbits > 8 ? idbits - 8 : 0;
#pragma unroll
  for (uint32_t k = 0; k < kPer; ++k) sm.cnt[wp][lane * kPer + k] = 0;
  __syncwarp();
  const uint32_t warps = gridDim.x * kTinyWarps;
  for (uint32_t j = blockIdx.x * kTinyWarps + wp; j < njobs; j += warps) {
    const Job jb = jobs[j];
    if (jb.size > kTinyCap) continue;  // warp-uniform
    warp_bucket_sort<kTinyCap>(out + jb.off, out + jb.off, jb.size, 0u, bshift, sm.stage[wp], sm.cnt[wp], sm.base[wp],
                               lane);
  }
}

// Windows of at most kWinWarpMax ids (listed by k_win_split), one warp
// each: the window's ids at src + wbase[g] in ascending order to
// dst + wbase[g], bucketed on their low wbits bits.
__global__ void __launch_bounds__(kTinyWarps * 32, 3) k_win_sort_warp(const uint32_t* __restrict__ list,
                                                                   const uint32_t* __restrict__ nlist_p, uint32_t G,
                                                                   uint32_t wbits, const uint32_t* __restrict__ whist,
                                                                   const unsigned long long* __restrict__ wbase,
                                                                   const int32_t* __restrict__ src, int32_t* dst) {
  const uint32_t nlist = *nlist_p;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  TinySmem& sm = *reinterpret_cast<TinySmem*>(smem_raw);
  const uint32_t lane = threadIdx.x & 31, wp = threadIdx.x >> 5;
  constexpr uint32_t kPer = kTinyBuckets / 32;
  const uint32_t bshift = wbits > 8 ? wbits - 8 : 0;
#pragma unroll
  for (uint32_t k = 0; k < kPer; ++k) sm.cnt[wp][lane * kPer + k] = 0;
  __syncwarp();
  const uint32_t warps = gridDim.x * kTinyWarps;
  for (uint32_t i = blockIdx.x * kTinyWarps + wp; i < nlist; i += warps) {
    const uint32_t g = list[i];
    const unsigned long long off = wbase[g];
    const uint32_t lo = (g & (G - 1)) << wbits;
    warp_bucket_sort<kWinWarpMax>(src + off, dst + off, whist[g], lo, bshift, sm.stage[wp], sm.cnt[wp], sm.base[wp],
                                  lane);
  }
}

// The (job, window) pairs into two lists: windows of 1..kWinWarpMax ids for
// k_win_sort_warp, larger ones for k_win_sort (one atomic per warp and
// list).  With big_ids, the ids of the large windows are added to it.
__global__ void k_win_split(const uint32_t* __restrict__ njobs_p, uint32_t G, const uint32_t* __restrict__ whist,
                            uint32_t* big, uint32_t* nbig, uint32_t* small, uint32_t* nsmall,
                            unsigned long long* big_ids) {
  const uint32_t total = *njobs_p * G;
  const uint32_t lane = threadIdx.x & 31;
  const uint32_t stride = gridDim.x * blockDim.x;
  for (uint32_t g0 = blockIdx.x * blockDim.x; g0 < total; g0 += stride) {  // warp-uniform rounds
    const uint32_t g = g0 + threadIdx.x;
    const uint32_t sz = g < total ? whist[g] : 0u;
    const bool is_small = sz >= 1 && sz <= kWinWarpMax, is_big = sz > kWinWarpMax;
    const uint32_t ms = __ballot_sync(0xffffffffu, is_small), mb = __ballot_sync(0xffffffffu, is_big);
    uint32_t bs = 0, bb = 0;
    if (lane == 0) {
      if (ms) bs = atomicAdd(nsmall, (uint32_t)__popc(ms));
      if (mb) bb = atomicAdd(nbig, (uint32_t)__popc(mb));
    }
    bs = __shfl_sync(0xffffffffu, bs, 0);
    bb = __shfl_sync(0xffffffffu, bb, 0);
    const uint32_t lt = lane_lt_mask();
    if (is_small) small[bs + __popc(ms & lt)] = g;
    if (is_big) big[bb + __popc(mb & lt)] = g;
    if (big_ids) {
      const uint32_t ids = __reduce_add_sync(0xffffffffu, is_big ? sz : 0u);
      if (lane == 0 && ids) atomicAdd(big_ids, (unsigned long long)ids);
    }
  }
}

// jobs_end: one past the last job; job j is jobs_end[-1 - j].
__global__ void __launch_bounds__(kSmallThreads) k_sort_small(const Job* __restrict__ jobs_end,
                                                              const uint32_t* __restrict__ njobs_p,
                                                              int32_t* out, uint32_t idbits) {
  const uint32_t njobs = *njobs_p;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  BucketSmem& s = *reinterpret_cast<BucketSmem*>(smem_raw);
  const uint32_t tid = threadIdx.x, lane = tid & 31, wp = tid >> 5;
  const uint32_t bshift = idbits > kBucketBits ? idbits - kBucketBits : 0;
  constexpr uint32_t kPer = kBuckets / kSmallThreads;  // buckets per thread
  for (uint32_t i = tid; i < kBuckets; i += kSmallThreads) s.cnt[i] = 0;
  __syncthreads();
  for (uint32_t j = blockIdx.x; j < njobs; j += gridDim.x) {
    const Job jb = jobs_end[-1 - (long long)j];
    const uint32_t size = jb.size;
    // 1. count into buckets; each id's slot in its bucket is kept by index
    for (uint32_t i0 = 0; i0 < size; i0 += kSmallThreads * 8) {
      uint32_t v[8];
#pragma unroll
      for (int k = 0; k < 8; ++k) {
        const uint32_t i = i0 + k * kSmallThreads + tid;
        v[k] = (i < size) ? (uint32_t)out[jb.off + i] : 0xffffffffu;
      }
#pragma unroll
      for (int k = 0; k < 8; ++k) {
        const uint32_t i = i0 + k * kSmallThreads + tid;
        if (v[k] != 0xffffffffu) s.slot[i] = (uint16_t)atomicAdd(&s.cnt[v[k] >> bshift], 1u);
      }
    }
    __syncthreads();
    // 2. bucket bases
    uint32_t c[kPer];
    uint32_t t = 0;
#pragma unroll
    for (uint32_t k = 0; k < kPer; ++k) {
      c[k] = s.cnt[tid * kPer + k];
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
      s.base[tid * kPer + k] = run;
      run += c[k];
    }
    __syncthreads();
    // 3. place (ids read again, from L2); every id is read before any write
    for (uint32_t i0 = 0; i0 < size; i0 += kSmallThreads * 8) {
      uint32_t v[8];
#pragma unroll
      for (int k = 0; k < 8; ++k) {
        const uint32_t i = i0 + k * kSmallThreads + tid;
        v[k] = (i < size) ? (uint32_t)out[jb.off + i] : 0xffffffffu;
      }
#pragma unroll
      for (int k = 0; k < 8; ++k) {
        const uint32_t i = i0 + k * kSmallThreads + tid;
        if (v[k] != 0xffffffffu) s.stage[s.base[v[k] >> bshift] + s.slot[i]] = v[k];
      }
    }
    __syncthreads();
    // 4. insertion sort inside each bucket, clear the counts
#pragma unroll
    for (uint32_t k = 0; k < kPer; ++k) {
      const uint32_t b0 = s.base[tid * kPer + k];
      const uint32_t n = c[k];
      for (uint32_t i = 1; i < n; ++i) {
        const uint32_t key = s.stage[b0 + i];
        uint32_t jj = i;
        while (jj > 0 && s.stage[b0 + jj - 1] > key) {
          s.stage[b0 + jj] = s.stage[b0 + jj - 1];
          --jj;
        }
        s.stage[b0 + jj] = key;
      }
      s.cnt[tid * kPer + k] = 0;
    }
    __syncthreads();
    for (uint32_t i = tid; i < size; i += kSmallThreads) __stcs(out + jb.off + i, (int32_t)s.stage[i]);
    __syncthreads();
  }
}

// ============================================================================
// Window partition
// ============================================================================
// Job lists by slice size: slices of <= kTinyCap ids from the front of
// `small` (count *ntiny), slices of <= kSmallCap ids from its back (small[cap -
// 1 - k], count *nsmall), larger ones in `big`.  Slices of 0 or 1 ids are
// sorted already.
__global__ void k_classify(const unsigned long long* __restrict__ offsets, uint32_t q, Job* small,
                           uint32_t* ntiny, uint32_t* nsmall, size_t cap, Job* big, uint32_t* nbig,
                           unsigned long long* big_ids) {
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < q; i += gridDim.x * blockDim.x) {
    const unsigned long long off = offsets[i];
    const unsigned long long sz = offsets[i + 1] - off;
    if (sz <= 1) continue;
    Job j;
    j.off = off;
    j.size = (uint32_t)sz;
    j.q = i;
    if (sz <= kTinyCap) {
      small[atomicAdd(ntiny, 1u)] = j;
    } else if (sz <= kSmallCap) {
      small[cap - 1 - atomicAdd(nsmall, 1u)] = j;
    } else {
      big[atomicAdd(nbig, 1u)] = j;
      if (big_ids) atomicAdd(big_ids, sz);
    }
  }
}

// tiles[j] for j < nmax: tiles of job j, 0 past the job count
__global__ void k_tiles_per_job(const Job* __restrict__ jobs, const uint32_t* __restrict__ njobs_p, uint32_t nmax,
                                uint32_t* tiles) {
  const uint32_t njobs = *njobs_p;
  for (uint32_t j = blockIdx.x * blockDim.x + threadIdx.x; j < nmax; j += gridDim.x * blockDim.x)
    tiles[j] = j < njobs ? (jobs[j].size + kTile - 1) / kTile : 0u;
}

__global__ void k_tile_map(const uint32_t* __restrict__ tiles, const uint32_t* __restrict__ tile_off,
                           const uint32_t* __restrict__ njobs_p, uint32_t* map) {
  const uint32_t njobs = *njobs_p;
  for (uint32_t j = blockIdx.x; j < njobs; j += gridDim.x) {
    const uint32_t t0 = tile_off[j], nt = tiles[j];
    for (uint32_t k = threadIdx.x; k < nt; k += blockDim.x) map[t0 + k] = j;
  }
}

// Window histogram of every tile -> whist[job * G + window].
__global__ void __launch_bounds__(kTileThreads) k_win_hist(const Job* __restrict__ jobs,
                                                           const uint32_t* __restrict__ map,
                                                           const uint32_t* __restrict__ tile_off,
                                                           const uint32_t* __restrict__ ntiles_p, const int32_t* __restrict__ src,
                                                           uint32_t G, uint32_t wbits, uint32_t* whist) {
  const uint32_t ntiles = *ntiles_p;
  extern __shared__ uint32_t h[];  // [G]
  for (uint32_t t = blockIdx.x; t < ntiles; t += gridDim.x) {
    for (uint32_t w = threadIdx.x; w < G; w += kTileThreads) h[w] = 0;
    __syncthreads();
    const uint32_t j = map[t];
    const Job jb = jobs[j];
    const uint32_t b0 = (t - tile_off[j]) * kTile;
    const uint32_t b1 = min(b0 + kTile, jb.size);
    uint32_t v[kTile / kTileThreads];
#pragma unroll
    for (uint32_t k = 0; k < kTile / kTileThreads; ++k) {
      const uint32_t i = b0 + k * kTileThreads + threadIdx.x;
      v[k] = (i < b1) ? (uint32_t)__ldcs(src + jb.off + i) : 0xffffffffu;
    }
#pragma unroll
    for (uint32_t k = 0; k < kTile / kTileThreads; ++k)
      if (v[k] != 0xffffffffu) atomicAdd(&h[v[k] >> wbits], 1u);
    __syncthreads();
    for (uint32_t w = threadIdx.x; w < G; w += kTileThreads)
      if (h[w]) atomicAdd(&whist[(size_t)j * G + w], h[w]);
    __syncthreads();
  }
}

// Per job: exclusive scan over its G window counts -> bases and cursors.
// With qwhist (the write pass's per-(query, window) counts) the job's counts
// are read from its query's row and copied to whist for k_win_sort.
__global__ void __launch_bounds__(kTileThreads) k_win_scan(const Job* __restrict__ jobs,
                                                           const uint32_t* __restrict__ njobs_p,
                                                           uint32_t G, uint32_t* __restrict__ whist,
                                                           const uint32_t* __restrict__ qwhist,
                                                           unsigned long long* wbase,
                                                           unsigned long long* wcur) {
  const uint32_t njobs = *njobs_p;
  __shared__ uint32_t wt[kTileWarps];
  const uint32_t lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  const uint32_t per = (G + kTileThreads - 1) / kTileThreads;
  for (uint32_t j = blockIdx.x; j < njobs; j += gridDim.x) {
    const size_t base = (size_t)j * G;
    const uint32_t w0 = threadIdx.x * per;
    if (qwhist) {
      const size_t qbase = (size_t)jobs[j].q * G;
      for (uint32_t k = 0; k < per; ++k)
        if (w0 + k < G) whist[base + w0 + k] = qwhist[qbase + w0 + k];
    }
    uint32_t s = 0;
    for (uint32_t k = 0; k < per; ++k)
      if (w0 + k < G) s += whist[base + w0 + k];
    uint32_t x = s;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const uint32_t y = __shfl_up_sync(0xffffffffu, x, o);
      if (lane >= (uint32_t)o) x += y;
    }
    if (lane == 31) wt[w] = x;
    __syncthreads();
    uint32_t before = 0;
    for (uint32_t k = 0; k < w; ++k) before += wt[k];
    unsigned long long run = jobs[j].off + before + x - s;
    for (uint32_t k = 0; k < per; ++k) {
      if (w0 + k < G) {
        wbase[base + w0 + k] = run;
        wcur[base + w0 + k] = run;
        run += whist[base + w0 + k];
      }
    }
    __syncthreads();
  }
}

// Each tile: regroup its ids by window in shared memory, reserve the window
// ranges with one atomic per nonempty window, write contiguous runs.  With
// G <= kPerWarpMaxG each warp counts into its own counters (the counter's
// old value is the id's slot among its warp's ids of that window); the
// order inside a window does not matter, the ranking orders it.
__global__ void __launch_bounds__(kTileThreads, kTileBlocks) k_win_scatter(const Job* __restrict__ jobs,
                                                              const uint32_t* __restrict__ map,
                                                              const uint32_t* __restrict__ tile_off,
                                                              const uint32_t* __restrict__ ntiles_p, const int32_t* __restrict__ src,
                                                              int32_t* __restrict__ dst, uint32_t G,
                                                              uint32_t wbits, unsigned long long* wcur) {
  const uint32_t ntiles = *ntiles_p;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const uint32_t nw = (G <= kPerWarpMaxG) ? kTileWarps : 1u;  // counter sets
  unsigned long long* gstart = reinterpret_cast<unsigned long long*>(smem_raw);  // [G]
  uint32_t* cnt = reinterpret_cast<uint32_t*>(gstart + G);                     // [nw][G]
  uint32_t* stage = cnt + nw * G;                                               // [kTile]
  __shared__ uint32_t wt[kTileWarps];
  const uint32_t lane = threadIdx.x & 31, wp = threadIdx.x >> 5;
  uint32_t* cw = cnt + (nw == 1 ? 0u : wp) * G;
  for (uint32_t t = blockIdx.x; t < ntiles; t += gridDim.x) {
    for (uint32_t w = threadIdx.x; w < nw * G; w += kTileThreads) cnt[w] = 0;
    __syncthreads();
    const uint32_t j = map[t];
    const Job jb = jobs[j];
    const uint32_t b0 = (t - tile_off[j]) * kTile;
    const uint32_t n = min(b0 + kTile, jb.size) - b0;
    uint32_t v[kTile / kTileThreads];
    uint32_t slot[kTile / kTileThreads];
#pragma unroll
    for (uint32_t k = 0; k < kTile / kTileThreads; ++k) {
      const uint32_t i = k * kTileThreads + threadIdx.x;
      v[k] = (i < n) ? (uint32_t)__ldcs(src + jb.off + b0 + i) : 0xffffffffu;
    }
#pragma unroll
    for (uint32_t k = 0; k < kTile / kTileThreads; ++k)
      slot[k] = (v[k] != 0xffffffffu) ? atomicAdd(&cw[v[k] >> wbits], 1u) : 0u;
    __syncthreads();
    // exclusive scan over (window, counter set) in window-major order
    const uint32_t per = (G + kTileThreads - 1) / kTileThreads;
    const uint32_t w0 = threadIdx.x * per;
    uint32_t s = 0;
    for (uint32_t k = 0; k < per; ++k)
      if (w0 + k < G)
        for (uint32_t q = 0; q < nw; ++q) s += cnt[q * G + w0 + k];
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
        uint32_t tot = 0;
        for (uint32_t q = 0; q < nw; ++q) {
          const uint32_t c = cnt[q * G + w];
          cnt[q * G + w] = run + tot;  // first slot of this counter set in the tile
          tot += c;
        }
        // output position of the tile's id at stage slot i of window w:
        // gstart[w] + i (the window's start minus its local base)
        if (tot) gstart[w] = atomicAdd(&wcur[(size_t)j * G + w], (unsigned long long)tot) - run;
        run += tot;
      }
    }
    __syncthreads();
#pragma unroll
    for (uint32_t k = 0; k < kTile / kTileThreads; ++k)
      if (v[k] != 0xffffffffu) stage[cw[v[k] >> wbits] + slot[k]] = v[k];
    __syncthreads();
    for (uint32_t i = threadIdx.x; i < n; i += kTileThreads) {
      const uint32_t id = stage[i];
      const uint32_t w = id >> wbits;
      dst[gstart[w] + i] = (int32_t)id;
    }
    __syncthreads();
  }
}

// ============================================================================
// Window sort
// ============================================================================
template <uint32_t BITS>
struct RankSmem {
  uint64_t bar;                             // completion of the window's bulk prefetch
  uint64_t pad_;
  uint32_t bm[WinCfg<BITS>::kWords];        // one bit per possible id of the window
  // output ranks [0, kStage) of the window, rank r at stage[r + (off & 3)] so
  // that the stage and the output share their 16-byte alignment
  int32_t stage[WinCfg<BITS>::kStage + 4];
  // first ids of the next window, loaded ahead: id i of a window at offset
  // off is at pf[i + (off & 3)]
  int32_t pf[WinCfg<BITS>::kPrefetch + 4];
  uint32_t wsum[WinCfg<BITS>::kWarps];      // set bits in each warp's word range
};

// Shared -> global bulk copy (the TMA unit) of `bytes` (a multiple of 16,
// both addresses 16-byte aligned), tracked as a bulk async-group.
__device__ __forceinline__ void bulk_copy_s2g(void* gdst, const void* ssrc, uint32_t bytes) {
  asm volatile("cp.async.bulk.global.shared::cta.bulk_group [%0], [%1], %2;\n" ::"l"(gdst),
               "r"(static_cast<uint32_t>(__cvta_generic_to_shared(ssrc))), "r"(bytes)
               : "memory");
  asm volatile("cp.async.bulk.commit_group;\n" ::: "memory");
}
// Until the issued bulk stores have read their shared-memory source.
__device__ __forceinline__ void bulk_wait_read() { asm volatile("cp.async.bulk.wait_group.read 0;\n" ::: "memory"); }
// Until the issued bulk stores are complete.
__device__ __forceinline__ void bulk_wait_all() { asm volatile("cp.async.bulk.wait_group 0;\n" ::: "memory"); }
// Generic-proxy writes to shared memory before async-proxy reads of them.
__device__ __forceinline__ void fence_proxy_async_smem() { asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory"); }

// Bit position of the highest set bit of x (x != 0).
__device__ __forceinline__ uint32_t bfind32(uint32_t x) {
  uint32_t b;
  asm("bfind.u32 %0, %1;" : "=r"(b) : "r"(x));
  return b;
}

// Position of bitmap word w in shared memory (see k_win_sort).
template <uint32_t BITS>
__device__ __forceinline__ uint32_t bm_at(uint32_t w) {
  return (w % WinCfg<BITS>::kLaneWords) * WinCfg<BITS>::kThreads + w / WinCfg<BITS>::kLaneWords;
}

// Persistent CTAs over the listed (job, window) pairs g = job * G + window
// (the windows of more than kWinWarpMax ids).
//   1. every id of window g (read from src, the scratch buffer) sets its bit
//      in a bitmap of the window's 2^wbits possible ids; its first kPrefetch
//      ids were brought into shared memory by a bulk copy (the TMA unit)
//      while the previous window ran;
//   2. every thread owns kLaneWords bitmap words: it counts their set bits,
//      takes its exclusive prefix over the CTA (warp scan + warp sums), i.e.
//      its ranks [pos, pos + cnt), then walks its nonzero words from the
//      highest down and emits the id of every set bit from its highest rank
//      down (bfind finds the highest set bit in one instruction), clearing
//      each word it read; ranks below kStage go to a shared-memory stage,
//      larger ones straight to the output;
//   3. the stage leaves by one bulk store (its 16-byte-aligned middle) and a
//      few plain stores (the ends).
// Warp 0 alone issues the next window's prefetch and the copy-out (their
// 64-bit offset arithmetic is per CTA, not per thread).  Three CTA barriers
// per window: bitmap complete, warp sums ready, stage complete (which also
// orders the bitmap's clearing before the next window's bits).  The ids of a
// window are distinct, so the set bits are the window's ids and their
// enumeration in bit order is the window in ascending order.  G is a power
// of two.
template <uint32_t BITS>
__global__ void __launch_bounds__(WinCfg<BITS>::kThreads, WinCfg<BITS>::kBlocks)
    k_win_sort(const uint32_t* __restrict__ list, const uint32_t* __restrict__ nlist_p, uint32_t G, uint32_t wbits,
               const uint32_t* __restrict__ whist, const unsigned long long* __restrict__ wbase,
               const int32_t* __restrict__ src, int32_t* __restrict__ out, uint32_t* err) {
  using C = WinCfg<BITS>;
  constexpr uint32_t kRankThreads = C::kThreads;
  constexpr uint32_t kRankWarps = C::kWarps;
  constexpr uint32_t kBmWords = C::kWords;
  constexpr uint32_t kStage = C::kStage;
  constexpr uint32_t kPrefetch = C::kPrefetch;
  const uint32_t total = *nlist_p;  // listed (job, window) pairs
  extern __shared__ __align__(16) unsigned char smem_raw[];
  RankSmem<BITS>& s = *reinterpret_cast<RankSmem<BITS>*>(smem_raw);
  const uint32_t tid = threadIdx.x, lane = tid & 31, wp = tid >> 5;
  uint4* bm4 = reinterpret_cast<uint4*>(s.bm);
  const uint32_t nwords = (1u << wbits) >> 5;   // 12 <= wbits <= BITS
  constexpr uint32_t kLaneWords = C::kLaneWords;
  const uint32_t tw0 = tid * kLaneWords;        // this thread's words [tw0, tw0 + kLaneWords)
  const bool owner = tw0 < nwords;
  // Word w of the bitmap (thread w / kLaneWords's word w % kLaneWords) is
  // stored at bm_at(w) = (w % kLaneWords) * kRankThreads + w / kLaneWords, so
  // that the lanes of a warp reading or clearing one word each of their own
  // ranges always hit 32 distinct banks.
  for (uint32_t i = tid; i < kBmWords / 4; i += kRankThreads) bm4[i] = make_uint4(0, 0, 0, 0);
  if (tid == 0) {
    mbar_init(&s.bar, 1);
    mbar_fence_init();
  }
  __syncthreads();
  // The first kPrefetch ids of window g + gridDim.x are copied into s.pf
  // while window g is enumerated: their 16-byte-aligned middle [a0, a1) by
  // one bulk copy (thread 0, completing on s.bar, one barrier phase per
  // window even when it is empty); the up to 3 + 3 ids around it are loaded
  // into registers by threads 0..5 and written to s.pf by store_edge.  Every
  // thread waits on s.bar itself, so the bulk part needs no CTA barrier.
  auto prefetch_range = [&](unsigned long long o, uint32_t sz, unsigned long long* a0,
                            unsigned long long* a1) {
    const uint32_t n = sz < kPrefetch ? sz : kPrefetch;
    *a0 = (o + 3) & ~3ull;
    *a1 = (o + n) & ~3ull;
    if (*a1 < *a0) *a1 = *a0;
  };
  // The up to 3 + 3 ids around the bulk part: threads 0..5 load one each
  // into a register when the prefetch is issued and store it into s.pf only
  // before the window's last barrier, so the load's latency is hidden behind
  // the enumeration.
  int32_t edge_v = 0;
  int32_t edge_at = -1;  // s.pf slot of this thread's edge id, -1: none
  auto prefetch = [&](unsigned long long o, uint32_t sz) {
    unsigned long long a0, a1;
    prefetch_range(o, sz, &a0, &a1);
    const unsigned long long al = o & ~3ull;
    if (tid == 0) {
      mbar_arrive_expect_tx(&s.bar, (uint32_t)(a1 - a0) * 4u);
      if (a1 > a0) bulk_copy_g2s(&s.pf[a0 - al], src + a0, (uint32_t)(a1 - a0) * 4u, &s.bar);
    }
    const unsigned long long end = o + (sz < kPrefetch ? sz : kPrefetch);
    const unsigned long long h1 = a0 < end ? a0 : end;          // head [o, h1)
    const unsigned long long t0 = a1 > h1 ? a1 : h1;            // tail [t0, end)
    unsigned long long e = ~0ull;
    if (tid < 3 && o + tid < h1) e = o + tid;
    else if (tid >= 3 && tid < 6 && t0 + (tid - 3) < end) e = t0 + (tid - 3);
    edge_at = -1;
    if (e != ~0ull) {
      edge_v = __ldcs(src + e);
      edge_at = (int32_t)(e - al);
    }
  };
  auto store_edge = [&]() {
    if (edge_at >= 0) s.pf[edge_at] = edge_v;
    edge_at = -1;
  };
  uint32_t phase = 0;
  uint32_t size = 0;
  unsigned long long off = 0;
  if (blockIdx.x < total) {
    const uint32_t g0 = list[blockIdx.x];
    size = whist[g0];
    off = wbase[g0];
    if (wp == 0) prefetch(off, size);
  }
  store_edge();
  __syncthreads();
  for (uint32_t li = blockIdx.x; li < total; li += gridDim.x) {
    const uint32_t g = list[li];
    const uint32_t ln = li + gridDim.x;  // this CTA's next listed window
    uint32_t nsize = 0;
    unsigned long long noff = 0;
    if (ln < total) {
      const uint32_t gn = list[ln];
      nsize = whist[gn];
      noff = wbase[gn];
    }
    const int32_t* in = src + off;
    int32_t* dst = out + off;
    const uint32_t lo = (g & (G - 1)) << wbits;
    const uint32_t sh = (uint32_t)(off & 3);  // 16-byte alignment offset of this window's ids
    // this window's prefetched ids (every thread waits itself; the bitmap
    // was cleared and the stage written before the previous window's last
    // barrier), and the stage free of the previous window's bulk store
    const bool ok = mbar_wait_bounded(&s.bar, phase);
    phase ^= 1u;
    if (tid == 0) bulk_wait_read();
    // 1. set one bit per id: the prefetched ones from shared memory, the
    //    rest in rounds whose loads are all issued before the first atomic
    if (size >= 2 && ok) {
      const uint32_t npf = size < kPrefetch ? size : kPrefetch;
      for (uint32_t i = tid; i < npf; i += kRankThreads) {
        const uint32_t x = (uint32_t)s.pf[i + sh] - lo;
        atomicOr(&s.bm[bm_at<BITS>(x >> 5)], 1u << (x & 31));
      }
      for (uint32_t i0 = kPrefetch; i0 < size; i0 += kBatch * kRankThreads) {
        uint32_t a[kBatch];
#pragma unroll
        for (uint32_t k = 0; k < kBatch; ++k) {
          const uint32_t i = i0 + k * kRankThreads + tid;
          a[k] = kNone;
          if (i0 + k * kRankThreads + (wp << 5) < size && i < size) a[k] = (uint32_t)__ldcs(in + i) - lo;
        }
#pragma unroll
        for (uint32_t k = 0; k < kBatch; ++k)
          if (i0 + k * kRankThreads + (wp << 5) < size && a[k] != kNone)
            atomicOr(&s.bm[bm_at<BITS>(a[k] >> 5)], 1u << (a[k] & 31));
      }
    } else if (size == 1 && tid == 0) {
      dst[0] = s.pf[sh];
    }
    if (__syncthreads_or(!ok)) {  // bitmap complete; s.pf free
      // a bulk copy did not complete in time: flag it and stop (the results
      // are invalid); wait once more, again bounded, for that copy
      if (tid == 0) atomicOr(err, 1u);
      mbar_wait_bounded(&s.bar, phase ^ 1u);
      break;
    }
    if (ln < total && wp == 0) prefetch(noff, nsize);
    if (size < 2) {
      store_edge();
      __syncthreads();  // the next window's edge ids are in place
      size = nsize;
      off = noff;
      continue;  // uniform over the CTA
    }
    // 2a. set bits and nonzero words of this thread's range
    uint32_t cnt = 0, nz = 0;
    if (owner) {
#pragma unroll
      for (uint32_t k = 0; k < kLaneWords; ++k) {
        const uint32_t c = __popc(s.bm[k * kRankThreads + tid]);
        cnt += c;
        nz += min(c, 1u) << k;  // bit k: word k is nonzero
      }
    }
    uint32_t wtot;
    const uint32_t ex = warp_excl_sum(cnt, &wtot);
    if (lane == 0) s.wsum[wp] = wtot;
    __syncthreads();
    // 2b. enumerate the set bits in order
    const uint32_t ws = lane < kRankWarps ? s.wsum[lane] : 0u;
    uint32_t pos = __reduce_add_sync(0xffffffffu, lane < wp ? ws : 0u) + ex;
    // one iteration per set bit (a flat loop: a warp runs as many iterations
    // as its lane with the most bits), from rank pos + cnt - 1 down to pos;
    // the next lower nonzero word is fetched, and cleared, when the current
    // one is used up.  Ranks from kStage up go straight to the output, the
    // rest to the stage, in two loops so that no iteration tests the rank.
    uint32_t cur = 0, base = 0;
    const uint32_t base0 = lo + (tw0 << 5);  // id of bit 0 of this thread's first word
    uint32_t r = pos + cnt;
    const uint32_t split = max(pos, min(r, kStage));  // ranks >= split go straight out
    auto next_bit = [&]() -> uint32_t {
      if (cur == 0) {
        const uint32_t wi = bfind32(nz);
        nz ^= 1u << wi;
        cur = s.bm[wi * kRankThreads + tid];
        s.bm[wi * kRankThreads + tid] = 0u;
        base = base0 + (wi << 5);
      }
      const uint32_t b = bfind32(cur);
      cur ^= 1u << b;
      return base + b;
    };
    while (r > split) {
      const uint32_t id = next_bit();
      dst[--r] = (int32_t)id;
    }
    int32_t* st = s.stage + sh;
    while (r > pos) {
      const uint32_t id = next_bit();
      st[--r] = (int32_t)id;
    }
    store_edge();              // the next window's edge ids, before the last barrier
    fence_proxy_async_smem();  // the stage's writes before the bulk store reads them
    __syncthreads();
    // 3. staged ranks out (warp 0): the 16-byte-aligned middle by one bulk
    //    store, the up to 3 + 3 ids around it by plain stores; windows of
    //    fewer than 8 ids by plain stores
    const uint32_t ns = size < kStage ? size : kStage;
    if (wp == 0) {
      const unsigned long long al = off & ~3ull;
      const unsigned long long b0 = (off + 3) & ~3ull, b1 = (off + ns) & ~3ull;
      if (b1 > b0) {
        if (tid == 0) bulk_copy_s2g(out + b0, &s.stage[b0 - al], (uint32_t)(b1 - b0) * 4u);
        const uint32_t nh = (uint32_t)(b0 - off), nt = (uint32_t)(off + ns - b1);
        if (tid < nh) out[off + tid] = s.stage[sh + tid];
        else if (tid >= 4 && tid - 4 < nt) out[b1 + (tid - 4)] = s.stage[b1 - al + (tid - 4)];
      } else {
        for (uint32_t k = lane; k < ns; k += 32) dst[k] = s.stage[sh + k];
      }
    }
    size = nsize;
    off = noff;
  }
  if (tid == 0) bulk_wait_all();
}

}  // namespace

qcp_status ws_reserve_sort(qcp_index* ix, Workspace* ws, size_t jobs, size_t tiles);

// Blocks of k_win_scatter resident per SM with `smem` bytes of dynamic shared
// memory (its registers, not its shared memory, are the usual limit): the
// persistent grid is this many blocks per SM, so that no block waits for a
// second wave.
static uint32_t scatter_blocks_per_sm(size_t smem) {
  int b = 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b, k_win_scatter, kTileThreads, smem) != cudaSuccess || b < 1) {
    cudaGetLastError();
    b = 1;
  }
  return (uint32_t)b;
}

static uint32_t id_bits(uint64_t n) {
  uint32_t idbits = 1;
  while (idbits < 31 && (1ull << idbits) < n) ++idbits;
  return idbits;
}

// The window sort for 2^wbits-id windows (the instantiation whose bitmap
// holds them), over at most `max_pairs` (job, window) pairs.
template <uint32_t BITS>
static void launch_win_sort_t(uint64_t max_pairs, uint32_t sms, const uint32_t* list, const uint32_t* nlist,
                              uint32_t G, uint32_t wbits, const uint32_t* whist, const unsigned long long* wbase,
                              const int32_t* src, int32_t* out, uint32_t* err, cudaStream_t s) {
  using C = WinCfg<BITS>;
  // resident CTAs per SM from the occupancy API (its shared memory decides),
  // once per device and thread
  static thread_local int occ_dev = -1;
  static thread_local uint32_t occ = C::kBlocks;
  int dev = 0;
  if (cudaGetDevice(&dev) == cudaSuccess && dev != occ_dev) {
    int b = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b, k_win_sort<BITS>, C::kThreads, sizeof(RankSmem<BITS>)) ==
            cudaSuccess &&
        b > 0) {
      occ = (uint32_t)b;
      occ_dev = dev;
    } else {
      cudaGetLastError();
    }
  }
  const uint64_t cap = (uint64_t)sms * occ;
  const uint32_t grid = (uint32_t)(max_pairs < cap ? max_pairs : cap);
  if (grid)
    k_win_sort<BITS><<<grid, C::kThreads, sizeof(RankSmem<BITS>), s>>>(list, nlist, G, wbits, whist, wbase, src, out,
                                                                       err);
}

// The windows of a call: k_win_split lists them (counts in ctr[kCtrWinBig],
// ctr[kCtrWinSmall], zeroed by the caller), the bitmap sort takes the large
// ones and one warp each the small ones.  lists holds 2 * max_pairs entries;
// max_pairs bounds the (job, window) pairs.
static void launch_win_sort(Workspace* ws, uint64_t max_pairs, uint32_t sms, const uint32_t* njobs, uint32_t G,
                            uint32_t wbits, const uint32_t* whist, const unsigned long long* wbase, uint32_t* lists,
                            uint32_t* ctr, const int32_t* src, int32_t* out, uint32_t* err, cudaStream_t s,
                            bool stats) {
  uint32_t* big = lists;
  uint32_t* small = lists + max_pairs;
  const uint64_t split_blocks = (max_pairs + 255) / 256;
  k_win_split<<<(uint32_t)(split_blocks < (uint64_t)sms * 8 ? split_blocks : (uint64_t)sms * 8), 256, 0, s>>>(
      njobs, G, whist, big, ctr + kCtrWinBig, small, ctr + kCtrWinSmall,
      stats && ws->timing ? ws->d_stats + kStatBitmapIds : nullptr);
  if (wbits >= 18) launch_win_sort_t<18>(max_pairs, sms, big, ctr + kCtrWinBig, G, wbits, whist, wbase, src, out, err, s);
  else if (wbits == 17) launch_win_sort_t<17>(max_pairs, sms, big, ctr + kCtrWinBig, G, wbits, whist, wbase, src, out, err, s);
  else launch_win_sort_t<16>(max_pairs, sms, big, ctr + kCtrWinBig, G, wbits, whist, wbase, src, out, err, s);
  if (stats) mark(ws, kEvSortBitmap, s);
  const uint64_t warp_blocks = (max_pairs + kTinyWarps - 1) / kTinyWarps;
  k_win_sort_warp<<<(uint32_t)(warp_blocks < (uint64_t)sms * 4 ? warp_blocks : (uint64_t)sms * 4), kTinyWarps * 32,
                    sizeof(TinySmem), s>>>(small, ctr + kCtrWinSmall, G, wbits, whist, wbase, src, out);
}

static qcp_status set_sort_attrs(const qcp_index* ix, size_t scatter_max) {
  static thread_local int attrs_device = -1;  // attributes are per device
  if (attrs_device != ix->device) {
    QCP_CUDA(cudaFuncSetAttribute(k_sort_small, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  (int)sizeof(BucketSmem)));
    QCP_CUDA(cudaFuncSetAttribute(k_sort_tiny, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  (int)sizeof(TinySmem)));
    QCP_CUDA(cudaFuncSetAttribute(k_win_sort_warp, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  (int)sizeof(TinySmem)));
    QCP_CUDA(cudaFuncSetAttribute(k_win_sort<16>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  (int)sizeof(RankSmem<16>)));
    QCP_CUDA(cudaFuncSetAttribute(k_win_sort<17>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  (int)sizeof(RankSmem<17>)));
    QCP_CUDA(cudaFuncSetAttribute(k_win_sort<18>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  (int)sizeof(RankSmem<18>)));
    QCP_CUDA(cudaFuncSetAttribute(k_win_scatter, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  (int)scatter_max));
    attrs_device = ix->device;
  }
  return QCP_OK;
}

qcp_status sort_small_slices(qcp_index* ix, Workspace* ws, uint32_t q, cudaStream_t s,
                             const SortJob** big_out, uint32_t* nbig_out) {
  *big_out = nullptr;
  *nbig_out = 0;
  ws->sort_small_jobs = ws->sort_msd_jobs = 0;
  if (q == 0) return QCP_OK;
  const uint32_t idbits = id_bits(ix->n);
  const uint32_t sms = (uint32_t)num_sms();
  const size_t scatter_max = (size_t)(1u << (31 - kWinBits)) * 16 + kTile * 4;
  QCP_TRY(set_sort_attrs(ix, scatter_max));
  QCP_TRY(ws_reserve_sort(ix, ws, (size_t)q + 256, 0));
  uint32_t* ctr = ws->ctr;
  QCP_CUDA(cudaMemsetAsync(ctr + kCtrJobs0, 0, sizeof(uint32_t) * 3, s));  // jobs0, jobs1, small
  Job* small = reinterpret_cast<Job*>(ws->jobs[0]);
  Job* big = reinterpret_cast<Job*>(ws->jobs[1]);
  k_classify<<<(q + 255) / 256, 256, 0, s>>>((const unsigned long long*)ws->offsets, q, small,
                                             ctr + kCtrJobs0, ctr + kCtrSmall, ws->jobs_cap, big, ctr + kCtrJobs1,
                                             ws->timing ? ws->d_stats + kStatWindowIds : nullptr);
  note_launch();
  QCP_CUDA(cudaMemcpyAsync(ws->h_ctr, ctr, sizeof(uint32_t) * kCtrCount, cudaMemcpyDeviceToHost, s));
  QCP_CUDA(cudaStreamSynchronize(s));
  const uint32_t ntiny = ws->h_ctr[kCtrJobs0];
  const uint32_t nsmall = ws->h_ctr[kCtrSmall];
  const uint32_t nbig = ws->h_ctr[kCtrJobs1];
  ws->sort_small_jobs = ntiny + nsmall;
  ws->sort_msd_jobs = nbig;
  if (ntiny) {
    k_sort_tiny<<<min((ntiny + kTinyWarps - 1) / kTinyWarps, sms * 4), kTinyWarps * 32, sizeof(TinySmem), s>>>(
        small, ctr + kCtrJobs0, ws->out_ids, idbits);
    note_launch();
    QCP_TRY(check_launch("k_sort_tiny"));
  }
  if (nsmall) {
    k_sort_small<<<min(nsmall, sms * 3), kSmallThreads, sizeof(BucketSmem), s>>>(small + ws->jobs_cap,
                                                                                  ctr + kCtrSmall, ws->out_ids,
                                                                                  idbits);
    note_launch();
    QCP_TRY(check_launch("k_sort_small"));
  }
  *big_out = big;
  *nbig_out = nbig;
  return QCP_OK;
}

qcp_status segmented_sort(qcp_index* ix, Workspace* ws, uint32_t q, cudaStream_t s) {
  ws->sort_part_marked = false;
  const Job* bigc = nullptr;
  uint32_t nbig = 0;
  QCP_TRY(sort_small_slices(ix, ws, q, s, &bigc, &nbig));
  mark(ws, kEvSortSmall, s);
  if (nbig == 0) return QCP_OK;
  Job* big = const_cast<Job*>(bigc);
  uint32_t* ctr = ws->ctr;
  const uint32_t idbits = id_bits(ix->n);
  // window bits of this call: at most kWinBits (the bitmap), at least what
  // keeps the window count <= 8192 (the scatter's shared counters)
  uint32_t wb = ws->win_bits ? ws->win_bits : kDefaultWinBits;
  if (wb > kWinBits) wb = kWinBits;
  if (idbits > 13 && wb < idbits - 13) wb = idbits - 13;
  const uint32_t wbits = idbits < wb ? idbits : wb;
  const uint32_t G = 1u << (idbits - wbits);
  const uint32_t sms = (uint32_t)num_sms();
  const uint32_t nsets = (G <= kPerWarpMaxG) ? kTileWarps : 1u;
  const size_t scatter_bytes = (size_t)G * (8 + 4 * nsets) + kTile * 4;

  // tables per (job, window): counts (u32), bases and cursors (u64); tiles
  // and tile offsets per job
  const size_t nw = (size_t)nbig * G;
  const size_t hist_bytes = (nw * 4 + 15) & ~(size_t)15;
  const size_t lists_off = (hist_bytes + nw * 16 + (size_t)nbig * 8 + 15) & ~(size_t)15;
  const size_t bytes = lists_off + nw * 8 + 64;
  void* tables = nullptr;
  QCP_TRY(ix->pool.get(bytes, &tables));
  uint32_t* whist = reinterpret_cast<uint32_t*>(tables);
  unsigned long long* wbase = reinterpret_cast<unsigned long long*>(reinterpret_cast<char*>(tables) + hist_bytes);
  unsigned long long* wcur = wbase + nw;
  uint32_t* tiles = reinterpret_cast<uint32_t*>(wcur + nw);
  uint32_t* tile_off = tiles + nbig;
  uint32_t* lists = reinterpret_cast<uint32_t*>(reinterpret_cast<char*>(tables) + lists_off);  // 2 * nw
  qcp_status st = QCP_OK;
  do {
    k_tiles_per_job<<<(nbig + 255) / 256, 256, 0, s>>>(big, ctr + kCtrJobs1, nbig, tiles);
    note_launch();
    st = exclusive_scan<uint32_t>(tiles, tile_off, nbig, ctr + kCtrWork2, ix->pool, s);
    if (st != QCP_OK) break;
    if (cudaMemcpyAsync(ws->h_ctr + kCtrWork2, ctr + kCtrWork2, sizeof(uint32_t), cudaMemcpyDeviceToHost, s) !=
            cudaSuccess ||
        cudaStreamSynchronize(s) != cudaSuccess) {
      st = cuda_status(cudaGetLastError(), "segmented sort tiles");
      break;
    }
    const uint32_t ntiles = ws->h_ctr[kCtrWork2];
    st = ws_reserve_sort(ix, ws, 0, ntiles);
    if (st != QCP_OK) break;
    uint32_t* map = ws->seg_hist;
    k_tile_map<<<min(nbig, sms * 8), 256, 0, s>>>(tiles, tile_off, ctr + kCtrJobs1, map);
    // per-(job, window) counts: from the write pass when it gathered them
    const bool have_counts = ws->hist_G == G && ws->hist_bits == wbits;
    if (!have_counts) {
      if (cudaMemsetAsync(whist, 0, sizeof(uint32_t) * nw, s) != cudaSuccess) {
        st = cuda_status(cudaGetLastError(), "memset");
        break;
      }
      k_win_hist<<<min(ntiles, sms * 8), kTileThreads, sizeof(uint32_t) * G, s>>>(
          big, map, tile_off, ctr + kCtrWork2, ws->out_ids, G, wbits, whist);
    }
    k_win_scan<<<min(nbig, sms * 16), kTileThreads, 0, s>>>(big, ctr + kCtrJobs1, G, whist,
                                                            have_counts ? ws->qwhist : nullptr, wbase, wcur);
    k_win_scatter<<<min(ntiles, sms * scatter_blocks_per_sm(scatter_bytes)), kTileThreads, scatter_bytes, s>>>(
        big, map, tile_off, ctr + kCtrWork2, ws->out_ids, ws->tmp_ids, G, wbits, wcur);
    mark(ws, kEvSortPart, s);
    ws->sort_part_marked = ws->timing;
    if (cudaMemsetAsync(ctr + kCtrWinBig, 0, 2 * sizeof(uint32_t), s) != cudaSuccess) {
      st = cuda_status(cudaGetLastError(), "memset");
      break;
    }
    launch_win_sort(ws, nw, sms, ctr + kCtrJobs1, G, wbits, whist, wbase, lists, ctr, ws->tmp_ids, ws->out_ids,
                    ctr + kCtrTimeout, s, true);
    note_launch(7);
    st = check_launch("segmented sort windows");
    // the tables go back to the pool below: make sure the kernels are done
    if (st == QCP_OK && cudaStreamSynchronize(s) != cudaSuccess) st = cuda_status(cudaGetLastError(), "sort");
  } while (false);
  ix->pool.put(bytes, tables);
  return st;
}


// Window bits and window count of a call (ws->win_bits, bounded as in
// segmented_sort).
void sort_window_shape(const qcp_index* ix, const Workspace* ws, uint32_t* wbits, uint32_t* G);
static void window_shape(const qcp_index* ix, const Workspace* ws, uint32_t* wbits, uint32_t* G) {
  const uint32_t idbits = id_bits(ix->n);
  uint32_t wb = ws->win_bits ? ws->win_bits : kDefaultWinBits;
  if (wb > kWinBits) wb = kWinBits;
  if (idbits > 13 && wb < idbits - 13) wb = idbits - 13;
  *wbits = idbits < wb ? idbits : wb;
  *G = 1u << (idbits - *wbits);
}

void sort_window_shape(const qcp_index* ix, const Workspace* ws, uint32_t* wbits, uint32_t* G) {
  window_shape(ix, ws, wbits, G);
}

// Bytes of the per-(job, window) tables that segmented_sort_device needs for
// q queries with ws's window bits.
size_t sort_tables_bytes(const qcp_index* ix, const Workspace* ws, uint32_t q) {
  uint32_t wbits = 0, G = 0;
  window_shape(ix, ws, &wbits, &G);
  const size_t nw = (size_t)q * G;
  const size_t lists_off = ((((nw * 4 + 15) & ~(size_t)15) + nw * 16 + (size_t)q * 8) + 15) & ~(size_t)15;
  return lists_off + nw * 8 + 64;
}

// segmented_sort without host readbacks: job and tile counts stay on the
// device, every launch has a fixed grid and the kernels read the counts.
// Tables (sort_tables_bytes) and the tile map (at least total/kSortTile + q
// entries, ws->seg_hist) are the caller's.  Stream-capturable.
qcp_status segmented_sort_device(qcp_index* ix, Workspace* ws, uint32_t q, void* tables, cudaStream_t s) {
  if (q == 0) return QCP_OK;
  const uint32_t idbits = id_bits(ix->n);
  uint32_t wbits = 0, G = 0;
  window_shape(ix, ws, &wbits, &G);
  const uint32_t sms = (uint32_t)num_sms();
  const size_t scatter_max = (size_t)(1u << (31 - kWinBits)) * 16 + kTile * 4;
  QCP_TRY(set_sort_attrs(ix, scatter_max));
  const uint32_t nsets = (G <= kPerWarpMaxG) ? kTileWarps : 1u;
  const size_t scatter_bytes = (size_t)G * (8 + 4 * nsets) + kTile * 4;
  uint32_t* ctr = ws->ctr;
  Job* small = reinterpret_cast<Job*>(ws->jobs[0]);
  Job* big = reinterpret_cast<Job*>(ws->jobs[1]);
  const size_t nw = (size_t)q * G;
  const size_t hist_bytes = (nw * 4 + 15) & ~(size_t)15;
  uint32_t* whist = reinterpret_cast<uint32_t*>(tables);
  unsigned long long* wbase = reinterpret_cast<unsigned long long*>(reinterpret_cast<char*>(tables) + hist_bytes);
  unsigned long long* wcur = wbase + nw;
  uint32_t* tiles = reinterpret_cast<uint32_t*>(wcur + nw);
  uint32_t* tile_off = tiles + q;
  const size_t lists_off = (hist_bytes + nw * 16 + (size_t)q * 8 + 15) & ~(size_t)15;
  uint32_t* lists = reinterpret_cast<uint32_t*>(reinterpret_cast<char*>(tables) + lists_off);  // 2 * nw
  QCP_CUDA(cudaMemsetAsync(ctr + kCtrJobs0, 0, sizeof(uint32_t) * 3, s));  // jobs0, jobs1, small
  k_classify<<<(q + 255) / 256, 256, 0, s>>>((const unsigned long long*)ws->offsets, q, small, ctr + kCtrJobs0,
                                             ctr + kCtrSmall, ws->jobs_cap,
                                             big, ctr + kCtrJobs1, nullptr);
  k_sort_tiny<<<sms * 4, kTinyWarps * 32, sizeof(TinySmem), s>>>(small, ctr + kCtrJobs0, ws->out_ids, idbits);
  k_sort_small<<<sms * 3, kSmallThreads, sizeof(BucketSmem), s>>>(small + ws->jobs_cap, ctr + kCtrSmall,
                                                                  ws->out_ids, idbits);
  note_launch();
  k_tiles_per_job<<<(q + 255) / 256, 256, 0, s>>>(big, ctr + kCtrJobs1, q, tiles);
  note_launch(3);
  QCP_TRY(exclusive_scan<uint32_t>(tiles, tile_off, q, ctr + kCtrWork2, ix->pool, s, ws->scan_tmp,
                                   ws->scan_tmp_cap));
  k_tile_map<<<sms * 8, 256, 0, s>>>(tiles, tile_off, ctr + kCtrJobs1, ws->seg_hist);
  const bool have_counts = ws->hist_G == G && ws->hist_bits == wbits;
  if (!have_counts) {
    QCP_CUDA(cudaMemsetAsync(whist, 0, sizeof(uint32_t) * nw, s));
    k_win_hist<<<sms * 8, kTileThreads, sizeof(uint32_t) * G, s>>>(big, ws->seg_hist, tile_off, ctr + kCtrWork2,
                                                                   ws->out_ids, G, wbits, whist);
  }
  k_win_scan<<<sms * 16, kTileThreads, 0, s>>>(big, ctr + kCtrJobs1, G, whist, have_counts ? ws->qwhist : nullptr,
                                               wbase, wcur);
  k_win_scatter<<<sms * scatter_blocks_per_sm(scatter_bytes), kTileThreads, scatter_bytes, s>>>(
      big, ws->seg_hist, tile_off, ctr + kCtrWork2,
                                                             ws->out_ids, ws->tmp_ids, G, wbits, wcur);
  QCP_CUDA(cudaMemsetAsync(ctr + kCtrWinBig, 0, 2 * sizeof(uint32_t), s));
  launch_win_sort(ws, nw, sms, ctr + kCtrJobs1, G, wbits, whist, wbase, lists, ctr, ws->tmp_ids, ws->out_ids,
                  ctr + kCtrTimeout, s, false);
  note_launch(7);
  return check_launch("segmented sort (device counts)");
}

}  // namespace qcp
