// Range-search traversal kernels.
//
// Batched pipeline (QCP_ALGO_BATCHED), for the whole query batch at once:
//   1. k_expand, once per level above the leaves' parents: every
//      (query, node) item of level l becomes the (query, child) items of the
//      children whose MBR overlaps the query (warp per item, ballot
//      compaction, one atomic per warp).
//   2. k_leafscan<COUNT>: every (query, level-1 node) item is fetched
//      dynamically by a warp from a device work counter; the warp tests the
//      node's leaf MBRs, counts leaves whose MBR lies inside the query box
//      without touching their objects, and tests the objects of the other
//      overlapping leaves with 128-bit coalesced loads.
//   3. exclusive scan of the per-query counts -> CSR offsets.
//   4. k_leafscan<WRITE>: the same items again; each warp reserves its
//      item's slice of the query's output with one atomic and writes ids
//      (whole id runs for covered leaves, ballot-compacted ids otherwise).
//   5. per-query sort of the ids (qcp_segsort.cu).
//
// Plain traversal (QCP_ALGO_PLAIN): k_mprs, one query per CUDA block,
// restart scanning + parent check as the reference's
// global_RestartScanning_and_ParentCheck (src/tree/mphr.cpp:303-438) does,
// over the implicit node layout, run twice (count, then write).
//
// The hit predicate everywhere is the reference's closed-interval test
// (src/node/node_soa.cpp:94-113).
#include <algorithm>
#include <cfloat>
#include <thread>

#include "qcp_internal.cuh"
#include "qcp_tree.cuh"

namespace qcp {

namespace {

// ---------------------------------------------------------------------------
// Batched pipeline kernels
// ---------------------------------------------------------------------------
__global__ void k_init_items(uint2* items, uint32_t q, uint32_t node, uint32_t* count) {
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < q; i += gridDim.x * blockDim.x)
    items[i] = make_uint2(i, node);
  if (blockIdx.x == 0 && threadIdx.x == 0) *count = q;
}

// LPI lanes per (query, node) item (32, 16 or 8: 1, 2 or 4 items per warp
// at once); each group tests its item's children LPI at a time, compacts the
// overlapping ones with the group's part of one warp ballot and reserves
// their slots with one atomic per group and round.
template <int D, int LPI>
__global__ void __launch_bounds__(256) k_expand(const float* __restrict__ boxes,
                                                const uint2* __restrict__ in,
                                                const uint32_t* __restrict__ in_count,
                                                uint2* __restrict__ out, uint32_t* out_count,
                                                uint64_t out_cap, const float* __restrict__ child_mbr,
                                                uint64_t nchild, uint64_t child_pad, uint32_t fanout,
                                                uint32_t* overflow, uint32_t* need) {
  constexpr uint32_t kGroups = 32 / LPI;
  constexpr uint32_t kGroupMask = LPI == 32 ? 0xffffffffu : ((1u << LPI) - 1u);
  const uint32_t lane = threadIdx.x & 31;
  const uint32_t grp = lane / LPI, gl = lane % LPI;
  // the counter keeps counting past the capacity when a level overflowed
  const uint32_t nin = (uint32_t)min((uint64_t)*in_count, out_cap);
  const uint32_t warps = (gridDim.x * blockDim.x) >> 5;
  const uint32_t rounds = (fanout + LPI - 1) / LPI;  // warp-uniform
  for (uint32_t i0 = ((blockIdx.x * blockDim.x + threadIdx.x) >> 5) * kGroups; i0 < nin; i0 += warps * kGroups) {
    const uint32_t i = i0 + grp;
    const bool have = i < nin;
    uint2 it = make_uint2(0, 0);
    Box<D> b;
    uint64_t c0 = 0, c1 = 0;
    if (have) {
      it = in[i];
      b = load_box<D>(boxes, it.x);
      c0 = (uint64_t)it.y * fanout;
      c1 = (c0 + fanout < nchild) ? c0 + fanout : nchild;
    }
    for (uint32_t r = 0; r < rounds; ++r) {
      const uint64_t c = c0 + (uint64_t)r * LPI + gl;
      bool ov = false, in_ = false;
      if (have && c < c1) test_node<D>(b, child_mbr, child_pad, c, ov, in_);
      const uint32_t wm = __ballot_sync(0xffffffffu, ov);
      if (!wm) continue;  // warp-uniform
      const uint32_t m = (wm >> (grp * LPI)) & kGroupMask;
      uint32_t base = 0;
      if (gl == 0 && m) base = atomicAdd(out_count, (uint32_t)__popc(m));
      base = __shfl_sync(0xffffffffu, base, grp * LPI);
      if (ov) {
        const uint64_t pos = (uint64_t)base + __popc(m & ((1u << gl) - 1u));
        if (pos < out_cap) {
          out[pos] = make_uint2(it.x, (uint32_t)c);
        } else {
          atomicOr(overflow, 1u);
        }
      }
      if (gl == 0 && m && (uint64_t)base + __popc(m) > out_cap) atomicMax(need, base + __popc(m));
    }
  }
}

enum { kCount = 0, kWrite = 1 };

// Shared memory of one warp's leaf prefetch ring: kRingHeader bytes of
// mbarriers (one per buffer) and the list of the current item's partially
// covered leaves (offsets in the item), then `nbuf` leaf buffers of NR runs
// of F floats (the leaf's coordinate runs; in the write pass its ids too).
constexpr uint32_t kRingHeader = 384;
constexpr uint32_t kRingMaxBuf = 4;

__host__ __device__ constexpr uint32_t leaf_runs(int D, bool rect, int mode) {
  return (rect ? 2u * D : (uint32_t)D) + (mode == kWrite ? 1u : 0u);
}
__host__ __device__ inline uint32_t ring_warp_bytes(uint32_t runs, uint32_t F, uint32_t nbuf) {
  return kRingHeader + nbuf * runs * F * 4u;
}

// Hit cache handed from the count pass to the write pass of one call.  The
// count pass records, per item and 32-leaf group, the overlap and covered
// masks of the group's leaves and where the hit bits of its partially
// covered leaves start; per partially covered leaf and 128-object chunk it
// records four words, bit l of word k = object 4l + k is a hit.  The write
// pass then copies ids without testing a leaf MBR or a coordinate again.
// grp == nullptr: no cache.  A group whose hit bits did not fit (mask words
// past mask_cap) is marked kNoMask and the write pass tests its leaves.
struct HitCache {
  uint32_t* grp;       // [item][kMaxGroups][kGrpWords]
  uint32_t* mask;      // hit bits
  uint32_t mask_cap;   // words
  uint32_t* cursor;    // words asked for so far (may pass mask_cap)
};

__device__ __forceinline__ uint32_t words_per_leaf(uint32_t F) { return ((F + 127u) / 128u) * 4u; }
constexpr uint32_t kMaskChunk = 1024;  // hit-cache words a warp takes at a time

// Warp per (query, level-1 node) item.  COUNT: item_hits[i] and qcount[q].
// WRITE: ids at out[offsets[q] + reserved slice].
// PF: the partially covered leaves of an item are fetched into the warp's
// shared-memory ring by bulk copies (cp.async.bulk on the TMA unit, nbuf
// leaves ahead, completion on one mbarrier per buffer) while the warp tests
// the leaf before; without PF every lane loads its float4s from global
// memory.  A bulk-copy wait that runs out sets err[0] and the warp stops.
template <int D, bool RECT, int MODE, bool PF, bool CACHE>
__global__ void __launch_bounds__(256) k_leafscan(TreeView t, const float* __restrict__ boxes,
                                                  const uint2* __restrict__ items,
                                                  const uint32_t* __restrict__ item_count,
                                                  uint32_t* work, uint32_t* __restrict__ item_hits,
                                                  unsigned long long* qcount,
                                                  const unsigned long long* __restrict__ offsets,
                                                  unsigned long long* qcursor,
                                                  int32_t* __restrict__ out, uint64_t item_cap,
                                                  unsigned long long* stats, uint32_t* qwhist, uint32_t hist_G,
                                                  uint32_t hist_bits, uint32_t nbuf, uint32_t* err,
                                                  HitCache hc) {
  // write pass of the sorted path: per-(query, window) id counts in per-warp
  // shared counters, flushed once per item
  __shared__ uint32_t wcount[8][MODE == kWrite ? kHistMaxG : 1];
  extern __shared__ __align__(128) unsigned char ring_raw[];
  constexpr uint32_t NC = RECT ? 2 * D : D;       // coordinate runs of a leaf
  constexpr uint32_t NR = leaf_runs(D, RECT, MODE);
  const uint32_t lane = threadIdx.x & 31;
  const uint32_t wib = (threadIdx.x >> 5) & 7;
  uint32_t* wc = wcount[wib];
  const bool hist = MODE == kWrite && qwhist != nullptr;
  if (hist) {
    for (uint32_t w = lane; w < hist_G; w += 32) wc[w] = 0;
    __syncwarp();
  }
  const uint32_t F = t.fanout;
  unsigned char* ring = ring_raw + (size_t)wib * (PF ? ring_warp_bytes(NR, F, nbuf) : 0u);
  uint64_t* bars = reinterpret_cast<uint64_t*>(ring);
  uint8_t* plist = ring + 64;
  float* bufs = reinterpret_cast<float*>(ring + kRingHeader);
  const uint32_t buf_floats = NR * F;
  uint32_t phase = 0;     // bit b: parity of buffer b's next completion
  uint32_t pending = 0;   // bit b: a copy into buffer b has not been waited for
  bool dead = false;      // a bulk-copy wait ran out
  if (PF) {
    if (lane == 0) {
      for (uint32_t b = 0; b < nbuf; ++b) mbar_init(&bars[b], 1);
      mbar_fence_init();
    }
    __syncwarp();
  }
  // hit-bit room in per-warp chunks of the global cursor (one atomic per
  // chunk, not per group); kNoMask once the cache's capacity is used up
  // (the warp's chunk is kept in shared memory, not in registers: the count
  // pass is latency-bound and its occupancy is set by its registers)
  __shared__ uint32_t chunk[8][2];  // per warp: next word, end (end = kNoMask: no room left)
  if (CACHE) {
    if (lane == 0) chunk[wib][0] = chunk[wib][1] = 0;
    __syncwarp();
  }
  auto mask_alloc = [&](uint32_t want) -> uint32_t {
    uint32_t r = 0;
    if (lane == 0) {
      uint32_t pos = chunk[wib][0], end = chunk[wib][1];
      if (end == kNoMask) {
        r = kNoMask;
      } else {
        if (pos + want > end) {
          const uint32_t grab = want > kMaskChunk ? want : kMaskChunk;
          pos = atomicAdd(hc.cursor, grab);
          end = ((uint64_t)pos + grab > hc.mask_cap) ? kNoMask : pos + grab;
        }
        r = (end == kNoMask) ? kNoMask : pos;
        chunk[wib][0] = pos + want;
        chunk[wib][1] = end;
      }
    }
    return __shfl_sync(0xffffffffu, r, 0);
  };
  const uint32_t nitems = (uint32_t)min((uint64_t)*item_count, item_cap);
  const float* lmbr = t.mbr[0];
  const uint64_t lpad = t.pad[0];
  const uint64_t nleaves = t.nodes[0];
  for (;;) {
    uint32_t i = 0;
    if (lane == 0) i = atomicAdd(work, 1u);
    i = __shfl_sync(0xffffffffu, i, 0);
    if (i >= nitems) break;
    const uint2 it = items[i];
    const Box<D> b = load_box<D>(boxes, it.x);
    uint64_t wpos = 0;
    if (MODE == kWrite) {
      const uint32_t mine = item_hits[i];
      if (mine == 0) continue;
      if (lane == 0) wpos = offsets[it.x] + atomicAdd(qcursor + it.x, (unsigned long long)mine);
      wpos = __shfl_sync(0xffffffffu, wpos, 0);
    }
    uint32_t hits = 0;  // per lane (count mode)
    uint32_t n_cov = 0, n_part = 0, o_cov = 0;  // per lane work counters (count mode)
    uint32_t npart = 0;  // PF: partially covered leaves listed for the ring
    const uint64_t l0 = (uint64_t)it.y * F;
    const uint64_t l1 = (l0 + F < nleaves) ? l0 + F : nleaves;
    const bool cache = CACHE && hc.grp != nullptr;
    const uint32_t wpl = words_per_leaf(F);
    uint32_t* grec = cache ? hc.grp + (size_t)i * (kMaxGroups * kGrpWords) : nullptr;
    uint32_t g_mov = 0, g_min = 0;  // ring path: lane g holds group g's masks
    for (uint64_t lb = l0; lb < l1; lb += 32) {
      const uint32_t gi = (uint32_t)((lb - l0) >> 5);
      const uint64_t leaf = lb + lane;
      bool ov = false, in_ = false;
      uint32_t mov, min_, moff = kNoMask;
      if (MODE == kWrite && cache) {
        // the count pass's masks of this group
        mov = grec[gi * kGrpWords + 0];
        min_ = grec[gi * kGrpWords + 1];
        moff = grec[gi * kGrpWords + 2];
      } else {
        if (leaf < l1) test_node<D>(b, lmbr, lpad, leaf, ov, in_);
        mov = __ballot_sync(0xffffffffu, ov);
        min_ = __ballot_sync(0xffffffffu, in_ && ov);
        if (MODE == kCount && cache) {
          if (PF) {
            // recorded after the loop, with room for the whole item
            if (lane == gi) {
              g_mov = mov;
              g_min = min_;
            }
          } else {
            // record the group with room for its partial leaves' hit bits
            const uint32_t np = __popc(mov & ~min_);
            if (np) moff = mask_alloc(np * wpl);
            if (lane == 0) {
              grec[gi * kGrpWords + 0] = mov;
              grec[gi * kGrpWords + 1] = min_;
              grec[gi * kGrpWords + 2] = moff;
            }
          }
        }
      }
      if (!mov) continue;
      // leaves whose MBR lies inside the query: every object is a hit
      if (MODE == kCount) {
        if (in_ && ov) {
          const uint64_t e0 = leaf * F;
          const uint64_t e1 = (e0 + F < t.n) ? e0 + F : t.n;
          hits += (uint32_t)(e1 - e0);
          o_cov += (uint32_t)(e1 - e0);
          ++n_cov;
        } else if (ov) {
          ++n_part;
        }
      } else {
        uint32_t m = min_;
        while (m) {
          // a run of consecutive covered leaves is one contiguous id range
          const int s = __ffs(m) - 1;
          const uint32_t shifted = ~(m >> s);
          const int len = shifted ? (__ffs(shifted) - 1) : (32 - s);
          m &= ~((len >= 32 ? 0xffffffffu : ((1u << len) - 1u)) << s);
          const uint64_t e0 = (lb + s) * F;
          uint64_t e1 = (lb + s + len) * F;
          if (e1 > t.n) e1 = t.n;
          const int32_t* src = t.ids + e0;
          const uint64_t cnt = e1 - e0;
          // eight loads in flight per lane before their stores
          uint64_t j = lane;
          for (; j + 224 < cnt; j += 256) {
            int32_t v[8];
#pragma unroll
            for (int k = 0; k < 8; ++k) v[k] = __ldg(src + j + 32 * k);
#pragma unroll
            for (int k = 0; k < 8; ++k) out[wpos + j + 32 * k] = v[k];
            if (hist) {
#pragma unroll
              for (int k = 0; k < 8; ++k) atomicAdd(wc + ((uint32_t)v[k] >> hist_bits), 1u);
            }
          }
          for (; j + 96 < cnt; j += 128) {
            const int32_t a = __ldg(src + j), b = __ldg(src + j + 32);
            const int32_t c = __ldg(src + j + 64), d = __ldg(src + j + 96);
            out[wpos + j] = a;
            out[wpos + j + 32] = b;
            out[wpos + j + 64] = c;
            out[wpos + j + 96] = d;
            if (hist) {
              atomicAdd(wc + ((uint32_t)a >> hist_bits), 1u);
              atomicAdd(wc + ((uint32_t)b >> hist_bits), 1u);
              atomicAdd(wc + ((uint32_t)c >> hist_bits), 1u);
              atomicAdd(wc + ((uint32_t)d >> hist_bits), 1u);
            }
          }
          for (; j < cnt; j += 32) {
            const int32_t a = __ldg(src + j);
            out[wpos + j] = a;
            if (hist) atomicAdd(wc + ((uint32_t)a >> hist_bits), 1u);
          }
          wpos += cnt;
        }
      }
      uint32_t mp = mov & ~min_;
      const bool replay = MODE == kWrite && moff != kNoMask;  // hit bits cached by the count pass
      if constexpr (PF) {
        if (!replay) {
          // listed for the prefetch ring below
          if ((mp >> lane) & 1u) plist[npart + __popc(mp & lane_lt_mask())] = (uint8_t)(lb - l0 + lane);
          npart += __popc(mp);
          mp = 0;
        }
      }
      // partially covered leaves: test every object, or replay its hit bits
      uint32_t jl = 0;  // index of the leaf among the group's partial leaves
      while (mp) {
        const int s = __ffs(mp) - 1;
        mp &= mp - 1;
        const uint64_t e0 = (lb + s) * F;
        const uint32_t* mw = (moff != kNoMask) ? hc.mask + moff + jl * wpl : nullptr;
        ++jl;
        for (uint32_t g0 = 0; g0 < F; g0 += 128) {  // warp-uniform trip count
          const uint32_t g = g0 + lane * 4;
          const uint64_t p = e0 + g;
          uint32_t hm;
          if (replay) {
            const uint4 w = *reinterpret_cast<const uint4*>(mw + (g0 >> 5));
            hm = ((w.x >> lane) & 1u) | (((w.y >> lane) & 1u) << 1) | (((w.z >> lane) & 1u) << 2) |
                 (((w.w >> lane) & 1u) << 3);
          } else {
            hm = (g < F) ? test4<D, RECT>(b, t.coords, t.npad, p, t.n) : 0u;
          }
          if (MODE == kCount) {
            hits += __popc(hm);
            if (mw) {
              const uint32_t b0 = __ballot_sync(0xffffffffu, hm & 1u), b1 = __ballot_sync(0xffffffffu, hm & 2u);
              const uint32_t b2 = __ballot_sync(0xffffffffu, hm & 4u), b3 = __ballot_sync(0xffffffffu, hm & 8u);
              if (lane == 0) *reinterpret_cast<uint4*>(const_cast<uint32_t*>(mw) + (g0 >> 5)) = make_uint4(b0, b1, b2, b3);
            }
          } else {
            uint32_t tot;
            const uint32_t ex = warp_excl_sum(__popc(hm), &tot);
            if (hm) {
              const int4 idv = __ldg(reinterpret_cast<const int4*>(t.ids + p));
              uint64_t o = wpos + ex;
              if (hm & 1u) out[o++] = idv.x;
              if (hm & 2u) out[o++] = idv.y;
              if (hm & 4u) out[o++] = idv.z;
              if (hm & 8u) out[o++] = idv.w;
              if (hist) {
                if (hm & 1u) atomicAdd(wc + ((uint32_t)idv.x >> hist_bits), 1u);
                if (hm & 2u) atomicAdd(wc + ((uint32_t)idv.y >> hist_bits), 1u);
                if (hm & 4u) atomicAdd(wc + ((uint32_t)idv.z >> hist_bits), 1u);
                if (hm & 8u) atomicAdd(wc + ((uint32_t)idv.w >> hist_bits), 1u);
              }
            }
            wpos += tot;
          }
        }
      }
    }
    // ring path of the count pass with the cache: room for the hit bits of
    // the item's listed leaves (list order = group order); lane g records
    // group g
    uint32_t ring_moff = kNoMask;
    if (PF && MODE == kCount && cache) {
      const uint32_t ngroups = (uint32_t)((l1 - l0 + 31) >> 5);
      const uint32_t np = lane < ngroups ? __popc(g_mov & ~g_min) : 0u;
      uint32_t tot;
      const uint32_t before = warp_excl_sum(np, &tot);
      if (tot) ring_moff = mask_alloc(tot * wpl);
      if (lane < ngroups) {
        grec[lane * kGrpWords + 0] = g_mov;
        grec[lane * kGrpWords + 1] = g_min;
        grec[lane * kGrpWords + 2] = (np && ring_moff != kNoMask) ? ring_moff + before * wpl : kNoMask;
      }
    }
    if (PF && npart) {
      // partially covered leaves through the ring: leaf k of the list goes
      // to buffer k % nbuf, nbuf leaves ahead of the one being tested
      __syncwarp();  // the list is complete
      const uint32_t run_bytes = F * 4u;
      // one lane arms the buffer's barrier and issues the leaf's NR copies;
      // the warp's reads of the buffer's previous leaf are done (they fed
      // the tests before this point, and the syncwarp orders every lane's)
      auto issue = [&](uint32_t k, uint32_t bb) {
        __syncwarp();
        if (lane == 0) {
          const uint64_t leaf = l0 + plist[k];
          float* dst = bufs + (size_t)bb * buf_floats;
          mbar_arrive_expect_tx(&bars[bb], NR * run_bytes);
#pragma unroll
          for (uint32_t r = 0; r < NC; ++r)
            bulk_copy_g2s(dst + r * F, t.coords + (uint64_t)r * t.npad + leaf * F, run_bytes, &bars[bb]);
          if (NR > NC) bulk_copy_g2s(dst + NC * F, t.ids + leaf * F, run_bytes, &bars[bb]);
        }
        pending |= 1u << bb;
      };
      const uint32_t pre = npart < nbuf ? npart : nbuf;
      for (uint32_t k = 0; k < pre; ++k) issue(k, k);
      uint32_t bb = 0;
      for (uint32_t k = 0; k < npart; ++k) {
        const bool ok = __all_sync(0xffffffffu, mbar_wait_bounded(&bars[bb], (phase >> bb) & 1u));
        if (!ok) {
          dead = true;
          break;
        }
        phase ^= 1u << bb;
        pending &= ~(1u << bb);
        const float* sb = bufs + (size_t)bb * buf_floats;
        const uint64_t e0 = (l0 + plist[k]) * F;
        const uint32_t valid = (t.n > e0) ? (uint32_t)min((uint64_t)F, t.n - e0) : 0u;
        for (uint32_t g0 = 0; g0 < F; g0 += 128) {  // warp-uniform trip count
          const uint32_t g = g0 + lane * 4;
          const uint32_t hm = (g < F) ? test4_staged<D, RECT>(b, sb, F, g, valid) : 0u;
          if (MODE == kCount) {
            hits += __popc(hm);
            if (ring_moff != kNoMask) {
              const uint32_t b0 = __ballot_sync(0xffffffffu, hm & 1u), b1 = __ballot_sync(0xffffffffu, hm & 2u);
              const uint32_t b2 = __ballot_sync(0xffffffffu, hm & 4u), b3 = __ballot_sync(0xffffffffu, hm & 8u);
              if (lane == 0)
                *reinterpret_cast<uint4*>(hc.mask + ring_moff + k * wpl + (g0 >> 5)) = make_uint4(b0, b1, b2, b3);
            }
          } else {
            uint32_t tot;
            const uint32_t ex = warp_excl_sum(__popc(hm), &tot);
            if (hm) {
              const int4 idv = *reinterpret_cast<const int4*>(sb + NC * F + g);
              uint64_t o = wpos + ex;
              if (hm & 1u) out[o++] = idv.x;
              if (hm & 2u) out[o++] = idv.y;
              if (hm & 4u) out[o++] = idv.z;
              if (hm & 8u) out[o++] = idv.w;
              if (hist) {
                if (hm & 1u) atomicAdd(wc + ((uint32_t)idv.x >> hist_bits), 1u);
                if (hm & 2u) atomicAdd(wc + ((uint32_t)idv.y >> hist_bits), 1u);
                if (hm & 4u) atomicAdd(wc + ((uint32_t)idv.z >> hist_bits), 1u);
                if (hm & 8u) atomicAdd(wc + ((uint32_t)idv.w >> hist_bits), 1u);
              }
            }
            wpos += tot;
          }
        }
        if (k + nbuf < npart) issue(k + nbuf, bb);
        bb = (bb + 1 == nbuf) ? 0u : bb + 1;
      }
      if (dead) break;
    }
    if (hist) {
      __syncwarp();
      for (uint32_t w = lane; w < hist_G; w += 32) {
        const uint32_t c = wc[w];
        if (c) {
          atomicAdd(qwhist + (size_t)it.x * hist_G + w, c);
          wc[w] = 0;
        }
      }
      __syncwarp();
    }
    if (MODE == kCount) {
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) {
        hits += __shfl_xor_sync(0xffffffffu, hits, o);
        n_cov += __shfl_xor_sync(0xffffffffu, n_cov, o);
        n_part += __shfl_xor_sync(0xffffffffu, n_part, o);
        o_cov += __shfl_xor_sync(0xffffffffu, o_cov, o);
      }
      if (lane == 0) {
        item_hits[i] = hits;
        if (hits) atomicAdd(qcount + it.x, (unsigned long long)hits);
        if (n_cov) atomicAdd(stats + kStatCovered, (unsigned long long)n_cov);
        if (n_part) atomicAdd(stats + kStatPartial, (unsigned long long)n_part);
        if (o_cov) atomicAdd(stats + kStatObjCovered, (unsigned long long)o_cov);
      }
    }
  }
  if (PF && dead) {
    if (lane == 0) atomicOr(err, 1u);
    // copies still in flight land in this warp's ring: wait for them (again
    // bounded) before the CTA's shared memory goes away
    for (uint32_t bb = 0; bb < nbuf; ++bb)
      if ((pending >> bb) & 1u) mbar_wait_bounded(&bars[bb], (phase >> bb) & 1u);
  }
}

// ---------------------------------------------------------------------------
// Plain traversal: one query per block, blockDim.x == fanout threads.
// ---------------------------------------------------------------------------
__device__ __forceinline__ uint64_t span_of(uint32_t level, uint32_t F) {
  // objects covered by one node of `level` (level 0 = leaf)
  uint64_t s = F;
  for (uint32_t l = 0; l < level; ++l) s *= F;
  return s;
}

template <int D, bool RECT, int MODE>
__global__ void __launch_bounds__(256) k_mprs(TreeView t, const float* __restrict__ boxes, uint32_t nq,
                                              unsigned long long* __restrict__ counts,
                                              const unsigned long long* __restrict__ offsets,
                                              int32_t* __restrict__ out) {
  __shared__ uint32_t warp_min[8];
  __shared__ uint32_t warp_cnt[8];
  __shared__ uint32_t s_leftmost;
  const uint32_t tid = threadIdx.x, lane = tid & 31, w = tid >> 5;
  const uint32_t nwarps = blockDim.x >> 5;
  const uint32_t F = t.fanout;
  const uint32_t top = t.levels - 1;
  for (uint32_t q = blockIdx.x; q < nq; q += gridDim.x) {
    const Box<D> b = load_box<D>(boxes, q);
    uint64_t written = 0;
    uint64_t base = (MODE == kWrite) ? offsets[q] : 0;
    uint64_t visited = 0;  // every object before this position is settled
    uint32_t level = top;
    uint64_t node = 0;
    while (visited < t.n) {
      // internal phase: leftmost overlapping child not yet visited
      bool restart = false;
      while (level > 0) {
        const uint32_t cl = level - 1;
        const uint64_t c = node * F + tid;
        const uint64_t cspan = span_of(cl, F);
        bool cand = false;
        if (c < t.nodes[cl]) {
          uint64_t cend = (c + 1) * cspan;
          if (cend > t.n) cend = t.n;
          if (cend > visited) {
            bool ov, in_;
            test_node<D>(b, t.mbr[cl], t.pad[cl], c, ov, in_);
            cand = ov;
          }
        }
        const uint32_t m = __ballot_sync(0xffffffffu, cand);
        if (lane == 0) warp_min[w] = m ? (w * 32 + __ffs(m) - 1) : 0xffffffffu;
        __syncthreads();
        if (tid == 0) {
          uint32_t best = 0xffffffffu;
          for (uint32_t k = 0; k < nwarps; ++k) best = min(best, warp_min[k]);
          s_leftmost = best;
        }
        __syncthreads();
        const uint32_t leftmost = s_leftmost;
        __syncthreads();
        if (leftmost == 0xffffffffu) {
          // nothing left under this node: skip it and restart at the root
          uint64_t nend = (node + 1) * span_of(level, F);
          if (nend > t.n) nend = t.n;
          visited = nend;
          level = top;
          node = 0;
          restart = true;
          break;
        }
        node = node * F + leftmost;
        level = cl;
      }
      if (restart) continue;
      // leaf phase: scan leaves left to right while they hold hits
      for (;;) {
        const uint64_t e = node * F + tid;
        bool hit = false;
        if (e < t.n) {
          hit = true;
#pragma unroll
          for (int d = 0; d < D; ++d) {
            const float lo = t.coords[(uint64_t)d * t.npad + e];
            const float hi = RECT ? t.coords[(uint64_t)(D + d) * t.npad + e] : lo;
            hit &= overlaps1(b.lo[d], b.hi[d], lo, hi);
          }
        }
        const uint32_t hm = __ballot_sync(0xffffffffu, hit);
        if (lane == 0) warp_cnt[w] = __popc(hm);
        __syncthreads();
        uint32_t before = 0, total = 0;
        for (uint32_t k = 0; k < nwarps; ++k) {
          const uint32_t c = warp_cnt[k];
          if (k < w) before += c;
          total += c;
        }
        if (MODE == kWrite && hit) out[base + written + before + __popc(hm & lane_lt_mask())] = t.ids[e];
        written += total;
        __syncthreads();
        uint64_t lend = (node + 1) * F;
        if (lend > t.n) lend = t.n;
        visited = lend;
        if (lend >= t.n) break;
        if (total) {
          ++node;  // next leaf in key order
        } else {
          // back to the parent: its remaining children are checked next
          node /= F;
          level = 1;
          break;
        }
      }
      if (level == 0) break;  // reached the last leaf
      if (top == 0) break;
    }
    if (MODE == kCount && tid == 0) counts[q] = written;
  }
}

// Output capacity gate of the fixed-capacity pipeline: when the batch's
// total hits exceed the id buffer, flag it (bit 2 of *flag) and empty the
// write pass's item list; k_gate_zero then empties every slice, so the
// write and sort passes that follow do nothing.
__global__ void k_gate(const unsigned long long* __restrict__ offsets, uint32_t q, unsigned long long cap,
                       uint32_t* item_count, uint32_t* flag) {
  if (blockIdx.x == 0 && threadIdx.x == 0 && offsets[q] > cap) {
    atomicOr(flag, 2u);
    *item_count = 0;
  }
}

__global__ void k_gate_zero(unsigned long long* offsets, uint32_t q, const uint32_t* __restrict__ flag) {
  if (!(*flag & 2u)) return;
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i <= q; i += gridDim.x * blockDim.x) offsets[i] = 0;
}

template <int D>
void launch_expand(uint32_t grid, cudaStream_t s, const float* boxes, const uint2* in,
                   const uint32_t* in_count, uint2* out, uint32_t* out_count, uint64_t cap,
                   const float* child_mbr, uint64_t nchild, uint64_t child_pad, uint32_t fanout,
                   uint32_t* overflow, uint32_t* need, uint32_t lanes = 32) {
  if (lanes == 8)
    k_expand<D, 8><<<grid, 256, 0, s>>>(boxes, in, in_count, out, out_count, cap, child_mbr, nchild, child_pad,
                                        fanout, overflow, need);
  else if (lanes == 16)
    k_expand<D, 16><<<grid, 256, 0, s>>>(boxes, in, in_count, out, out_count, cap, child_mbr, nchild, child_pad,
                                         fanout, overflow, need);
  else
    k_expand<D, 32><<<grid, 256, 0, s>>>(boxes, in, in_count, out, out_count, cap, child_mbr, nchild, child_pad,
                                         fanout, overflow, need);
}

// Ring buffers per warp that fit the leaf prefetch of this launch: at most
// `want` (kRingMaxBuf), fewer when eight warps' rings would not leave room
// for two CTAs per SM; 0 = no ring (direct loads).
inline uint32_t ring_buffers(uint32_t runs, uint32_t F, uint32_t want) {
  if (want < 2) return 0;
  uint32_t nb = want > kRingMaxBuf ? kRingMaxBuf : want;
  while (nb >= 2 && 8u * ring_warp_bytes(runs, F, nb) > 100u * 1024u) --nb;
  return nb >= 2 ? nb : 0;
}

template <int D, bool RECT, int MODE>
void launch_leafscan_t(uint32_t grid, cudaStream_t s, const TreeView& t, const float* boxes, const uint2* items,
                       const uint32_t* item_count, uint32_t* work, uint32_t* item_hits, uint64_t* qcount,
                       const uint64_t* offsets, uint64_t* qcursor, int32_t* out, uint64_t item_cap,
                       unsigned long long* stats, uint32_t* qwhist, uint32_t hist_G, uint32_t hist_bits,
                       uint32_t ring, uint32_t* err, HitCache hc) {
  const uint32_t nb = ring_buffers(leaf_runs(D, RECT, MODE), t.fanout, ring);
  // the hit-cache code costs registers (occupancy of a latency-bound pass):
  // calls without a cache run an instantiation without it
  if (nb) {
    const size_t smem = 8u * (size_t)ring_warp_bytes(leaf_runs(D, RECT, MODE), t.fanout, nb);
    auto* kern = hc.grp ? k_leafscan<D, RECT, MODE, true, true> : k_leafscan<D, RECT, MODE, true, false>;
    if (smem > 48u * 1024u) cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    // no more CTAs than fit on the SMs at once (the static counters and 1 KB
    // per CTA of reserved shared memory included)
    const size_t per_cta = smem + sizeof(uint32_t) * 8 * (MODE == kWrite ? kHistMaxG : 1) + 1024;
    const uint32_t fit = (uint32_t)((228u * 1024u) / per_cta);
    const uint32_t sms = (uint32_t)num_sms();
    if (fit >= 1 && grid > sms * fit) grid = sms * fit;
    kern<<<grid, 256, smem, s>>>(t, boxes, items, item_count, work, item_hits, (unsigned long long*)qcount,
                                 (const unsigned long long*)offsets, (unsigned long long*)qcursor, out, item_cap,
                                 stats, qwhist, hist_G, hist_bits, nb, err, hc);
  } else {
    auto* kern = hc.grp ? k_leafscan<D, RECT, MODE, false, true> : k_leafscan<D, RECT, MODE, false, false>;
    kern<<<grid, 256, 0, s>>>(t, boxes, items, item_count, work, item_hits, (unsigned long long*)qcount,
                              (const unsigned long long*)offsets, (unsigned long long*)qcursor, out, item_cap, stats,
                              qwhist, hist_G, hist_bits, 0u, err, hc);
  }
}

template <int D, int MODE>
void launch_leafscan(bool rect, uint32_t grid, cudaStream_t s, const TreeView& t, const float* boxes,
                     const uint2* items, const uint32_t* item_count, uint32_t* work,
                     uint32_t* item_hits, uint64_t* qcount, const uint64_t* offsets,
                     uint64_t* qcursor, int32_t* out, uint64_t item_cap,
                     unsigned long long* stats, uint32_t* qwhist, uint32_t hist_G,
                     uint32_t hist_bits, uint32_t ring, uint32_t* err, HitCache hc = HitCache{}) {
  if (rect)
    launch_leafscan_t<D, true, MODE>(grid, s, t, boxes, items, item_count, work, item_hits, qcount, offsets, qcursor,
                                     out, item_cap, stats, qwhist, hist_G, hist_bits, ring, err, hc);
  else
    launch_leafscan_t<D, false, MODE>(grid, s, t, boxes, items, item_count, work, item_hits, qcount, offsets,
                                      qcursor, out, item_cap, stats, qwhist, hist_G, hist_bits, ring, err, hc);
}

template <int D, int MODE>
void launch_mprs(bool rect, uint32_t grid, uint32_t threads, cudaStream_t s, const TreeView& t,
                 const float* boxes, uint32_t nq, uint64_t* counts, const uint64_t* offsets,
                 int32_t* out) {
  if (rect)
    k_mprs<D, true, MODE><<<grid, threads, 0, s>>>(t, boxes, nq, (unsigned long long*)counts,
                                                   (const unsigned long long*)offsets, out);
  else
    k_mprs<D, false, MODE><<<grid, threads, 0, s>>>(t, boxes, nq, (unsigned long long*)counts,
                                                    (const unsigned long long*)offsets, out);
}

}  // namespace

// Grows the workspace buffers a batch of q queries needs before its items
// are known (items and output grow on demand below).
qcp_status ws_reserve_queries(qcp_index* ix, Workspace* ws, uint32_t q);
qcp_status ws_reserve_items(qcp_index* ix, Workspace* ws, size_t items);
qcp_status ws_reserve_out(qcp_index* ix, Workspace* ws, size_t ids);

qcp_status init_items(Workspace* ws, uint32_t q, cudaStream_t s) {
  k_init_items<<<(q + 255) / 256, 256, 0, s>>>(ws->items[0], q, 0, ws->ctr + kCtrFrontier0);
  note_launch();
  return QCP_OK;
}

qcp_status expand_level(qcp_index* ix, Workspace* ws, uint32_t l, int cur, cudaStream_t s) {
  const TreeView t = view_of(ix);
  const uint32_t grid = (uint32_t)num_sms() * ws->blocks_per_sm;
  const int nxt = cur ^ 1;
  uint32_t* ctr = ws->ctr;
  QCP_DISPATCH_D(ix->dims, launch_expand<DD>(grid, s, ws->boxes, ws->items[cur], ctr + kCtrFrontier0 + cur,
                                             ws->items[nxt], ctr + kCtrFrontier0 + nxt, ws->items_cap,
                                             t.mbr[l - 1], t.nodes[l - 1], t.pad[l - 1], t.fanout,
                                             ctr + kCtrOverflow, ctr + kCtrNeedItems, ws->lanes_per_item));
  note_launch();
  return check_launch("k_expand");
}

// The hit cache of this call (ws->use_hit_cache), or none.
static HitCache hit_cache_of(Workspace* ws) {
  if (!ws->use_hit_cache || !ws->item_grp || !ws->hmask) return HitCache{nullptr, nullptr, 0, nullptr};
  return HitCache{ws->item_grp, ws->hmask, (uint32_t)(ws->hmask_cap > 0xfffffff0u ? 0xfffffff0u : ws->hmask_cap),
                  ws->ctr + kCtrMaskWords};
}

qcp_status write_items(qcp_index* ix, Workspace* ws, int cur, cudaStream_t s) {
  const TreeView t = view_of(ix);
  const uint32_t grid = (uint32_t)num_sms() * ws->blocks_per_sm;
  uint32_t* ctr = ws->ctr;
  QCP_DISPATCH_D(ix->dims, launch_leafscan<DD, kWrite>(ix->is_rect != 0, grid, s, t, ws->boxes, ws->items[cur],
                                                       ctr + kCtrFrontier0 + cur, ctr + kCtrWork,
                                                       ws->item_hits, nullptr, ws->offsets, ws->qcursor,
                                                       ws->out_ids, ws->items_cap, ws->d_stats,
                                                       ws->hist_G ? ws->qwhist : nullptr, ws->hist_G,
                                                       ws->hist_bits, ws->leaf_ring, ctr + kCtrTimeout,
                                                       hit_cache_of(ws)));
  note_launch();
  return check_launch("k_leafscan<write>");
}

qcp_status run_batched(qcp_index* ix, Workspace* ws, uint32_t q, bool counts_only, bool sort,
                       cudaStream_t s) {
  const TreeView t = view_of(ix);
  const uint32_t D = ix->dims;
  const bool rect = ix->is_rect != 0;
  const uint32_t sms = (uint32_t)num_sms();
  const uint32_t grid = sms * ws->blocks_per_sm;  // 256-thread blocks
  uint32_t* ctr = ws->ctr;
  // start level: items at level `start` are (query, node) pairs
  const uint32_t start = (ix->levels >= 2) ? ix->levels - 1 : 1;
  ws->use_hit_cache = false;
  for (int attempt = 0; attempt < 8; ++attempt) {
    mark(ws, kEvStart, s);
    QCP_CUDA(cudaMemsetAsync(ctr, 0, sizeof(uint32_t) * kCtrCount, s));
    QCP_CUDA(cudaMemsetAsync(ws->d_stats, 0, sizeof(unsigned long long) * kStatCount, s));
    QCP_CUDA(cudaMemsetAsync(ws->qcount, 0, sizeof(uint64_t) * q, s));
    // the GPU's first level: the root's, or the hand-off level of a CPU + GPU
    // co-processing call whose host threads walked the levels above
    uint32_t gpu_start = start;
    if (ws->hybrid) {
      gpu_start = ws->handoff_level < 1 ? 1u : (ws->handoff_level > start ? start : ws->handoff_level);
    }
    if (gpu_start < start) {
      QCP_TRY(host_frontier(ix, ws, q, gpu_start, s));
    } else {
      QCP_TRY(init_items(ws, q, s));
    }
    QCP_CUDA(cudaMemcpyAsync(ws->d_stats + kStatLevel0 + gpu_start, ctr + kCtrFrontier0, sizeof(uint32_t),
                             cudaMemcpyDeviceToDevice, s));
    int cur = 0;
    for (uint32_t l = gpu_start; l > 1; --l) {
      const int nxt = cur ^ 1;
      QCP_CUDA(cudaMemsetAsync(ctr + kCtrFrontier0 + nxt, 0, sizeof(uint32_t), s));
      QCP_TRY(expand_level(ix, ws, l, cur, s));
      QCP_CUDA(cudaMemcpyAsync(ws->d_stats + kStatLevel0 + (l - 1), ctr + kCtrFrontier0 + nxt,
                               sizeof(uint32_t), cudaMemcpyDeviceToDevice, s));
      cur = nxt;
    }
    mark(ws, kEvExpand, s);
    // the level-1 items must fit the per-item hit array too
    QCP_TRY(ws_reserve_items(ix, ws, 0));
    // a call that writes ids keeps the count pass's hits for the write pass
    ws->use_hit_cache = !counts_only && ws->hit_cache_on;
    if (ws->use_hit_cache) QCP_TRY(ws_reserve_hitcache(ws, ws->items_cap, ws->hmask_cap ? 0 : (size_t)1 << 20));
    QCP_DISPATCH_D(D, launch_leafscan<DD, kCount>(rect, grid, s, t, ws->boxes, ws->items[cur],
                                                  ctr + kCtrFrontier0 + cur, ctr + kCtrWork,
                                                  ws->item_hits, ws->qcount, nullptr, nullptr, nullptr,
                                                  ws->items_cap, ws->d_stats, nullptr, 0, 0, ws->leaf_ring,
                                                  ctr + kCtrTimeout, hit_cache_of(ws)));
    note_launch();
    QCP_TRY(check_launch("k_leafscan<count>"));
    mark(ws, kEvCount, s);
    QCP_TRY(exclusive_scan_counts(ws->qcount, ws->offsets, q, ix->pool, s));
    mark(ws, kEvScan, s);
    // one readback: overflow flags, items needed, total hits
    QCP_CUDA(cudaMemcpyAsync(ws->h_ctr, ctr, sizeof(uint32_t) * kCtrCount, cudaMemcpyDeviceToHost, s));
    QCP_CUDA(cudaMemcpyAsync(ws->h_total, ws->offsets + q, sizeof(uint64_t), cudaMemcpyDeviceToHost, s));
    QCP_CUDA(cudaStreamSynchronize(s));
    if (ws->h_ctr[kCtrTimeout]) {
      set_error("a bounded wait for a leaf's bulk copy ran out in the count pass");
      return QCP_ERR_TIMEOUT;
    }
    if (ws->h_ctr[kCtrOverflow]) {
      size_t need = (size_t)ws->h_ctr[kCtrNeedItems];
      if (need < ws->items_cap * 2) need = ws->items_cap * 2;
      QCP_TRY(ws_reserve_items(ix, ws, need));
      continue;
    }
    if (counts_only) return QCP_OK;
    const uint64_t total = *ws->h_total;
    QCP_TRY(ws_reserve_out(ix, ws, (size_t)total));
    if (total) {
      QCP_CUDA(cudaMemsetAsync(ws->qcursor, 0, sizeof(uint64_t) * q, s));
      QCP_CUDA(cudaMemsetAsync(ctr + kCtrWork, 0, sizeof(uint32_t), s));
      ws->hist_G = 0;
      if (sort) {  // the write pass counts ids per (query, sort window)
        uint32_t wbits = 0, G = 0;
        sort_window_shape(ix, ws, &wbits, &G);
        if (G <= kHistMaxG) {
          QCP_TRY(ws_reserve_qwhist(ws, (size_t)q * G));
          QCP_CUDA(cudaMemsetAsync(ws->qwhist, 0, sizeof(uint32_t) * q * G, s));
          ws->hist_G = G;
          ws->hist_bits = wbits;
        }
      }
      QCP_TRY(write_items(ix, ws, cur, s));
      mark(ws, kEvWrite, s);
      if (sort) QCP_TRY(segmented_sort(ix, ws, q, s));
      mark(ws, kEvSort, s);
      // bounded waits of the write pass's leaf ring and the window sort's
      // bulk prefetch
      QCP_CUDA(cudaMemcpyAsync(ws->h_ctr + kCtrTimeout, ctr + kCtrTimeout, sizeof(uint32_t),
                               cudaMemcpyDeviceToHost, s));
      QCP_CUDA(cudaStreamSynchronize(s));
      if (ws->h_ctr[kCtrTimeout]) {
        set_error("a bounded wait for a bulk copy ran out in the write pass or the sort");
        return QCP_ERR_TIMEOUT;
      }
    }
    // hit bits that did not fit this call were tested again by the write
    // pass; the next call gets room for them (after this call's passes)
    if (ws->use_hit_cache && ws->h_ctr[kCtrMaskWords] > ws->hmask_cap) {
      QCP_CUDA(cudaStreamSynchronize(s));
      QCP_TRY(ws_reserve_hitcache(ws, 0, ws->h_ctr[kCtrMaskWords]));
    }
    ws->use_hit_cache = false;
    return QCP_OK;
  }
  set_error("query frontier did not fit after repeated growth");
  return QCP_ERR_OOM;
}

qcp_status run_plain(qcp_index* ix, Workspace* ws, uint32_t q, bool counts_only, bool sort,
                     cudaStream_t s) {
  const TreeView t = view_of(ix);
  const uint32_t D = ix->dims;
  const bool rect = ix->is_rect != 0;
  const uint32_t threads = ix->fanout;
  uint32_t grid = q ? q : 1;
  if (grid > (uint32_t)num_sms() * 64) grid = (uint32_t)num_sms() * 64;
  mark(ws, kEvStart, s);
  mark(ws, kEvExpand, s);
  QCP_DISPATCH_D(D, launch_mprs<DD, kCount>(rect, grid, threads, s, t, ws->boxes, q, ws->qcount,
                                            nullptr, nullptr));
  note_launch();
  QCP_TRY(check_launch("k_mprs<count>"));
  mark(ws, kEvCount, s);
  QCP_TRY(exclusive_scan_counts(ws->qcount, ws->offsets, q, ix->pool, s));
  mark(ws, kEvScan, s);
  QCP_CUDA(cudaMemcpyAsync(ws->h_total, ws->offsets + q, sizeof(uint64_t), cudaMemcpyDeviceToHost, s));
  QCP_CUDA(cudaStreamSynchronize(s));
  if (counts_only) return QCP_OK;
  const uint64_t total = *ws->h_total;
  QCP_TRY(ws_reserve_out(ix, ws, (size_t)total));
  if (total) {
    ws->hist_G = 0;  // the sort counts its windows itself
    QCP_DISPATCH_D(D, launch_mprs<DD, kWrite>(rect, grid, threads, s, t, ws->boxes, q, nullptr,
                                              ws->offsets, ws->out_ids));
    note_launch();
    QCP_TRY(check_launch("k_mprs<write>"));
    mark(ws, kEvWrite, s);
    if (sort) QCP_TRY(segmented_sort(ix, ws, q, s));
    mark(ws, kEvSort, s);
  }
  return QCP_OK;
}

// Batched per-query hit counts into caller-provided device buffers (boxes,
// counts) with scratch supplied by the caller as well: two frontier buffers
// of item_cap items, item_cap per-item counts, kCtrCount counters and
// kStatCount statistics words.  Nothing is allocated.  Returns
// QCP_ERR_OUTPUT_OVERFLOW when the batch's frontier exceeds item_cap.
qcp_status run_batched_counts_into(qcp_index* ix, const float* boxes, uint32_t q, uint64_t* counts,
                                   uint2* items0, uint2* items1, uint32_t* item_hits, size_t item_cap,
                                   uint32_t* ctr, unsigned long long* stats, cudaStream_t s) {
  const TreeView t = view_of(ix);
  const uint32_t D = ix->dims;
  const bool rect = ix->is_rect != 0;
  const uint32_t grid = (uint32_t)num_sms() * 8;
  uint2* items[2] = {items0, items1};
  const uint32_t start = (ix->levels >= 2) ? ix->levels - 1 : 1;
  QCP_CUDA(cudaMemsetAsync(ctr, 0, sizeof(uint32_t) * kCtrCount, s));
  QCP_CUDA(cudaMemsetAsync(stats, 0, sizeof(unsigned long long) * kStatCount, s));
  QCP_CUDA(cudaMemsetAsync(counts, 0, sizeof(uint64_t) * q, s));
  k_init_items<<<(q + 255) / 256, 256, 0, s>>>(items[0], q, 0, ctr + kCtrFrontier0);
  note_launch();
  int cur = 0;
  for (uint32_t l = start; l > 1; --l) {
    const int nxt = cur ^ 1;
    QCP_CUDA(cudaMemsetAsync(ctr + kCtrFrontier0 + nxt, 0, sizeof(uint32_t), s));
    QCP_DISPATCH_D(D, launch_expand<DD>(grid, s, boxes, items[cur], ctr + kCtrFrontier0 + cur, items[nxt],
                                        ctr + kCtrFrontier0 + nxt, item_cap, t.mbr[l - 1], t.nodes[l - 1],
                                        t.pad[l - 1], t.fanout, ctr + kCtrOverflow, ctr + kCtrNeedItems));
    note_launch();
    cur = nxt;
  }
  QCP_DISPATCH_D(D, launch_leafscan<DD, kCount>(rect, grid, s, t, boxes, items[cur], ctr + kCtrFrontier0 + cur,
                                                ctr + kCtrWork, item_hits, counts, nullptr, nullptr, nullptr,
                                                item_cap, stats, nullptr, 0, 0, 0, ctr + kCtrTimeout));
  note_launch();
  QCP_TRY(check_launch("batched counts"));
  uint32_t overflow = 0;  // pageable host word: no pinned buffer is allocated
  QCP_CUDA(cudaMemcpyAsync(&overflow, ctr + kCtrOverflow, sizeof(uint32_t), cudaMemcpyDeviceToHost, s));
  QCP_CUDA(cudaStreamSynchronize(s));
  if (overflow) {
    set_error("query frontier exceeds the fixed scratch of this entry point; split the batch");
    return QCP_ERR_OUTPUT_OVERFLOW;
  }
  return QCP_OK;
}


// The batched pipeline with fixed capacities and no host readback: the
// frontier overflow (bit 1) and the id-capacity overflow (bit 2) are left in
// ws->ctr[kCtrOverflow] for the caller to read after the stream has run; on
// either, the results are incomplete.  All buffers must be reserved before
// (ws_reserve_*, ws->out_cap >= ids_cap); sort tables as segmented_sort_device.
// Stream-capturable.
qcp_status run_batched_device(qcp_index* ix, Workspace* ws, uint32_t q, uint64_t ids_cap, bool sort,
                              void* sort_tables, cudaStream_t s) {
  const TreeView t = view_of(ix);
  const uint32_t D = ix->dims;
  const bool rect = ix->is_rect != 0;
  const uint32_t grid = (uint32_t)num_sms() * ws->blocks_per_sm;
  uint32_t* ctr = ws->ctr;
  const uint32_t start = (ix->levels >= 2) ? ix->levels - 1 : 1;
  ws->use_hit_cache = false;  // the captured pipeline tests every leaf in both passes
  QCP_CUDA(cudaMemsetAsync(ctr, 0, sizeof(uint32_t) * kCtrCount, s));
  QCP_CUDA(cudaMemsetAsync(ws->qcount, 0, sizeof(uint64_t) * q, s));
  QCP_TRY(init_items(ws, q, s));
  int cur = 0;
  for (uint32_t l = start; l > 1; --l) {
    QCP_CUDA(cudaMemsetAsync(ctr + kCtrFrontier0 + (cur ^ 1), 0, sizeof(uint32_t), s));
    QCP_TRY(expand_level(ix, ws, l, cur, s));
    cur ^= 1;
  }
  QCP_DISPATCH_D(D, launch_leafscan<DD, kCount>(rect, grid, s, t, ws->boxes, ws->items[cur],
                                                ctr + kCtrFrontier0 + cur, ctr + kCtrWork, ws->item_hits,
                                                ws->qcount, nullptr, nullptr, nullptr, ws->items_cap,
                                                ws->d_stats, nullptr, 0, 0, ws->leaf_ring, ctr + kCtrTimeout));
  note_launch();
  QCP_TRY(exclusive_scan_counts(ws->qcount, ws->offsets, q, ix->pool, s, ws->scan_tmp, ws->scan_tmp_cap));
  k_gate<<<1, 32, 0, s>>>((const unsigned long long*)ws->offsets, q, ids_cap, ctr + kCtrFrontier0 + cur,
                          ctr + kCtrOverflow);
  k_gate_zero<<<(q + 256) / 256, 256, 0, s>>>((unsigned long long*)ws->offsets, q, ctr + kCtrOverflow);
  note_launch(2);
  QCP_CUDA(cudaMemsetAsync(ws->qcursor, 0, sizeof(uint64_t) * q, s));
  QCP_CUDA(cudaMemsetAsync(ctr + kCtrWork, 0, sizeof(uint32_t), s));
  if (ws->hist_G) QCP_CUDA(cudaMemsetAsync(ws->qwhist, 0, sizeof(uint32_t) * q * ws->hist_G, s));
  QCP_TRY(write_items(ix, ws, cur, s));
  if (sort) QCP_TRY(segmented_sort_device(ix, ws, q, sort_tables, s));
  return check_launch("batched pipeline (device counts)");
}


// ---------------------------------------------------------------------------
// CPU + GPU co-processing: the host walks the internal levels.
//
// The reference's Hybrid::Search (src/tree/hybrid.cpp:451-760) gives every
// host thread a share of the queries; per query the thread walks the upper
// tree (Hybrid::TraverseInternalNodes, :801-960) to a run of leaf nodes and
// launches a GPU scan of that run, one launch per run.  Here the host threads
// walk every query of the batch down to the hand-off level at once and the
// GPU gets the whole frontier in one copy; expansion below the hand-off
// level, the leaf scan, the write and the sort stay on the GPU.  The host
// uses a copy of the internal levels' MBRs and the same closed-interval
// predicate as the kernels.
// ---------------------------------------------------------------------------
static qcp_status ensure_host_mbr(qcp_index* ix) {
  std::lock_guard<std::mutex> g(ix->host_mbr_mu);
  if (ix->host_mbr_ready) return QCP_OK;
  for (uint32_t l = 1; l < ix->levels; ++l) {
    const size_t n = 2 * (size_t)ix->dims * ix->level_pad[l];
    ix->host_mbr[l].resize(n);
    QCP_CUDA(cudaMemcpy(ix->host_mbr[l].data(), ix->mbr[l], sizeof(float) * n, cudaMemcpyDeviceToHost));
  }
  ix->host_mbr_ready = true;
  return QCP_OK;
}

qcp_status host_frontier(qcp_index* ix, Workspace* ws, uint32_t q, uint32_t level, cudaStream_t s) {
  QCP_TRY(ensure_host_mbr(ix));
  const uint32_t D = ix->dims, F = ix->fanout, top = ix->levels - 1;
  const float* boxes = ws->h_boxes;
  uint32_t T = ws->cpu_threads ? ws->cpu_threads : std::thread::hardware_concurrency();
  if (T == 0) T = 1;
  if (T > 64) T = 64;
  if (T > q) T = q ? q : 1;
  std::vector<std::vector<uint2>> part(T);
  auto walk = [&](uint32_t t) {
    const uint32_t q0 = (uint32_t)((uint64_t)q * t / T), q1 = (uint32_t)((uint64_t)q * (t + 1) / T);
    std::vector<std::pair<uint32_t, uint64_t>> stack;  // (level, node)
    auto& out = part[t];
    for (uint32_t qq = q0; qq < q1; ++qq) {
      const float* b = boxes + (size_t)qq * 2 * D;
      stack.clear();
      stack.emplace_back(top, 0);
      while (!stack.empty()) {
        const uint32_t l = stack.back().first;
        const uint64_t node = stack.back().second;
        stack.pop_back();
        const uint32_t cl = l - 1;
        const float* m = ix->host_mbr[cl].data();
        const uint64_t pad = ix->level_pad[cl];
        const uint64_t c0 = node * F;
        const uint64_t c1 = std::min<uint64_t>(c0 + F, ix->level_nodes[cl]);
        // children in reverse so that the stack pops them in order
        for (uint64_t c = c1; c-- > c0;) {
          bool ov = true;
          for (uint32_t d = 0; d < D && ov; ++d) ov = overlaps1(b[d], b[D + d], m[d * pad + c], m[(D + d) * pad + c]);
          if (!ov) continue;
          if (cl == level) out.push_back(make_uint2(qq, (uint32_t)c));
          else stack.emplace_back(cl, c);
        }
      }
    }
  };
  std::vector<std::thread> pool;
  for (uint32_t t = 1; t < T; ++t) pool.emplace_back(walk, t);
  walk(0);
  for (auto& th : pool) th.join();
  size_t n = 0;
  for (auto& p : part) n += p.size();
  ws->h_items.resize(n ? n : 1);
  size_t k = 0;
  for (auto& p : part) {
    std::copy(p.begin(), p.end(), ws->h_items.begin() + k);
    k += p.size();
  }
  if (n > 0xffffffffull) {
    set_error("co-processing frontier exceeds 2^32 items");
    return QCP_ERR_OOM;
  }
  QCP_TRY(ws_reserve_items(ix, ws, n));
  ws->h_nitems = (uint32_t)n;
  if (n) QCP_CUDA(cudaMemcpyAsync(ws->items[0], ws->h_items.data(), sizeof(uint2) * n, cudaMemcpyHostToDevice, s));
  QCP_CUDA(cudaMemcpyAsync(ws->ctr + kCtrFrontier0, &ws->h_nitems, sizeof(uint32_t), cudaMemcpyHostToDevice, s));
  // pageable sources: wait for the copies before the host vectors change
  QCP_CUDA(cudaStreamSynchronize(s));
  return QCP_OK;
}

}  // namespace qcp
