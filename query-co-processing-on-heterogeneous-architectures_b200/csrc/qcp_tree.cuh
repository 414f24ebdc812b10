// Device-side view of the implicit R-tree and the per-object tests of the
// traversal kernels.
#pragma once

#include "qcp_internal.cuh"

namespace qcp {

struct TreeView {
  const float* coords;
  const int32_t* ids;
  uint64_t n, npad;
  uint32_t fanout, levels;
  const float* mbr[kMaxLevels];
  uint64_t nodes[kMaxLevels];
  uint64_t pad[kMaxLevels];
};

inline TreeView view_of(const qcp_index* ix) {
  TreeView v;
  v.coords = ix->coords;
  v.ids = ix->ids;
  v.n = ix->n;
  v.npad = ix->npad;
  v.fanout = ix->fanout;
  v.levels = ix->levels;
  for (int l = 0; l < kMaxLevels; ++l) {
    v.mbr[l] = ix->mbr[l];
    v.nodes[l] = ix->level_nodes[l];
    v.pad[l] = ix->level_pad[l];
  }
  return v;
}

template <int D>
struct Box {
  float lo[D], hi[D];
};

template <int D>
__device__ __forceinline__ Box<D> load_box(const float* boxes, uint32_t q) {
  Box<D> b;
  const float* p = boxes + (uint64_t)q * 2 * D;
#pragma unroll
  for (int d = 0; d < D; ++d) {
    b.lo[d] = __ldg(p + d);
    b.hi[d] = __ldg(p + D + d);
  }
  return b;
}

// MBR overlap / containment of node c of a level.
template <int D>
__device__ __forceinline__ void test_node(const Box<D>& b, const float* mbr, uint64_t pad, uint64_t c,
                                          bool& ov, bool& in) {
  ov = true;
  in = true;
#pragma unroll
  for (int d = 0; d < D; ++d) {
    const float lo = __ldg(mbr + (uint64_t)d * pad + c);
    const float hi = __ldg(mbr + (uint64_t)(D + d) * pad + c);
    ov &= overlaps1(b.lo[d], b.hi[d], lo, hi);
    in &= inside1(b.lo[d], b.hi[d], lo, hi);
  }
}

// Hit mask of 4 consecutive objects starting at position p (p % 4 == 0).
template <int D, bool RECT>
__device__ __forceinline__ uint32_t test4(const Box<D>& b, const float* coords, uint64_t npad, uint64_t p,
                                          uint64_t n) {
  uint32_t m = 0xfu;
#pragma unroll
  for (int d = 0; d < D; ++d) {
    const float4 lo = __ldg(reinterpret_cast<const float4*>(coords + (uint64_t)d * npad + p));
    float4 hi = lo;
    if (RECT) hi = __ldg(reinterpret_cast<const float4*>(coords + (uint64_t)(D + d) * npad + p));
    m &= (overlaps1(b.lo[d], b.hi[d], lo.x, hi.x) ? 1u : 0u) | (overlaps1(b.lo[d], b.hi[d], lo.y, hi.y) ? 2u : 0u) |
         (overlaps1(b.lo[d], b.hi[d], lo.z, hi.z) ? 4u : 0u) | (overlaps1(b.lo[d], b.hi[d], lo.w, hi.w) ? 8u : 0u);
  }
  // objects past n (padding of the last leaf) never hit
  if (p + 4 > n) {
    const uint64_t valid = (n > p) ? (n - p) : 0;
    m &= (1u << valid) - 1u;
  }
  return m;
}

// Hit mask of objects g..g+3 of a leaf staged in shared memory: coordinate
// run c of the leaf at s + c * F (lo0..lo(D-1), then hi.. for rectangles);
// objects at or past `valid` (padding of the last leaf) never hit.
template <int D, bool RECT>
__device__ __forceinline__ uint32_t test4_staged(const Box<D>& b, const float* s, uint32_t F, uint32_t g,
                                                 uint32_t valid) {
  uint32_t m = 0xfu;
#pragma unroll
  for (int d = 0; d < D; ++d) {
    const float4 lo = *reinterpret_cast<const float4*>(s + (uint32_t)d * F + g);
    float4 hi = lo;
    if (RECT) hi = *reinterpret_cast<const float4*>(s + (uint32_t)(D + d) * F + g);
    m &= (overlaps1(b.lo[d], b.hi[d], lo.x, hi.x) ? 1u : 0u) | (overlaps1(b.lo[d], b.hi[d], lo.y, hi.y) ? 2u : 0u) |
         (overlaps1(b.lo[d], b.hi[d], lo.z, hi.z) ? 4u : 0u) | (overlaps1(b.lo[d], b.hi[d], lo.w, hi.w) ? 8u : 0u);
  }
  if (g + 4 > valid) m &= (g < valid) ? (1u << (valid - g)) - 1u : 0u;
  return m;
}

// ---------------------------------------------------------------------------
// Bulk copies (the TMA unit's non-tensor cp.async.bulk, global -> this CTA's
// shared memory, no multicast) completing on an mbarrier.  Every wait is
// bounded: after kBulkWaitCycles of clock it gives up and reports false.
// ---------------------------------------------------------------------------
constexpr long long kBulkWaitCycles = 4ll << 30;  // ~2 s at 2 GHz

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}
__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;\n" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_fence_init() {
  asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
}
__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t* bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;\n" ::"r"(smem_u32(bar)), "r"(bytes)
               : "memory");
}
__device__ __forceinline__ void bulk_copy_g2s(void* dst, const void* src, uint32_t bytes, uint64_t* bar) {
  asm volatile(
      "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];\n" ::"r"(
          smem_u32(dst)),
      "l"(src), "r"(bytes), "r"(smem_u32(bar))
      : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
      : "=r"(ok)
      : "r"(smem_u32(bar)), "r"(parity)
      : "memory");
  return ok != 0;
}
// Waits for phase `parity` of `bar` to complete; false if it did not within
// kBulkWaitCycles.
__device__ __forceinline__ bool mbar_wait_bounded(uint64_t* bar, uint32_t parity) {
  if (mbar_try_wait(bar, parity)) return true;
  const long long t0 = clock64();
  while (!mbar_try_wait(bar, parity)) {
    if (clock64() - t0 > kBulkWaitCycles) return false;
  }
  return true;
}

__device__ __forceinline__ uint32_t lane_lt_mask() {
  uint32_t m;
  asm("mov.u32 %0, %%lanemask_lt;" : "=r"(m));
  return m;
}

__device__ __forceinline__ uint32_t warp_excl_sum(uint32_t v, uint32_t* total) {
  const uint32_t lane = threadIdx.x & 31;
  uint32_t x = v;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    uint32_t y = __shfl_up_sync(0xffffffffu, x, o);
    if (lane >= (uint32_t)o) x += y;
  }
  *total = __shfl_sync(0xffffffffu, x, 31);
  return x - v;
}

#define QCP_DISPATCH_D(D_, ...)                  \
  switch (D_) {                                  \
    case 1: { constexpr int DD = 1; __VA_ARGS__; } break; \
    case 2: { constexpr int DD = 2; __VA_ARGS__; } break; \
    case 3: { constexpr int DD = 3; __VA_ARGS__; } break; \
    case 4: { constexpr int DD = 4; __VA_ARGS__; } break; \
    case 5: { constexpr int DD = 5; __VA_ARGS__; } break; \
    case 6: { constexpr int DD = 6; __VA_ARGS__; } break; \
    case 7: { constexpr int DD = 7; __VA_ARGS__; } break; \
    case 8: { constexpr int DD = 8; __VA_ARGS__; } break; \
    default: break;                              \
  }


}  // namespace qcp
