// k-means-clustered Hilbert keys (QCP_KEY_KMEANS).
//
// The reference's KmeansMapper (src/mapper/kmeans_mapper.cpp:15-259) clusters
// the objects with k-means, orders the clusters by the Hilbert key of their
// centres and derives each object's key from its cluster's rank and its own
// Hilbert index, so that objects of one cluster end up in consecutive
// leaves -- meant for skewed data.  This is the same idea, made
// deterministic and cluster-major:
//
//   representative point  the object (points) or its centre (rectangles), as
//                         for the plain keys;
//   initial centres       the objects at positions floor(k * n / K) (the
//                         reference draws them with rand());
//   assignment            nearest centre by squared Euclidean distance in
//                         FP32, evaluated term by term without contraction,
//                         ties to the lowest centre index (find_nearest_cluster);
//   update                centre = mean of its members, with the sums kept in
//                         64-bit fixed point relative to the data's bounding
//                         box (32 fractional bits), so that the atomics are
//                         exact and the result does not depend on their
//                         order; an empty cluster keeps its centre;
//   stop                  when the fraction of objects that changed cluster
//                         is <= 1e-5 (DFN_KmeansThreashhold) or after
//                         max_iters assignments;
//   key                   rank of the cluster among the centres ordered by
//                         their normalised Hilbert key (ties by index) in the
//                         top ceil(log2 K) bits, the object's own normalised
//                         Hilbert key below it.
//
// The reference computes rank * n + own_index, where the 60-bit own index
// outweighs the rank; here the rank leads, so the key is cluster-major.
#include <algorithm>
#include <cmath>
#include <vector>

#include "qcp_internal.cuh"

namespace qcp {

namespace {

constexpr uint32_t kCentreTile = 1024;  // centres staged in shared memory per pass

__global__ void k_rep(const float* __restrict__ objs, uint64_t n, uint32_t dims, uint32_t is_rect,
                      float* __restrict__ rep) {
  const uint32_t stride = is_rect ? 2 * dims : dims;
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x) {
    const float* o = objs + i * stride;
    for (uint32_t d = 0; d < dims; ++d)
      rep[(uint64_t)d * n + i] = is_rect ? __fmul_rn(0.5f, __fadd_rn(o[d], o[dims + d])) : o[d];
  }
}

// per-dimension min / max: bounds[2d] = min, bounds[2d + 1] = max (as
// order-preserving unsigned keys of the floats)
__device__ __forceinline__ uint32_t f2key(float f) {
  const uint32_t u = __float_as_uint(f);
  return (u & 0x80000000u) ? ~u : (u | 0x80000000u);
}

__global__ void k_bounds(const float* __restrict__ rep, uint64_t n, uint32_t dims, uint32_t* bounds) {
  for (uint32_t d = 0; d < dims; ++d) {
    uint32_t lo = 0xffffffffu, hi = 0u;
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x) {
      const uint32_t k = f2key(rep[(uint64_t)d * n + i]);
      lo = min(lo, k);
      hi = max(hi, k);
    }
    for (int o = 16; o > 0; o >>= 1) {
      lo = min(lo, __shfl_xor_sync(0xffffffffu, lo, o));
      hi = max(hi, __shfl_xor_sync(0xffffffffu, hi, o));
    }
    if ((threadIdx.x & 31) == 0) {
      atomicMin(bounds + 2 * d, lo);
      atomicMax(bounds + 2 * d + 1, hi);
    }
  }
}

__global__ void k_init_centres(const float* __restrict__ rep, uint64_t n, uint32_t dims, uint32_t K,
                               float* __restrict__ centres) {
  for (uint32_t k = blockIdx.x * blockDim.x + threadIdx.x; k < K; k += gridDim.x * blockDim.x) {
    const uint64_t i = (uint64_t)k * n / K;
    for (uint32_t d = 0; d < dims; ++d) centres[(uint64_t)d * K + k] = rep[(uint64_t)d * n + i];
  }
}

// One assignment: nearest centre of every object, change count, fixed-point
// sums and counts of the new clusters.
__global__ void __launch_bounds__(256) k_assign(const float* __restrict__ rep, uint64_t n, uint32_t dims,
                                                const float* __restrict__ centres, uint32_t K,
                                                const double* __restrict__ lo, const double* __restrict__ scale,
                                                int32_t* __restrict__ member, unsigned long long* sums,
                                                unsigned long long* counts, unsigned long long* changes) {
  __shared__ float c[kCentreTile * kMaxDims];
  const uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
  float p[kMaxDims];
  for (uint32_t d = 0; d < dims; ++d) p[d] = i < n ? rep[(uint64_t)d * n + i] : 0.f;
  float best = INFINITY;
  int32_t arg = 0;
  for (uint32_t k0 = 0; k0 < K; k0 += kCentreTile) {
    const uint32_t kt = min(kCentreTile, K - k0);
    __syncthreads();
    for (uint32_t j = threadIdx.x; j < kt * dims; j += blockDim.x) {
      const uint32_t d = j / kt, k = j % kt;
      c[d * kCentreTile + k] = centres[(uint64_t)d * K + k0 + k];
    }
    __syncthreads();
    if (i < n) {
      for (uint32_t k = 0; k < kt; ++k) {
        float dist = 0.f;
        for (uint32_t d = 0; d < dims; ++d) {
          const float t = __fsub_rn(p[d], c[d * kCentreTile + k]);
          dist = __fadd_rn(dist, __fmul_rn(t, t));
        }
        if (dist < best) {
          best = dist;
          arg = (int32_t)(k0 + k);
        }
      }
    }
  }
  if (i >= n) return;
  if (member[i] != arg) {
    atomicAdd(changes, 1ull);
    member[i] = arg;
  }
  atomicAdd(counts + arg, 1ull);
  for (uint32_t d = 0; d < dims; ++d) {
    double f = ((double)p[d] - lo[d]) * scale[d];
    if (!(f > 0.0)) f = 0.0;
    if (f > 4294967296.0) f = 4294967296.0;
    atomicAdd(sums + (uint64_t)d * K + arg, (unsigned long long)f);
  }
}

__global__ void k_update(uint32_t dims, uint32_t K, const double* __restrict__ lo, const double* __restrict__ scale,
                         unsigned long long* sums, unsigned long long* counts, float* centres) {
  for (uint32_t k = blockIdx.x * blockDim.x + threadIdx.x; k < K; k += gridDim.x * blockDim.x) {
    const unsigned long long cnt = counts[k];
    for (uint32_t d = 0; d < dims; ++d) {
      if (cnt && scale[d] > 0.0)
        centres[(uint64_t)d * K + k] = (float)(lo[d] + ((double)sums[(uint64_t)d * K + k] / (double)cnt) / scale[d]);
      sums[(uint64_t)d * K + k] = 0;
    }
    counts[k] = 0;
  }
}

__global__ void k_combine(const int32_t* __restrict__ member, const uint32_t* __restrict__ rank, uint64_t n,
                          uint32_t rbits, uint32_t own_shift, uint64_t* keys) {
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x)
    keys[i] = ((uint64_t)rank[member[i]] << (64 - rbits)) | (keys[i] >> own_shift);
}

float key2f(uint32_t k) {
  const uint32_t u = (k & 0x80000000u) ? (k & 0x7fffffffu) : ~k;
  float f;
  memcpy(&f, &u, 4);
  return f;
}

// The plain normalised quantisation of the key kernel, on the host.
int64_t quantise_norm(float p, uint32_t bits) {
  float v = (p > 0.0f) ? p : 0.0f;
  const uint64_t maxq = low_ones64(bits);
  if (!(v < 1.0f)) return (int64_t)maxq;
  const uint64_t q = (uint64_t)(v * (float)(1ull << bits));
  return (int64_t)(q > maxq ? maxq : q);
}

}  // namespace

uint32_t kmeans_rank_bits(uint32_t K) {
  uint32_t r = 1;
  while (r < 32 && (1ull << r) < K) ++r;
  return r;
}

qcp_status build_keys_kmeans(const float* objs, uint64_t n, uint32_t dims, uint32_t is_rect, uint32_t bits,
                             uint32_t K, uint32_t max_iters, uint64_t* keys, uint32_t* vals, cudaStream_t s) {
  if (K > n) K = (uint32_t)n;
  if (K == 0) K = 1;
  const uint32_t sms = (uint32_t)num_sms();
  const size_t rep_b = sizeof(float) * dims * n;
  const size_t cen_b = sizeof(float) * dims * K;
  const size_t sum_b = sizeof(unsigned long long) * dims * K;
  const size_t cnt_b = sizeof(unsigned long long) * K;
  const size_t mem_b = sizeof(int32_t) * n;
  const size_t aux_b = 1024;  // bounds, lo, scale, change counter
  void* buf = nullptr;
  const size_t total = rep_b + cen_b + sum_b + cnt_b + mem_b + aux_b + sizeof(uint32_t) * K + 6 * 256;
  QCP_CUDA(cudaMalloc(&buf, total));
  char* p = reinterpret_cast<char*>(buf);
  auto take = [&](size_t b) {
    char* r = p;
    p += (b + 255) & ~(size_t)255;
    return r;
  };
  float* rep = (float*)take(rep_b);
  float* centres = (float*)take(cen_b);
  unsigned long long* sums = (unsigned long long*)take(sum_b);
  unsigned long long* counts = (unsigned long long*)take(cnt_b);
  int32_t* member = (int32_t*)take(mem_b);
  char* aux = take(aux_b);
  uint32_t* bounds = (uint32_t*)aux;                        // 2 * dims
  double* lo = (double*)(aux + 128);                        // dims
  double* scale = (double*)(aux + 256);                     // dims
  unsigned long long* changes = (unsigned long long*)(aux + 512);
  uint32_t* rank = (uint32_t*)take(sizeof(uint32_t) * K);
  qcp_status st = QCP_OK;
  do {
    const uint32_t grid = sms * 8;
    k_rep<<<grid, 256, 0, s>>>(objs, n, dims, is_rect, rep);
    std::vector<uint32_t> hb(2 * dims);
    for (uint32_t d = 0; d < dims; ++d) {
      hb[2 * d] = 0xffffffffu;
      hb[2 * d + 1] = 0u;
    }
    if (cudaMemcpyAsync(bounds, hb.data(), sizeof(uint32_t) * 2 * dims, cudaMemcpyHostToDevice, s) != cudaSuccess) {
      st = cuda_status(cudaGetLastError(), "kmeans bounds");
      break;
    }
    k_bounds<<<grid, 256, 0, s>>>(rep, n, dims, bounds);
    if (cudaMemcpyAsync(hb.data(), bounds, sizeof(uint32_t) * 2 * dims, cudaMemcpyDeviceToHost, s) != cudaSuccess ||
        cudaStreamSynchronize(s) != cudaSuccess) {
      st = cuda_status(cudaGetLastError(), "kmeans bounds");
      break;
    }
    std::vector<double> hlo(dims), hscale(dims);
    for (uint32_t d = 0; d < dims; ++d) {
      const double a = key2f(hb[2 * d]), b = key2f(hb[2 * d + 1]);
      hlo[d] = a;
      hscale[d] = (b > a && std::isfinite(b - a)) ? 4294967296.0 / (b - a) : 0.0;
    }
    if (cudaMemcpyAsync(lo, hlo.data(), sizeof(double) * dims, cudaMemcpyHostToDevice, s) != cudaSuccess ||
        cudaMemcpyAsync(scale, hscale.data(), sizeof(double) * dims, cudaMemcpyHostToDevice, s) != cudaSuccess ||
        cudaMemsetAsync(member, 0xff, mem_b, s) != cudaSuccess ||
        cudaMemsetAsync(sums, 0, sum_b, s) != cudaSuccess || cudaMemsetAsync(counts, 0, cnt_b, s) != cudaSuccess) {
      st = cuda_status(cudaGetLastError(), "kmeans setup");
      break;
    }
    k_init_centres<<<(K + 255) / 256, 256, 0, s>>>(rep, n, dims, K, centres);
    note_launch(3);
    unsigned long long h_changes = 0;
    for (uint32_t it = 0; it < max_iters; ++it) {
      if (cudaMemsetAsync(changes, 0, sizeof(unsigned long long), s) != cudaSuccess) {
        st = cuda_status(cudaGetLastError(), "kmeans");
        break;
      }
      k_assign<<<(uint32_t)((n + 255) / 256), 256, 0, s>>>(rep, n, dims, centres, K, lo, scale, member, sums, counts,
                                                           changes);
      k_update<<<(K + 255) / 256, 256, 0, s>>>(dims, K, lo, scale, sums, counts, centres);
      note_launch(2);
      if (cudaMemcpyAsync(&h_changes, changes, sizeof(h_changes), cudaMemcpyDeviceToHost, s) != cudaSuccess ||
          cudaStreamSynchronize(s) != cudaSuccess) {
        st = cuda_status(cudaGetLastError(), "kmeans");
        break;
      }
      if ((double)h_changes / (double)n <= 1e-5) break;
    }
    if (st != QCP_OK) break;
    // cluster ranks by the normalised Hilbert key of the centres
    std::vector<float> hc((size_t)dims * K);
    if (cudaMemcpy(hc.data(), centres, cen_b, cudaMemcpyDeviceToHost) != cudaSuccess) {
      st = cuda_status(cudaGetLastError(), "kmeans centres");
      break;
    }
    std::vector<std::pair<uint64_t, uint32_t>> ck(K);
    for (uint32_t k = 0; k < K; ++k) {
      int64_t cq[kMaxDims];
      for (uint32_t d = 0; d < dims; ++d) cq[d] = quantise_norm(hc[(size_t)d * K + k], bits);
      ck[k] = {hilbert_index(dims, bits, cq), k};
    }
    std::sort(ck.begin(), ck.end());
    std::vector<uint32_t> hr(K);
    for (uint32_t r = 0; r < K; ++r) hr[ck[r].second] = r;
    if (cudaMemcpyAsync(rank, hr.data(), sizeof(uint32_t) * K, cudaMemcpyHostToDevice, s) != cudaSuccess) {
      st = cuda_status(cudaGetLastError(), "kmeans ranks");
      break;
    }
    // own keys, then cluster-major keys
    if ((st = build_keys(objs, n, dims, is_rect, QCP_KEY_NORM, bits, keys, vals, s)) != QCP_OK) break;
    const uint32_t rbits = kmeans_rank_bits(K);
    const uint32_t own_bits = dims * bits;
    const uint32_t own_shift = own_bits > 64 - rbits ? own_bits - (64 - rbits) : 0;
    k_combine<<<grid, 256, 0, s>>>(member, rank, n, rbits, own_shift, keys);
    note_launch();
    st = check_launch("kmeans keys");
    if (st == QCP_OK && cudaStreamSynchronize(s) != cudaSuccess) st = cuda_status(cudaGetLastError(), "kmeans");
  } while (false);
  cudaFree(buf);
  return st;
}

}  // namespace qcp
