// Per-query sort of the output ids.
//
// The reference returns hit counts only; this library returns every query's
// hits as ascending input ids.  The traversal writes each query's ids in
// arbitrary order into its CSR slice; this file sorts every slice in place.
// Ids of one slice are distinct and lie in [0, n), so only the low
// `idbits` = ceil(log2 n) bits carry order.
//
//   slice <= kCap ids:  one CTA loads it into shared memory and runs a stable
//                       LSD radix sort with 8-bit digits (warp-match ranks),
//                       then writes it back.
//   slice >  kCap ids:  MSD rounds.  A round buckets the slice by the next 8
//                       bits below `hibit` (tile histograms -> per-slice
//                       bucket bases -> unordered scatter into the other
//                       buffer); every bucket of <= kCap ids is then sorted
//                       in shared memory into the output buffer, larger
//                       buckets go to the next round.  Distinct ids with at
//                       most 12 significant bits left always fit kCap, so
//                       31-bit ids need at most three rounds.
#include "qcp_internal.cuh"

namespace qcp {

namespace {

constexpr int SS_THREADS = 256;
constexpr int SS_WARPS = SS_THREADS / 32;
constexpr uint32_t kCap = 4096;
constexpr uint32_t SS_PER_WARP = kCap / SS_WARPS;  // 512
constexpr uint32_t SS_ROUNDS = SS_PER_WARP / 32;   // 16
constexpr uint32_t kTile = 4096;

struct Job {
  unsigned long long off;
  uint32_t size;
  uint32_t info;  // bit 0: data in tmp (1) or out (0); bits 8..15: hibit
};

__device__ __forceinline__ uint32_t lanemask_lt_() {
  uint32_t m;
  asm("mov.u32 %0, %%lanemask_lt;" : "=r"(m));
  return m;
}

// Stable LSD sort of a[0..n) (n <= kCap) on bits [0, hibit); the result ends
// in a.  b is scratch of kCap words.
__device__ void smem_sort(uint32_t* a, uint32_t* b, uint32_t n, uint32_t hibit,
                          uint32_t (*wcnt)[256], uint32_t* dig_excl, uint32_t* wtot) {
  const uint32_t tid = threadIdx.x, lane = tid & 31, w = tid >> 5;
  const uint32_t passes = (hibit + 7) / 8;
  for (uint32_t p = 0; p < passes; ++p) {
    const uint32_t shift = 8 * p;
    for (uint32_t i = tid; i < SS_WARPS * 256; i += SS_THREADS) (&wcnt[0][0])[i] = 0;
    __syncthreads();
    uint32_t rank[SS_ROUNDS];
    uint32_t key[SS_ROUNDS];
#pragma unroll
    for (uint32_t r = 0; r < SS_ROUNDS; ++r) {
      const uint32_t li = w * SS_PER_WARP + r * 32 + lane;
      const bool valid = li < n;
      key[r] = valid ? a[li] : 0u;
      rank[r] = 0;
      const uint32_t active = __ballot_sync(0xffffffffu, valid);
      if (valid) {
        const uint32_t d = (key[r] >> shift) & 255u;
        const uint32_t peers = __match_any_sync(active, d);
        const uint32_t prev = wcnt[w][d];
        rank[r] = prev + __popc(peers & lanemask_lt_());
        __syncwarp(active);
        if (lane == (uint32_t)(__ffs(peers) - 1)) wcnt[w][d] = prev + __popc(peers);
        __syncwarp(active);
      }
    }
    __syncthreads();
    // per digit (thread = digit): exclusive across warps, then across digits
    uint32_t run = 0;
    for (int k = 0; k < SS_WARPS; ++k) {
      const uint32_t c = wcnt[k][tid];
      wcnt[k][tid] = run;
      run += c;
    }
    // block exclusive scan of run over the 256 digits
    uint32_t x = run;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const uint32_t y = __shfl_up_sync(0xffffffffu, x, o);
      if (lane >= (uint32_t)o) x += y;
    }
    if (lane == 31) wtot[w] = x;
    __syncthreads();
    if (w == 0) {
      uint32_t t = (lane < SS_WARPS) ? wtot[lane] : 0u;
#pragma unroll
      for (int o = 1; o < SS_WARPS; o <<= 1) {
        const uint32_t y = __shfl_up_sync(0xffffffffu, t, o);
        if (lane >= (uint32_t)o) t += y;
      }
      if (lane < SS_WARPS) wtot[lane] = t;
    }
    __syncthreads();
    dig_excl[tid] = ((w > 0) ? wtot[w - 1] : 0u) + x - run;
    __syncthreads();
#pragma unroll
    for (uint32_t r = 0; r < SS_ROUNDS; ++r) {
      const uint32_t li = w * SS_PER_WARP + r * 32 + lane;
      if (li < n) {
        const uint32_t d = (key[r] >> shift) & 255u;
        b[dig_excl[d] + wcnt[w][d] + rank[r]] = key[r];
      }
    }
    __syncthreads();
    uint32_t* t = a;
    a = b;
    b = t;
  }
  if (passes & 1) {  // result is in the original b: copy back to a
    for (uint32_t i = tid; i < n; i += SS_THREADS) b[i] = a[i];
    __syncthreads();
  }
}

// Sorts `size` ids from src[off..) into out[off..) (src may equal out).
__device__ void sort_slice(const int32_t* src, int32_t* out, unsigned long long off, uint32_t size,
                           uint32_t hibit, uint32_t* sa, uint32_t* sb, uint32_t (*wcnt)[256],
                           uint32_t* dig_excl, uint32_t* wtot) {
  for (uint32_t i = threadIdx.x; i < size; i += SS_THREADS) sa[i] = (uint32_t)src[off + i];
  __syncthreads();
  if (size > 1) smem_sort(sa, sb, size, hibit, wcnt, dig_excl, wtot);
  for (uint32_t i = threadIdx.x; i < size; i += SS_THREADS) out[off + i] = (int32_t)sa[i];
  __syncthreads();
}

// Splits the queries into small jobs (sorted directly) and big jobs (MSD).
__global__ void k_classify(const unsigned long long* __restrict__ offsets, uint32_t q, uint32_t idbits,
                           Job* small, uint32_t* nsmall, Job* big, uint32_t* nbig) {
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < q; i += gridDim.x * blockDim.x) {
    const unsigned long long off = offsets[i];
    const unsigned long long sz = offsets[i + 1] - off;
    if (sz <= 1) continue;
    Job j;
    j.off = off;
    j.size = (uint32_t)sz;
    j.info = idbits << 8;
    if (sz <= kCap) {
      small[atomicAdd(nsmall, 1u)] = j;
    } else {
      big[atomicAdd(nbig, 1u)] = j;
    }
  }
}

__global__ void __launch_bounds__(SS_THREADS) k_sort_small(const Job* __restrict__ jobs, uint32_t njobs,
                                                           int32_t* out, int32_t* tmp) {
  __shared__ uint32_t sa[kCap];
  __shared__ uint32_t sb[kCap];
  __shared__ uint32_t wcnt[SS_WARPS][256];
  __shared__ uint32_t dig_excl[256];
  __shared__ uint32_t wtot[SS_WARPS];
  for (uint32_t j = blockIdx.x; j < njobs; j += gridDim.x) {
    const Job jb = jobs[j];
    const int32_t* src = (jb.info & 1u) ? tmp : out;
    sort_slice(src, out, jb.off, jb.size, (jb.info >> 8) & 255u, sa, sb, wcnt, dig_excl, wtot);
  }
}

__global__ void k_tiles_per_job(const Job* __restrict__ jobs, uint32_t njobs, uint32_t* tiles) {
  for (uint32_t j = blockIdx.x * blockDim.x + threadIdx.x; j < njobs; j += gridDim.x * blockDim.x)
    tiles[j] = (jobs[j].size + kTile - 1) / kTile;
}

__global__ void k_tile_map(const uint32_t* __restrict__ tiles, const uint32_t* __restrict__ tile_off,
                           uint32_t njobs, uint32_t* map) {
  for (uint32_t j = blockIdx.x; j < njobs; j += gridDim.x) {
    const uint32_t t0 = tile_off[j], nt = tiles[j];
    for (uint32_t k = threadIdx.x; k < nt; k += blockDim.x) map[t0 + k] = j;
  }
}

__device__ __forceinline__ uint32_t msd_digit(uint32_t id, uint32_t hibit) {
  const uint32_t lo = hibit > 8 ? hibit - 8 : 0;
  return (id >> lo) & 255u;
}

__global__ void __launch_bounds__(SS_THREADS) k_msd_hist(const Job* __restrict__ jobs,
                                                         const uint32_t* __restrict__ map,
                                                         const uint32_t* __restrict__ tile_off,
                                                         uint32_t ntiles, const int32_t* out,
                                                         const int32_t* tmp, uint32_t* hist) {
  __shared__ uint32_t h[256];
  for (uint32_t t = blockIdx.x; t < ntiles; t += gridDim.x) {
    h[threadIdx.x] = 0;
    __syncthreads();
    const uint32_t j = map[t];
    const Job jb = jobs[j];
    const int32_t* src = (jb.info & 1u) ? tmp : out;
    const uint32_t hibit = (jb.info >> 8) & 255u;
    const uint32_t k = t - tile_off[j];
    const uint32_t b0 = k * kTile;
    const uint32_t b1 = min(b0 + kTile, jb.size);
    for (uint32_t i = b0 + threadIdx.x; i < b1; i += SS_THREADS)
      atomicAdd(&h[msd_digit((uint32_t)src[jb.off + i], hibit)], 1u);
    __syncthreads();
    if (h[threadIdx.x]) atomicAdd(&hist[(size_t)j * 256 + threadIdx.x], h[threadIdx.x]);
    __syncthreads();
  }
}

// Per job: exclusive scan of its 256 bucket counts -> absolute bucket bases
// (base) and write cursors (cursor).
__global__ void __launch_bounds__(SS_THREADS) k_msd_scan(const Job* __restrict__ jobs, uint32_t njobs,
                                                         const uint32_t* __restrict__ hist,
                                                         unsigned long long* base,
                                                         unsigned long long* cursor) {
  __shared__ uint32_t wtot[SS_WARPS];
  const uint32_t lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  for (uint32_t j = blockIdx.x; j < njobs; j += gridDim.x) {
    const uint32_t c = hist[(size_t)j * 256 + threadIdx.x];
    uint32_t x = c;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const uint32_t y = __shfl_up_sync(0xffffffffu, x, o);
      if (lane >= (uint32_t)o) x += y;
    }
    if (lane == 31) wtot[w] = x;
    __syncthreads();
    uint32_t before = 0;
    for (uint32_t k = 0; k < w; ++k) before += wtot[k];
    const unsigned long long b = jobs[j].off + before + x - c;
    base[(size_t)j * 256 + threadIdx.x] = b;
    cursor[(size_t)j * 256 + threadIdx.x] = b;
    __syncthreads();
  }
}

__global__ void __launch_bounds__(SS_THREADS) k_msd_scatter(const Job* __restrict__ jobs,
                                                            const uint32_t* __restrict__ map,
                                                            const uint32_t* __restrict__ tile_off,
                                                            uint32_t ntiles, int32_t* out, int32_t* tmp,
                                                            unsigned long long* cursor) {
  __shared__ uint32_t h[256];
  __shared__ unsigned long long start[256];
  for (uint32_t t = blockIdx.x; t < ntiles; t += gridDim.x) {
    h[threadIdx.x] = 0;
    __syncthreads();
    const uint32_t j = map[t];
    const Job jb = jobs[j];
    const bool in_tmp = (jb.info & 1u) != 0;
    const int32_t* src = in_tmp ? tmp : out;
    int32_t* dst = in_tmp ? out : tmp;
    const uint32_t hibit = (jb.info >> 8) & 255u;
    const uint32_t k = t - tile_off[j];
    const uint32_t b0 = k * kTile;
    const uint32_t b1 = min(b0 + kTile, jb.size);
    for (uint32_t i = b0 + threadIdx.x; i < b1; i += SS_THREADS)
      atomicAdd(&h[msd_digit((uint32_t)src[jb.off + i], hibit)], 1u);
    __syncthreads();
    const uint32_t c = h[threadIdx.x];
    if (c) start[threadIdx.x] = atomicAdd(&cursor[(size_t)j * 256 + threadIdx.x], (unsigned long long)c);
    h[threadIdx.x] = 0;
    __syncthreads();
    for (uint32_t i = b0 + threadIdx.x; i < b1; i += SS_THREADS) {
      const int32_t id = src[jb.off + i];
      const uint32_t d = msd_digit((uint32_t)id, hibit);
      const uint32_t r = atomicAdd(&h[d], 1u);
      dst[start[d] + r] = id;
    }
    __syncthreads();
  }
}

// One CTA per (job, bucket): sort buckets that fit shared memory into out,
// queue the others for the next round.
__global__ void __launch_bounds__(SS_THREADS) k_msd_buckets(const Job* __restrict__ jobs, uint32_t njobs,
                                                            const uint32_t* __restrict__ hist,
                                                            const unsigned long long* __restrict__ base,
                                                            int32_t* out, int32_t* tmp, Job* next,
                                                            uint32_t* nnext, uint32_t next_cap,
                                                            uint32_t* overflow) {
  __shared__ uint32_t sa[kCap];
  __shared__ uint32_t sb[kCap];
  __shared__ uint32_t wcnt[SS_WARPS][256];
  __shared__ uint32_t dig_excl[256];
  __shared__ uint32_t wtot[SS_WARPS];
  const uint64_t total = (uint64_t)njobs * 256;
  for (uint64_t g = blockIdx.x; g < total; g += gridDim.x) {
    const uint32_t j = (uint32_t)(g >> 8), bkt = (uint32_t)(g & 255);
    const uint32_t size = hist[(size_t)j * 256 + bkt];
    if (size == 0) continue;
    const Job jb = jobs[j];
    const bool data_in_tmp = (jb.info & 1u) == 0;  // the scatter moved it to the other buffer
    const uint32_t hibit = (jb.info >> 8) & 255u;
    const uint32_t lo = hibit > 8 ? hibit - 8 : 0;
    const unsigned long long off = base[(size_t)j * 256 + bkt];
    if (size <= kCap) {
      sort_slice(data_in_tmp ? tmp : out, out, off, size, lo, sa, sb, wcnt, dig_excl, wtot);
    } else if (lo == 0) {
      // more than kCap ids share every bit: only possible with repeated ids
      if (threadIdx.x == 0) atomicOr(overflow, 2u);
    } else if (threadIdx.x == 0) {
      const uint32_t slot = atomicAdd(nnext, 1u);
      if (slot < next_cap) {
        Job nj;
        nj.off = off;
        nj.size = size;
        nj.info = (lo << 8) | (data_in_tmp ? 1u : 0u);
        next[slot] = nj;
      } else {
        atomicOr(overflow, 1u);
      }
    }
  }
}

}  // namespace

qcp_status ws_reserve_sort(qcp_index* ix, Workspace* ws, size_t jobs, size_t tiles);

// Workspace layout used here: ws->jobs[0] small jobs, ws->jobs[1] big jobs
// (both `jobs_cap` entries of 16 bytes); the MSD tables live in ix->pool.
qcp_status segmented_sort(qcp_index* ix, Workspace* ws, uint32_t q, cudaStream_t s) {
  ws->sort_small_jobs = ws->sort_msd_jobs = 0;
  if (q == 0) return QCP_OK;
  uint32_t idbits = 1;
  while (idbits < 31 && (1ull << idbits) < ix->n) ++idbits;
  const uint32_t sms = (uint32_t)num_sms();
  // job lists: one entry per query, and at most total/kCap oversized buckets
  const size_t njobs_max = (size_t)q + (size_t)(*ws->h_total / kCap) + 256;
  QCP_TRY(ws_reserve_sort(ix, ws, njobs_max, 0));
  uint32_t* ctr = ws->ctr;
  QCP_CUDA(cudaMemsetAsync(ctr + kCtrJobs0, 0, sizeof(uint32_t) * 3, s));
  Job* small = reinterpret_cast<Job*>(ws->jobs[0]);
  Job* big = reinterpret_cast<Job*>(ws->jobs[1]);
  k_classify<<<(q + 255) / 256, 256, 0, s>>>((const unsigned long long*)ws->offsets, q, idbits, small,
                                             ctr + kCtrJobs0, big, ctr + kCtrJobs1);
  note_launch();
  QCP_CUDA(cudaMemcpyAsync(ws->h_ctr, ctr, sizeof(uint32_t) * kCtrCount, cudaMemcpyDeviceToHost, s));
  QCP_CUDA(cudaStreamSynchronize(s));
  const uint32_t nsmall = ws->h_ctr[kCtrJobs0];
  uint32_t nbig = ws->h_ctr[kCtrJobs1];
  ws->sort_small_jobs = nsmall;
  ws->sort_msd_jobs = 0;
  if (nsmall) {
    k_sort_small<<<min(nsmall, sms * 16), SS_THREADS, 0, s>>>(small, nsmall, ws->out_ids, ws->tmp_ids);
    note_launch();
  }
  QCP_TRY(check_launch("k_sort_small"));
  // MSD rounds over the big jobs; the job list of a round lives in `cur`.
  Job* cur = big;
  void* tables = nullptr;
  size_t tables_bytes = 0;
  qcp_status st = QCP_OK;
  for (int round = 0; round < 4 && nbig > 0 && st == QCP_OK; ++round) {
    ws->sort_msd_jobs += nbig;
    const size_t need = (size_t)nbig * 256 * (4 + 8 + 8) + (size_t)nbig * 8 + 16;
    if (need > tables_bytes) {
      if (tables) ix->pool.put(tables_bytes, tables);
      tables = nullptr;
      tables_bytes = need;
      st = ix->pool.get(tables_bytes, &tables);
      if (st != QCP_OK) {
        tables_bytes = 0;
        break;
      }
    }
    uint32_t* hist = reinterpret_cast<uint32_t*>(tables);
    unsigned long long* base = reinterpret_cast<unsigned long long*>(hist + (size_t)nbig * 256);
    unsigned long long* cursor = base + (size_t)nbig * 256;
    uint32_t* tiles = reinterpret_cast<uint32_t*>(cursor + (size_t)nbig * 256);
    uint32_t* tile_off = tiles + nbig;
    // tiles per job -> offsets -> tile map
    k_tiles_per_job<<<(nbig + 255) / 256, 256, 0, s>>>(cur, nbig, tiles);
    note_launch();
    st = exclusive_scan<uint32_t>(tiles, tile_off, nbig, ctr + kCtrWork2, ix->pool, s);
    if (st != QCP_OK) break;
    QCP_CUDA(cudaMemcpyAsync(ws->h_ctr + kCtrWork2, ctr + kCtrWork2, sizeof(uint32_t),
                             cudaMemcpyDeviceToHost, s));
    QCP_CUDA(cudaStreamSynchronize(s));
    const uint32_t ntiles = ws->h_ctr[kCtrWork2];
    st = ws_reserve_sort(ix, ws, 0, ntiles);
    if (st != QCP_OK) break;
    uint32_t* map = reinterpret_cast<uint32_t*>(ws->seg_hist);
    k_tile_map<<<min(nbig, sms * 8), 256, 0, s>>>(tiles, tile_off, nbig, map);
    QCP_CUDA(cudaMemsetAsync(hist, 0, sizeof(uint32_t) * 256 * (size_t)nbig, s));
    k_msd_hist<<<min(ntiles, sms * 16), SS_THREADS, 0, s>>>(cur, map, tile_off, ntiles, ws->out_ids,
                                                            ws->tmp_ids, hist);
    k_msd_scan<<<min(nbig, sms * 16), SS_THREADS, 0, s>>>(cur, nbig, hist, base, cursor);
    k_msd_scatter<<<min(ntiles, sms * 16), SS_THREADS, 0, s>>>(cur, map, tile_off, ntiles, ws->out_ids,
                                                               ws->tmp_ids, cursor);
    note_launch(4);
    // next round's jobs go to the other list
    Job* next = (cur == big) ? small : big;
    QCP_CUDA(cudaMemsetAsync(ctr + kCtrJobs0, 0, sizeof(uint32_t), s));
    QCP_CUDA(cudaMemsetAsync(ctr + kCtrOverflow, 0, sizeof(uint32_t), s));
    const uint64_t grid = (uint64_t)nbig * 256;
    k_msd_buckets<<<(uint32_t)(grid < (uint64_t)sms * 16 ? grid : (uint64_t)sms * 16), SS_THREADS, 0, s>>>(
        cur, nbig, hist, base, ws->out_ids, ws->tmp_ids, next, ctr + kCtrJobs0,
        (uint32_t)ws->jobs_cap, ctr + kCtrOverflow);
    note_launch();
    st = check_launch("segmented_sort MSD round");
    if (st != QCP_OK) break;
    QCP_CUDA(cudaMemcpyAsync(ws->h_ctr, ctr, sizeof(uint32_t) * kCtrCount, cudaMemcpyDeviceToHost, s));
    QCP_CUDA(cudaStreamSynchronize(s));
    if (ws->h_ctr[kCtrOverflow]) {
      set_error((ws->h_ctr[kCtrOverflow] & 2u) ? "segmented sort: repeated ids in one result"
                                               : "segmented sort: job list overflow");
      st = QCP_ERR_CUDA;
      break;
    }
    nbig = ws->h_ctr[kCtrJobs0];
    cur = next;
  }
  if (tables) ix->pool.put(tables_bytes, tables);
  return st;
}

}  // namespace qcp
