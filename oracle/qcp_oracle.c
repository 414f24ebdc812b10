/*
 * CPU oracle for the spatial-index range-search path.
 *
 * TEST INFRASTRUCTURE ONLY: the checker the CUDA path is compared against,
 * never the product.  Every function cites the reference file:line it
 * restates (paths inside the reference project).  Pinned against the
 * reference compiled from its own sources (oracle/_ref) through the golden
 * vectors in tests/golden/.
 */
#include "qcp_oracle.h"

#include <math.h>
#include <pthread.h>
#include <stdlib.h>
#include <string.h>

static uint64_t low_ones(uint32_t k) { return k >= 64 ? ~0ull : ((1ull << k) - 1ull); }

/* Rotate the low `nd` bits of v right by r (hilbert_macro.h:17-18). */
static uint64_t rotr_nd(uint64_t v, uint32_t r, uint32_t nd) {
  uint64_t m = low_ones(nd);
  v &= m;
  if (r == 0) return v;
  return ((v >> r) | (v << (nd - r))) & m;
}

uint64_t oracle_hilbert_coords(uint32_t dims, uint32_t bits, const int64_t* coord) {
  if (dims <= 1) return (uint64_t)coord[0]; /* hilbert_mapper.cpp:65-66 */
  const uint32_t total = dims * bits;

  /* The coordinates are OR-ed into one word, dim dims-1 highest
   * (hilbert_mapper.cpp:31-34); only its low dims*bits bits are used below. */
  uint64_t packed = 0;
  for (uint32_t d = dims; d-- > 0;) {
    packed = (bits >= 64) ? 0 : (packed << bits);
    packed |= (uint64_t)coord[d];
  }

  /* Bit transpose (hilbert_mapper.cpp:135-183): level b of the result holds
   * bit b of every coordinate, coordinate d at bit d of that level. */
  uint64_t t = 0;
  for (uint32_t b = 0; b < bits; ++b) {
    for (uint32_t d = 0; d < dims; ++d) {
      uint64_t bit = (packed >> (d * bits + b)) & 1ull;
      t |= bit << (b * dims + d);
    }
  }

  uint64_t index;
  if (bits > 1) {
    const uint64_t nd_ones = low_ones(dims);
    const uint64_t nd1_ones = nd_ones >> 1;
    /* one set bit at the bottom of every level (hilbert_mapper.cpp:42) */
    uint64_t level_low = 0;
    for (uint32_t b = 0; b < bits; ++b) level_low |= 1ull << (b * dims);

    t ^= t >> dims; /* :44 */
    index = 0;
    uint32_t rotation = 0;
    uint64_t flip = 0;
    for (uint32_t lvl = bits; lvl-- > 0;) { /* :47-54, top level first */
      uint64_t g = (t >> (lvl * dims)) & nd_ones;
      g = rotr_nd(flip ^ g, rotation, dims);
      index = (dims >= 64) ? g : ((index << dims) | g);
      flip = 1ull << rotation;
      /* adjust_rotation (hilbert_macro.h:4-11): advance the rotation by one
       * plus the position of the lowest set bit among the low dims-1 bits */
      uint64_t low = g & (0ull - g) & nd1_ones;
      while (low) {
        low >>= 1;
        ++rotation;
      }
      if (++rotation >= dims) rotation -= dims;
    }
    index ^= level_low >> 1; /* :55 */
  } else {
    index = t;
  }
  /* prefix XOR over the whole index (:60-62) */
  for (uint32_t s = 1; s < total; s *= 2) index ^= index >> s;
  return index & low_ones(total);
}

static int64_t quantise(float p, uint32_t bits, uint32_t mode) {
  if (mode == ORACLE_KEY_REF) {
    /* (ll)(1000000*points[i]): float multiply then truncation (:21-23) */
    float s = 1000000.0f * p;
    return (int64_t)s;
  }
  float v = p;
  if (!(v > 0.0f)) v = 0.0f; /* negatives and NaN map to 0 */
  uint64_t maxq = low_ones(bits);
  if (v >= 1.0f) return (int64_t)maxq;
  float s = ldexpf(v, (int)bits); /* exact power-of-two scaling */
  uint64_t q = (uint64_t)s;
  if (q > maxq) q = maxq;
  return (int64_t)q;
}

void oracle_hilbert_keys(const float* objs, uint64_t n, uint32_t dims, uint32_t is_rect,
                         uint32_t bits, uint32_t mode, uint64_t* keys) {
  int64_t coord[64];
  const uint32_t stride = is_rect ? 2 * dims : dims;
  for (uint64_t i = 0; i < n; ++i) {
    const float* o = objs + i * stride;
    for (uint32_t d = 0; d < dims; ++d) {
      float p = is_rect ? 0.5f * (o[d] + o[dims + d]) : o[d];
      coord[d] = quantise(p, bits, mode);
    }
    keys[i] = oracle_hilbert_coords(dims, bits, coord);
  }
}

int oracle_overlap(const float* query, const float* lo, const float* hi, uint32_t dims) {
  for (uint32_t d = 0; d < dims; ++d) {
    if (query[d] > hi[d] || query[dims + d] < lo[d]) return 0;
  }
  return 1;
}

typedef struct {
  const float* objs;
  uint64_t n;
  uint32_t dims, is_rect;
  const float* boxes;
  uint32_t q0, q1;
  uint64_t* counts;      /* per-query counts (count mode) */
  const uint64_t* offs;  /* write mode */
  int32_t* ids;
} range_job;

static void* range_worker(void* arg) {
  range_job* j = (range_job*)arg;
  const uint32_t dims = j->dims;
  const uint32_t stride = j->is_rect ? 2 * dims : dims;
  for (uint32_t qi = j->q0; qi < j->q1; ++qi) {
    const float* box = j->boxes + (uint64_t)qi * 2 * dims;
    uint64_t c = 0;
    int32_t* out = j->ids ? j->ids + j->offs[qi] : NULL;
    for (uint64_t i = 0; i < j->n; ++i) {
      const float* o = j->objs + i * stride;
      const float* hi = j->is_rect ? o + dims : o;
      if (oracle_overlap(box, o, hi, dims)) {
        if (out) out[c] = (int32_t)i;
        ++c;
      }
    }
    if (j->counts) j->counts[qi] = c;
  }
  return NULL;
}

static void run_jobs(range_job base, uint32_t q, uint32_t threads) {
  if (threads < 1) threads = 1;
  if (threads > q) threads = q ? q : 1;
  pthread_t tid[256];
  range_job jobs[256];
  if (threads > 256) threads = 256;
  for (uint32_t t = 0; t < threads; ++t) {
    jobs[t] = base;
    jobs[t].q0 = (uint32_t)((uint64_t)q * t / threads);
    jobs[t].q1 = (uint32_t)((uint64_t)q * (t + 1) / threads);
  }
  if (threads == 1) {
    range_worker(&jobs[0]);
    return;
  }
  for (uint32_t t = 0; t < threads; ++t) pthread_create(&tid[t], NULL, range_worker, &jobs[t]);
  for (uint32_t t = 0; t < threads; ++t) pthread_join(tid[t], NULL);
}

void oracle_range_counts(const float* objs, uint64_t n, uint32_t dims, uint32_t is_rect,
                         const float* boxes, uint32_t q, uint32_t threads, uint64_t* counts) {
  range_job b;
  memset(&b, 0, sizeof(b));
  b.objs = objs; b.n = n; b.dims = dims; b.is_rect = is_rect; b.boxes = boxes;
  b.counts = counts;
  run_jobs(b, q, threads);
}

uint64_t oracle_range_ids(const float* objs, uint64_t n, uint32_t dims, uint32_t is_rect,
                          const float* boxes, uint32_t q, uint32_t threads,
                          uint64_t* offsets, int32_t* ids, uint64_t cap) {
  uint64_t* counts = (uint64_t*)malloc(sizeof(uint64_t) * (q ? q : 1));
  oracle_range_counts(objs, n, dims, is_rect, boxes, q, threads, counts);
  offsets[0] = 0;
  for (uint32_t i = 0; i < q; ++i) offsets[i + 1] = offsets[i] + counts[i];
  free(counts);
  uint64_t total = offsets[q];
  if (total > cap || ids == NULL) return total;
  range_job b;
  memset(&b, 0, sizeof(b));
  b.objs = objs; b.n = n; b.dims = dims; b.is_rect = is_rect; b.boxes = boxes;
  b.offs = offsets; b.ids = ids;
  run_jobs(b, q, threads);
  return total;
}

static const uint64_t* g_sort_keys; /* qsort has no context argument */
static int cmp_perm(const void* a, const void* b) {
  uint32_t ia = *(const uint32_t*)a, ib = *(const uint32_t*)b;
  uint64_t ka = g_sort_keys[ia], kb = g_sort_keys[ib];
  if (ka < kb) return -1;
  if (ka > kb) return 1;
  return (ia > ib) - (ia < ib);
}

void oracle_sort_perm(const uint64_t* keys, uint64_t n, uint32_t* perm) {
  for (uint64_t i = 0; i < n; ++i) perm[i] = (uint32_t)i;
  g_sort_keys = keys;
  qsort(perm, n, sizeof(uint32_t), cmp_perm);
  g_sort_keys = NULL;
}

uint32_t oracle_level_sizes(uint64_t n, uint32_t fanout, uint64_t* out, uint32_t max_levels) {
  uint32_t L = 0;
  uint64_t cur = n;
  do {
    cur = (cur + fanout - 1) / fanout;
    if (L < max_levels) out[L] = cur;
    ++L;
  } while (cur > 1);
  return L;
}

void oracle_node_mbrs(const float* sorted_objs, uint64_t n, uint32_t dims, uint32_t is_rect,
                      uint32_t fanout, float* mbr) {
  uint64_t sizes[64];
  uint32_t L = oracle_level_sizes(n, fanout, sizes, 64);
  const uint32_t stride = is_rect ? 2 * dims : dims;
  const uint32_t m = 2 * dims;
  /* leaves: min lo / max hi over the entries of each leaf */
  for (uint64_t j = 0; j < sizes[0]; ++j) {
    float* out = mbr + j * m;
    uint64_t e0 = j * fanout, e1 = e0 + fanout;
    if (e1 > n) e1 = n;
    for (uint32_t d = 0; d < dims; ++d) {
      float lo = INFINITY, hi = -INFINITY;
      for (uint64_t e = e0; e < e1; ++e) {
        const float* o = sorted_objs + e * stride;
        float l = o[d], h = is_rect ? o[dims + d] : o[d];
        if (l < lo) lo = l;
        if (h > hi) hi = h;
      }
      out[d] = lo;
      out[dims + d] = hi;
    }
  }
  /* upper levels: min/max over the children's MBRs */
  uint64_t below = 0;
  for (uint32_t l = 1; l < L; ++l) {
    const float* child = mbr + below * m;
    float* cur = mbr + (below + sizes[l - 1]) * m;
    for (uint64_t j = 0; j < sizes[l]; ++j) {
      uint64_t c0 = j * fanout, c1 = c0 + fanout;
      if (c1 > sizes[l - 1]) c1 = sizes[l - 1];
      for (uint32_t d = 0; d < dims; ++d) {
        float lo = INFINITY, hi = -INFINITY;
        for (uint64_t c = c0; c < c1; ++c) {
          if (child[c * m + d] < lo) lo = child[c * m + d];
          if (child[c * m + dims + d] > hi) hi = child[c * m + dims + d];
        }
        cur[j * m + d] = lo;
        cur[j * m + dims + d] = hi;
      }
    }
    below += sizes[l - 1];
  }
}
