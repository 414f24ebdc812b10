/*
 * CPU oracle for the spatial-index range-search path.
 *
 * TEST INFRASTRUCTURE ONLY.  This library is the checker that the CUDA path
 * is compared against; it is never part of the product.  Only the tests,
 * __graft_entry__.smoke() and the CPU-baseline leg of bench.py load it.
 *
 * Each function restates the reference algorithm it cites (paths are inside
 * the reference project JinwoongKim/Query-Co-processing-on-Heterogeneous-
 * Architectures).  The restatement is pinned against the reference itself,
 * compiled from its own sources into oracle/_ref by oracle/Makefile, through
 * the golden vectors under tests/golden/.
 */
#ifndef QCP_ORACLE_H_
#define QCP_ORACLE_H_

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Quantisation modes for the Hilbert key. */
#define ORACLE_KEY_REF 0  /* (long long)(1000000.0f * p), hilbert_mapper.cpp:21-23 */
#define ORACLE_KEY_NORM 1 /* floor(clamp(p,0,1) * 2^bits), clamped to 2^bits-1  */

/* Hilbert index of integer coordinates coord[0..dims) with `bits` bits each.
 * Restates HilbertMapper::MappingIntoSingle (src/mapper/hilbert_mapper.cpp:25-64)
 * and the macros of src/mapper/hilbert_macro.h:4-22, in unsigned 64-bit
 * arithmetic so that dims*bits == 64 is defined. */
uint64_t oracle_hilbert_coords(uint32_t dims, uint32_t bits, const int64_t* coord);

/* Hilbert keys of n objects.  Points are row-major n x dims floats; rects
 * (is_rect=1) are row-major n x 2*dims floats [lo.., hi..] and are keyed on
 * their centre 0.5f*(lo+hi).  mode is ORACLE_KEY_REF or ORACLE_KEY_NORM. */
void oracle_hilbert_keys(const float* objs, uint64_t n, uint32_t dims, uint32_t is_rect,
                         uint32_t bits, uint32_t mode, uint64_t* keys);

/* The hit predicate of src/node/node_soa.cpp:94-113: entry overlaps query iff
 * for every dim d: !(q.lo[d] > e.hi[d] || q.hi[d] < e.lo[d]).  Closed intervals,
 * FP32 compares only, a NaN coordinate counts as overlap. */
int oracle_overlap(const float* query, const float* lo, const float* hi, uint32_t dims);

/* Per-query hit counts by brute force over every object (threads >= 1). */
void oracle_range_counts(const float* objs, uint64_t n, uint32_t dims, uint32_t is_rect,
                         const float* boxes, uint32_t q, uint32_t threads, uint64_t* counts);

/* Per-query sorted hit ids (0-based input positions) by brute force.
 * offsets has q+1 entries (offsets[0]=0); ids has offsets[q] entries and is
 * filled in ascending id order per query.  Returns offsets[q]; if that exceeds
 * cap nothing is written to ids. */
uint64_t oracle_range_ids(const float* objs, uint64_t n, uint32_t dims, uint32_t is_rect,
                          const float* boxes, uint32_t q, uint32_t threads,
                          uint64_t* offsets, int32_t* ids, uint64_t cap);

/* Stable order of keys: perm[i] = position of the i-th smallest key, equal keys
 * in input order.  Stands in for sort::Sorter::Sort (src/sort/sorter.cpp:11-29)
 * whose thrust/TBB sorts order equal keys arbitrarily. */
void oracle_sort_perm(const uint64_t* keys, uint64_t n, uint32_t* perm);

/* Node count per level, leaves first, for n entries packed `fanout` per node:
 * n <- ceil(n/fanout) until one node is left (src/tree/tree.cpp:654-667, which
 * lists the levels root first).  n == 1 gives one leaf.  Returns the number of
 * levels written to out (at most max_levels). */
uint32_t oracle_level_sizes(uint64_t n, uint32_t fanout, uint64_t* out, uint32_t max_levels);

/* MBRs of every node of the bottom-up packed tree over entries already in
 * sorted order (src/tree/tree.cpp:683-745 packing, :1025-1133 min/max build).
 * sorted_objs: n entries in sorted order, each dims (points) or 2*dims (rects)
 * floats.  mbr: for each level from the leaves up, for each node, 2*dims
 * floats [lo.., hi..]; total size = 2*dims*sum(level_sizes). */
void oracle_node_mbrs(const float* sorted_objs, uint64_t n, uint32_t dims, uint32_t is_rect,
                      uint32_t fanout, float* mbr);

#ifdef __cplusplus
}
#endif
#endif /* QCP_ORACLE_H_ */
