/* CPU oracle for the triangle-counting path: TEST INFRASTRUCTURE ONLY.
 *
 * A plain-C restatement of the reference's triangle counting, used by tests/, by
 * __graft_entry__.smoke() and by bench.py's CPU-baseline leg as the checker. Nothing in the
 * product library links or calls it.
 *
 * Parity pin: oracle_host_count_triangles is checked against the reference's own
 * hostCountTriangles (tests/cct.cpp:71-89), compiled from the reference sources into
 * oracle/_ref/ by oracle/Makefile, on the test graphs in tests/ and against the committed
 * known-answer fixtures in tests/golden/.
 *
 * Conventions (all integer, no floating point):
 *   - offsets are int64 (the reference's length_t is int32; int64 is a superset);
 *   - per-vertex outputs are int32 accumulated with two's-complement wrap, like the
 *     reference's int32 triangle_t arithmetic.
 */
#ifndef TC_ORACLE_H_
#define TC_ORACLE_H_

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* |a ∩ b| of two ascending lists; restates hostSingleIntersection (tests/cct.cpp:32-69). */
int32_t oracle_single_intersection(int32_t alen, const int32_t* a, int32_t blen, const int32_t* b);

/* Per-edge intersection counts and their int64 sum (= 6T on a symmetric simple graph);
 * restates hostCountTriangles (tests/cct.cpp:71-89). triNE may be NULL. */
void oracle_host_count_triangles(int32_t nv, const int64_t* off, const int32_t* ind, int32_t* triNE,
                                 int64_t* all_triangles);

/* out[src] = sum over dest in N(src), dest != src, deg(src) >= 2, deg(dest) >= 2 of
 * |N(src) ∩ N(dest)| (= 2 t(src)); what devicecuStingerAllTriangles writes
 * (src/static_triangle_counting/cct.cu:216-270). out has nv entries, overwritten. */
void oracle_static_per_vertex(int32_t nv, const int64_t* off, const int32_t* ind, int32_t* out);

/* The raw-CSR kernel's per-vertex output: as above but dest < src skipped
 * (tests/cct_csr.cu:228-276); its sum is 3T. */
void oracle_csr_per_vertex(int32_t nv, const int64_t* off, const int32_t* ind, int32_t* out);

/* Sorted batch as the streaming kernels consume it: entries sorted by (src, dst), batch CSR
 * offsets boff[nv+1] over src, dup[e] = 1 for a self-loop, a repeated entry, or an edge
 * already present before the batch was applied. */
typedef struct oracle_batch {
  int64_t b;
  const int32_t* src;
  const int32_t* dst;
  const int64_t* boff;
  const int32_t* dup;
} oracle_batch;

/* Accumulate into out[] (nv entries) the per-vertex deltas of the three streaming kernels
 * on the graph AFTER insertion (off/ind):
 *   K1 devicecuStingerNewTriangles  (src/streaming_triangle_counting/cct_upd.cu:231-285)
 *   K2 deviceBUThreeTriangles       (cct_upd.cu:287-341)
 *   K3 deviceBUTwoCUOneTriangles    (cct_upd.cu:343-410)
 * For a symmetric batch every vertex of every new triangle nets +2. */
void oracle_new_triangles(int32_t nv, const int64_t* off, const int32_t* ind, const oracle_batch* bt,
                          int32_t* out);

/* Sort a directed batch by (src, dst), build boff, and flag duplicates against the graph
 * BEFORE insertion (off/ind) and against earlier equal entries. Arrays are caller-owned:
 * src/dst (b entries, sorted in place), boff (nv+1), dup (b). */
void oracle_sort_batch(int32_t nv, const int64_t* off, const int32_t* ind, int64_t b, int32_t* src,
                       int32_t* dst, int64_t* boff, int32_t* dup);

/* Scaled oracle for large graphs (OpenMP, nthreads <= 0 means all): total = 6T and, when
 * per_vertex != NULL, per_vertex[v] = 2 t(v) (int32 wrap). Counts each triangle once over a
 * degree orientation; checked against the literal restatements above on every test graph. */
void oracle_fast_count(int32_t nv, const int64_t* off, const int32_t* ind, int nthreads,
                       int64_t* total, int32_t* per_vertex);

/* The same restricted to the triangles x < y < z (degree order) whose edge {x, y} has its
 * centre c with c % nshards == shard, the centre being the endpoint with the larger
 * out-degree (ties: the smaller id): the work split of the multi-GPU count. Summing the shards'
 * totals and per-vertex arrays gives the full count. */
void oracle_fast_count_shard(int32_t nv, const int64_t* off, const int32_t* ind, int nthreads, int32_t shard,
                             int32_t nshards, int64_t* total, int32_t* per_vertex);

/* The same restricted to the triangles whose edge {x, y} has its centre in [lo, hi): a shard of
 * the multi-GPU count as it splits the centres into contiguous ranges. */
void oracle_fast_count_range(int32_t nv, const int64_t* off, const int32_t* ind, int nthreads, int32_t lo,
                             int32_t hi, int64_t* total, int32_t* per_vertex);

/* Both restrictions at once (modulo shard and centre range). */
void oracle_fast_count_split(int32_t nv, const int64_t* off, const int32_t* ind, int nthreads, int32_t shard,
                             int32_t nshards, int32_t lo, int32_t hi, int64_t* total, int32_t* per_vertex);

/* Predicted work of each centre c, the quantity the multi-GPU split balances: over the edges
 * {c, o} that c is the centre of (o with out-degree b >= 1 and b < d+(c), or b == d+(c) and
 * c < o), b + 2 each, plus deg(c); in units of 16, rounded up, clamped to int32. */
void oracle_centre_cost(int32_t nv, const int64_t* off, const int32_t* ind, int nthreads, int32_t* cost);

/* The per-edge loop of hostCountTriangles over a list of source vertices (bounded sample). */
int64_t oracle_host_count_sample(int32_t nv, const int64_t* off, const int32_t* ind, const int32_t* verts,
                                 int32_t nverts, int nthreads);

#ifdef __cplusplus
}
#endif
#endif /* TC_ORACLE_H_ */
