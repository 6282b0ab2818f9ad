/* CPU oracle for the triangle-counting path: TEST INFRASTRUCTURE ONLY (see tc_oracle.h).
 * Plain C; the product library never links this file. */
#include "tc_oracle.h"

#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

/* Restates hostSingleIntersection (tests/cct.cpp:32-69): early-out on empty or disjoint
 * ranges, then a merge in which a mismatch advances the smaller side with a linear skip.
 * The reference's optional self-edge skip is compiled out (#if(0), tests/cct.cpp:43-55),
 * so it is not restated. */
int32_t oracle_single_intersection(int32_t alen, const int32_t* a, int32_t blen, const int32_t* b) {
  int32_t ka = 0, kb = 0;
  uint32_t out = 0;
  if (!alen || !blen || a[alen - 1] < b[0] || b[blen - 1] < a[0]) return 0;
  while (ka < alen && kb < blen) {
    int32_t va = a[ka], vb = b[kb];
    if (va == vb) {
      ++ka;
      ++kb;
      ++out;
    } else if (va < vb) {
      ++ka;
      while (ka < alen && a[ka] < vb) ++ka;
    } else {
      ++kb;
      while (kb < blen && va > b[kb]) ++kb;
    }
  }
  return (int32_t)out;
}

/* Restates hostCountTriangles (tests/cct.cpp:71-89): one intersection per directed edge,
 * in CSR order, summed into an int64. */
void oracle_host_count_triangles(int32_t nv, const int64_t* off, const int32_t* ind, int32_t* triNE,
                                 int64_t* all_triangles) {
  int64_t sum = 0, edge = 0;
  for (int32_t src = 0; src < nv; ++src) {
    int32_t srclen = (int32_t)(off[src + 1] - off[src]);
    for (int64_t it = off[src]; it < off[src + 1]; ++it) {
      int32_t dest = ind[it];
      int32_t destlen = (int32_t)(off[dest + 1] - off[dest]);
      int32_t c = oracle_single_intersection(srclen, ind + off[src], destlen, ind + off[dest]);
      if (triNE) triNE[edge] = c;
      ++edge;
      sum += c;
    }
  }
  *all_triangles = sum;
}

/* Per-vertex output of devicecuStingerAllTriangles (src/static_triangle_counting/cct.cu:216-270)
 * with one lane per intersection: every neighbour dest of src is visited (the dest < src skip
 * is commented out at cct.cu:244-245), (src == dest) or a list shorter than 2 is skipped
 * (cct.cu:247-249), and the block sum overwrites out[src] (cct.cu:267-268). */
void oracle_static_per_vertex(int32_t nv, const int64_t* off, const int32_t* ind, int32_t* out) {
  for (int32_t src = 0; src < nv; ++src) {
    int32_t srclen = (int32_t)(off[src + 1] - off[src]);
    uint32_t t = 0;
    for (int64_t k = off[src]; k < off[src + 1]; ++k) {
      int32_t dest = ind[k];
      int32_t destlen = (int32_t)(off[dest + 1] - off[dest]);
      if (src == dest || destlen < 2 || srclen < 2) continue;
      t += (uint32_t)oracle_single_intersection(srclen, ind + off[src], destlen, ind + off[dest]);
    }
    out[src] = (int32_t)t;
  }
}

/* Per-vertex output of count_all_trianglesGPU (tests/cct_csr.cu:228-276): as above with
 * `if (dest < src) continue` (tests/cct_csr.cu:252-253). */
void oracle_csr_per_vertex(int32_t nv, const int64_t* off, const int32_t* ind, int32_t* out) {
  for (int32_t src = 0; src < nv; ++src) {
    int32_t srclen = (int32_t)(off[src + 1] - off[src]);
    uint32_t t = 0;
    for (int64_t k = off[src]; k < off[src + 1]; ++k) {
      int32_t dest = ind[k];
      int32_t destlen = (int32_t)(off[dest + 1] - off[dest]);
      if (dest < src) continue;
      if (src == dest || destlen < 2 || srclen < 2) continue;
      t += (uint32_t)oracle_single_intersection(srclen, ind + off[src], destlen, ind + off[dest]);
    }
    out[src] = (int32_t)t;
  }
}

/* The masked merge of intersectCount<uMasked, vMasked, subtract, upd3rdV>
 * (src/streaming_triangle_counting/cct_upd.cu:146-176) with one lane per intersection:
 * a masked entry is stepped over, a match of two unmasked entries counts, and when
 * `third` is non-NULL each match adds `third_delta` to the matched vertex (cct_upd.cu:163-165). */
static int32_t masked_intersection(int32_t ulen, const int32_t* u, const int32_t* umask, int32_t vlen,
                                   const int32_t* v, const int32_t* vmask, uint32_t* third,
                                   uint32_t third_delta) {
  int32_t i = 0, j = 0;
  uint32_t tri = 0;
  while (i < ulen && j < vlen) {
    int um = umask ? umask[i] : 0;
    int vm = vmask ? vmask[j] : 0;
    int32_t a = u[i], b = v[j];
    int hit = (a == b) && !um && !vm;
    if (hit) {
      ++tri;
      if (third) third[a] += third_delta;
    }
    i += ((a <= b) && !vm) || um;
    j += ((a >= b) && !um) || vm;
  }
  return (int32_t)tri;
}

void oracle_new_triangles(int32_t nv, const int64_t* off, const int32_t* ind, const oracle_batch* bt,
                          int32_t* out_signed) {
  uint32_t* out = (uint32_t*)out_signed; /* wrap-around int32 accumulation */
  const int32_t* bsrc = bt->src;
  const int32_t* bdst = bt->dst;
  const int64_t* boff = bt->boff;
  const int32_t* dup = bt->dup;
  (void)nv;
  /* K1: every non-duplicate batch edge, intersected in the updated graph; +c to src and dst,
   * +1 to each third vertex (cct_upd.cu:251-283). */
  for (int64_t e = 0; e < bt->b; ++e) {
    if (dup[e] == 1) continue;
    int32_t s = bsrc[e], d = bdst[e];
    int32_t sl = (int32_t)(off[s + 1] - off[s]), dl = (int32_t)(off[d + 1] - off[d]);
    if (s == d || dl < 2 || sl < 2) continue;
    int ss = sl < dl;
    int32_t sm = ss ? s : d, lg = ss ? d : s;
    int32_t sml = ss ? sl : dl, lgl = ss ? dl : sl;
    uint32_t c = (uint32_t)masked_intersection(sml, ind + off[sm], NULL, lgl, ind + off[lg], NULL, out, 1u);
    out[s] += c;
    out[d] += c;
  }
  /* K2: batch-only lists of src and dst, both masked by the duplicate flags; +c to src only
   * (cct_upd.cu:307-339). */
  for (int64_t e = 0; e < bt->b; ++e) {
    if (dup[e]) continue;
    int32_t s = bsrc[e], d = bdst[e];
    int32_t sl = (int32_t)(boff[s + 1] - boff[s]), dl = (int32_t)(boff[d + 1] - boff[d]);
    if (s == d || dl < 2 || sl < 2) continue;
    int ss = sl < dl;
    int32_t sm = ss ? s : d, lg = ss ? d : s;
    int32_t sml = ss ? sl : dl, lgl = ss ? dl : sl;
    uint32_t c = (uint32_t)masked_intersection(sml, bdst + boff[sm], dup + boff[sm], lgl, bdst + boff[lg],
                                               dup + boff[lg], NULL, 0u);
    out[s] += c;
  }
  /* K3: the masked batch list of src against the updated graph list of dst; -c from src
   * and dst, -1 from each third vertex (cct_upd.cu:363-408). */
  for (int64_t e = 0; e < bt->b; ++e) {
    if (dup[e]) continue;
    int32_t s = bsrc[e], d = bdst[e];
    int32_t sl = (int32_t)(boff[s + 1] - boff[s]);
    int32_t dl = (int32_t)(off[d + 1] - off[d]);
    if (s == d || dl < 2 || sl < 2) continue;
    const int32_t* sp = bdst + boff[s];
    const int32_t* smk = dup + boff[s];
    const int32_t* dp = ind + off[d];
    uint32_t c;
    if (sl < dl)
      c = (uint32_t)masked_intersection(sl, sp, smk, dl, dp, NULL, out, (uint32_t)-1);
    else
      c = (uint32_t)masked_intersection(dl, dp, NULL, sl, sp, smk, out, (uint32_t)-1);
    out[s] -= c;
    out[d] -= c;
  }
}

/* ---- batch preparation -------------------------------------------------------------- */

static int cmp_pair(const void* x, const void* y) {
  const int64_t a = *(const int64_t*)x, b = *(const int64_t*)y;
  return (a > b) - (a < b);
}

static int has_edge(const int64_t* off, const int32_t* ind, int32_t s, int32_t d) {
  int64_t lo = off[s], hi = off[s + 1];
  while (lo < hi) {
    int64_t mid = lo + ((hi - lo) >> 1);
    if (ind[mid] < d) lo = mid + 1;
    else hi = mid;
  }
  return lo < off[s + 1] && ind[lo] == d;
}

void oracle_sort_batch(int32_t nv, const int64_t* off, const int32_t* ind, int64_t b, int32_t* src,
                       int32_t* dst, int64_t* boff, int32_t* dup) {
  int64_t* key = (int64_t*)malloc(sizeof(int64_t) * (size_t)(b > 0 ? b : 1));
  for (int64_t e = 0; e < b; ++e) key[e] = ((int64_t)src[e] << 32) | (uint32_t)dst[e];
  qsort(key, (size_t)b, sizeof(int64_t), cmp_pair);
  for (int64_t e = 0; e < b; ++e) {
    src[e] = (int32_t)(key[e] >> 32);
    dst[e] = (int32_t)(uint32_t)key[e];
  }
  free(key);
  memset(boff, 0, sizeof(int64_t) * ((size_t)nv + 1));
  for (int64_t e = 0; e < b; ++e) boff[src[e] + 1]++;
  for (int32_t v = 0; v < nv; ++v) boff[v + 1] += boff[v];
  for (int64_t e = 0; e < b; ++e) {
    int repeat = e > 0 && src[e] == src[e - 1] && dst[e] == dst[e - 1];
    dup[e] = (src[e] == dst[e]) || repeat || has_edge(off, ind, src[e], dst[e]);
  }
}

/* ---- scaled oracle ------------------------------------------------------------------ */

/* u precedes v in the degree orientation when (deg u, u) < (deg v, v). */
static inline int precedes(const int64_t* off, int32_t u, int32_t v) {
  int64_t du = off[u + 1] - off[u], dv = off[v + 1] - off[v];
  return du < dv || (du == dv && u < v);
}

void oracle_fast_count(int32_t nv, const int64_t* off, const int32_t* ind, int nthreads,
                       int64_t* total, int32_t* per_vertex) {
  oracle_fast_count_range(nv, off, ind, nthreads, 0, nv, total, per_vertex);
}

/* Out-degrees of the degree orientation. */
static int32_t* out_degrees(int32_t nv, const int64_t* off, const int32_t* ind, int nt) {
  int32_t* dp = (int32_t*)malloc(sizeof(int32_t) * (size_t)(nv > 0 ? nv : 1));
  (void)nt;
#pragma omp parallel for num_threads(nt) schedule(dynamic, 4096)
  for (int32_t u = 0; u < nv; ++u) {
    int32_t c = 0;
    for (int64_t k = off[u]; k < off[u + 1]; ++k) c += precedes(off, u, ind[k]);
    dp[u] = c;
  }
  return dp;
}

void oracle_centre_cost(int32_t nv, const int64_t* off, const int32_t* ind, int nthreads, int32_t* cost) {
#ifdef _OPENMP
  int nt = nthreads > 0 ? nthreads : omp_get_max_threads();
#else
  int nt = 1;
  (void)nthreads;
#endif
  int32_t* dp = out_degrees(nv, off, ind, nt);
#pragma omp parallel for num_threads(nt) schedule(dynamic, 1024)
  for (int32_t c = 0; c < nv; ++c) {
    const int32_t a = dp[c];
    uint64_t w = (uint64_t)(off[c + 1] - off[c]);
    for (int64_t k = off[c]; k < off[c + 1]; ++k) {
      const int32_t o = ind[k];
      const int32_t b = dp[o];
      if (b > 0 && (b < a || (b == a && c < o))) w += (uint64_t)b + 2u;
    }
    const uint64_t q = (w + 15u) / 16u;
    cost[c] = q > (uint64_t)INT32_MAX ? INT32_MAX : (int32_t)q;
  }
  free(dp);
}

void oracle_fast_count_shard(int32_t nv, const int64_t* off, const int32_t* ind, int nthreads, int32_t shard,
                             int32_t nshards, int64_t* total, int32_t* per_vertex) {
  oracle_fast_count_split(nv, off, ind, nthreads, shard, nshards, 0, nv, total, per_vertex);
}

void oracle_fast_count_range(int32_t nv, const int64_t* off, const int32_t* ind, int nthreads, int32_t lo,
                             int32_t hi, int64_t* total, int32_t* per_vertex) {
  oracle_fast_count_split(nv, off, ind, nthreads, 0, 1, lo, hi, total, per_vertex);
}

void oracle_fast_count_split(int32_t nv, const int64_t* off, const int32_t* ind, int nthreads, int32_t shard,
                             int32_t nshards, int32_t lo, int32_t hi, int64_t* total, int32_t* per_vertex) {
#ifdef _OPENMP
  int nt = nthreads > 0 ? nthreads : omp_get_max_threads();
#else
  int nt = 1;
  (void)nthreads;
#endif
  /* Oriented CSR: keep v in N(u) when u precedes v; lists stay ascending by id. */
  int64_t* poff = (int64_t*)malloc(sizeof(int64_t) * ((size_t)nv + 1));
  poff[0] = 0;
#pragma omp parallel for num_threads(nt) schedule(dynamic, 4096)
  for (int32_t u = 0; u < nv; ++u) {
    int64_t c = 0;
    for (int64_t k = off[u]; k < off[u + 1]; ++k) c += precedes(off, u, ind[k]);
    poff[u + 1] = c;
  }
  for (int32_t u = 0; u < nv; ++u) poff[u + 1] += poff[u];
  int32_t* pind = (int32_t*)malloc(sizeof(int32_t) * (size_t)(poff[nv] > 0 ? poff[nv] : 1));
#pragma omp parallel for num_threads(nt) schedule(dynamic, 4096)
  for (int32_t u = 0; u < nv; ++u) {
    int64_t p = poff[u];
    for (int64_t k = off[u]; k < off[u + 1]; ++k)
      if (precedes(off, u, ind[k])) pind[p++] = ind[k];
  }
  uint32_t* t = per_vertex ? (uint32_t*)per_vertex : NULL;
  if (t) memset(t, 0, sizeof(uint32_t) * (size_t)nv);
  int64_t tri = 0;
#pragma omp parallel for num_threads(nt) schedule(dynamic, 64) reduction(+ : tri)
  for (int32_t u = 0; u < nv; ++u) {
    const int32_t* a = pind + poff[u];
    int64_t al = poff[u + 1] - poff[u];
    uint32_t tu = 0;
    for (int64_t i = 0; i < al; ++i) {
      int32_t v = a[i];
      const int32_t* bb = pind + poff[v];
      int64_t bl = poff[v + 1] - poff[v];
      if (nshards > 1 || lo > 0 || hi < nv) {
        /* A shard owns the edges whose centre (the endpoint with the larger out-degree, ties to
         * the smaller id: the GPU count's hash side) is one of its vertices. */
        const int32_t centre = (bl < al || (bl == al && u < v)) ? u : v;
        if (centre % nshards != shard || centre < lo || centre >= hi) continue;
      }
      int64_t x = 0, y = 0;
      uint32_t c = 0;
      while (x < al && y < bl) {
        int32_t p = a[x], q = bb[y];
        if (p == q) {
          ++c;
          if (t) __atomic_fetch_add(&t[p], 1u, __ATOMIC_RELAXED);
          ++x;
          ++y;
        } else if (p < q) {
          ++x;
        } else {
          ++y;
        }
      }
      tu += c;
      tri += c;
      if (t && c) __atomic_fetch_add(&t[v], c, __ATOMIC_RELAXED);
    }
    if (t && tu) __atomic_fetch_add(&t[u], tu, __ATOMIC_RELAXED);
  }
  if (t) {
#pragma omp parallel for num_threads(nt) schedule(static)
    for (int32_t v = 0; v < nv; ++v) t[v] = 2u * t[v];
  }
  *total = 6 * tri;
  free(poff);
  free(pind);
}

/* hostCountTriangles' per-edge loop (tests/cct.cpp:76-87) restricted to a list of source
 * vertices, on nthreads threads: the bounded CPU sample used when the reference's own
 * counter is not built. Returns the sum of the per-edge counts. */
int64_t oracle_host_count_sample(int32_t nv, const int64_t* off, const int32_t* ind, const int32_t* verts,
                                 int32_t nverts, int nthreads) {
  (void)nv;
#ifdef _OPENMP
  int nt = nthreads > 0 ? nthreads : omp_get_max_threads();
#else
  int nt = 1;
  (void)nthreads;
#endif
  int64_t sum = 0;
#pragma omp parallel for num_threads(nt) schedule(dynamic, 16) reduction(+ : sum)
  for (int32_t i = 0; i < nverts; ++i) {
    int32_t src = verts[i];
    int32_t srclen = (int32_t)(off[src + 1] - off[src]);
    for (int64_t it = off[src]; it < off[src + 1]; ++it) {
      int32_t dest = ind[it];
      int32_t destlen = (int32_t)(off[dest + 1] - off[dest]);
      sum += oracle_single_intersection(srclen, ind + off[src], destlen, ind + off[dest]);
    }
  }
  return sum;
}
