// C-ABI wrappers around the reference's own CPU triangle counter, compiled together with the
// reference source tests/cct.cpp (see oracle/Makefile). TEST / BASELINE INFRASTRUCTURE ONLY.
//
//   ref_host_count_triangles      -> hostCountTriangles (tests/cct.cpp:71-89), as written,
//                                    single thread: the reference CPU baseline.
//   ref_host_count_triangles_omp  -> the unmodified hostSingleIntersection (tests/cct.cpp:32-69)
//                                    called once per directed edge from an OpenMP loop over
//                                    source vertices: the same arithmetic on all host cores.
//   ref_host_count_triangles_omp_sample -> the same over a list of source vertices.
//   ref_host_count_triangles_omp_pervertex -> the same over all directed edges, each edge's count
//                                    summed into its source vertex (2 t(v), and the forward
//                                    counts of the raw-CSR convention): the per-vertex pin.
#include <cstdint>
#include <omp.h>
#include "cuStinger.hpp"
#include "static_triangle_counting/cct.hpp"

int hostSingleIntersection(const vertexId_t ai, const length_t alen, const vertexId_t* a,
                           const vertexId_t bi, const length_t blen, const vertexId_t* b);
void hostCountTriangles(const vertexId_t nv, const length_t* off, const vertexId_t* ind, int* triNE,
                        int64_t* allTriangles);

// The reference driver references these GPU entry points; they are never reached here.
void callDeviceAllTriangles(cuStinger&, triangle_t* const __restrict__, const int, const int,
                            const int, const int, const int) {
  ref_shim_unreachable("callDeviceAllTriangles");
}
void callDeviceAllTrianglesCSR(const vertexId_t, length_t const* const __restrict__,
                               vertexId_t const* const __restrict__, int* const __restrict__,
                               const int, const int, const int, const int, const int) {
  ref_shim_unreachable("callDeviceAllTrianglesCSR");
}

extern "C" {

int ref_host_single_intersection(int32_t ai, int32_t alen, const int32_t* a, int32_t bi, int32_t blen,
                                 const int32_t* b) {
  return hostSingleIntersection(ai, alen, a, bi, blen, b);
}

void ref_host_count_triangles(int32_t nv, const int32_t* off, const int32_t* ind, int32_t* triNE,
                              int64_t* all) {
  hostCountTriangles(nv, off, ind, triNE, all);
}

int64_t ref_host_count_triangles_omp(int32_t nv, const int32_t* off, const int32_t* ind, int nthreads) {
  int nt = nthreads > 0 ? nthreads : omp_get_max_threads();
  int64_t sum = 0;
#pragma omp parallel for num_threads(nt) schedule(dynamic, 256) reduction(+ : sum)
  for (int32_t src = 0; src < nv; ++src) {
    length_t srcLen = off[src + 1] - off[src];
    for (length_t it = off[src]; it < off[src + 1]; ++it) {
      vertexId_t dest = ind[it];
      length_t destLen = off[dest + 1] - off[dest];
      sum += hostSingleIntersection(src, srcLen, ind + off[src], dest, destLen, ind + off[dest]);
    }
  }
  return sum;
}

// The same per-edge calls restricted to the listed source vertices (a bounded sample of a
// full count, for timing on large graphs).
int64_t ref_host_count_triangles_omp_sample(int32_t nv, const int32_t* off, const int32_t* ind,
                                            const int32_t* verts, int32_t nverts, int nthreads) {
  (void)nv;
  int nt = nthreads > 0 ? nthreads : omp_get_max_threads();
  int64_t sum = 0;
#pragma omp parallel for num_threads(nt) schedule(dynamic, 16) reduction(+ : sum)
  for (int32_t i = 0; i < nverts; ++i) {
    const vertexId_t src = verts[i];
    length_t srcLen = off[src + 1] - off[src];
    for (length_t it = off[src]; it < off[src + 1]; ++it) {
      vertexId_t dest = ind[it];
      length_t destLen = off[dest + 1] - off[dest];
      sum += hostSingleIntersection(src, srcLen, ind + off[src], dest, destLen, ind + off[dest]);
    }
  }
  return sum;
}

// Per-vertex form of hostCountTriangles (tests/cct.cpp:71-89): the same unmodified
// hostSingleIntersection per directed edge, with each edge's count (the reference's triNE[edge])
// added to its source vertex, so pv[src] = sum of triNE over src's edges = 2 t(src), exact in
// int64. pv_fwd (nullable) gets the same sum over the edges with dest > src only: the raw-CSR
// GPU counter's forward convention (tests/cct_csr.cu:246-249). The loop runs over edges, not
// sources, so a hub's edges spread over all threads. Returns the sum over all edges (the
// reference's allTriangles, 6T).
int64_t ref_host_count_triangles_omp_pervertex(int32_t nv, const int32_t* off, const int32_t* ind,
                                               int64_t* pv, int64_t* pv_fwd, int nthreads) {
  int nt = nthreads > 0 ? nthreads : omp_get_max_threads();
  const int64_t m = off[nv];
  for (int32_t v = 0; v < nv; ++v) pv[v] = 0;
  if (pv_fwd)
    for (int32_t v = 0; v < nv; ++v) pv_fwd[v] = 0;
  int64_t sum = 0;
#pragma omp parallel num_threads(nt) reduction(+ : sum)
  {
    int32_t cur = -1;  // source of the last edge this thread took, and its running counts
    int64_t acc = 0, acc_fwd = 0;
#pragma omp for schedule(dynamic, 4096)
    for (int64_t e = 0; e < m; ++e) {
      if (cur < 0 || e < off[cur] || e >= off[cur + 1]) {
        if (cur >= 0 && acc) {
#pragma omp atomic
          pv[cur] += acc;
        }
        if (cur >= 0 && acc_fwd) {
#pragma omp atomic
          pv_fwd[cur] += acc_fwd;
        }
        acc = 0;
        acc_fwd = 0;
        int32_t lo = 0, hi = nv - 1;  // last vertex whose list starts at or before e
        while (lo < hi) {
          int32_t mid = lo + (hi - lo + 1) / 2;
          if (off[mid] <= e) lo = mid; else hi = mid - 1;
        }
        while (off[lo + 1] <= e) ++lo;  // skip empty lists that start at e
        cur = lo;
      }
      const vertexId_t src = cur;
      const length_t srcLen = off[src + 1] - off[src];
      const vertexId_t dest = ind[e];
      const length_t destLen = off[dest + 1] - off[dest];
      const int c = hostSingleIntersection(src, srcLen, ind + off[src], dest, destLen, ind + off[dest]);
      acc += c;
      if (pv_fwd && dest > src) acc_fwd += c;
      sum += c;
    }
    if (cur >= 0 && acc) {
#pragma omp atomic
      pv[cur] += acc;
    }
    if (cur >= 0 && acc_fwd) {
#pragma omp atomic
      pv_fwd[cur] += acc_fwd;
    }
  }
  return sum;
}

}  // extern "C"
