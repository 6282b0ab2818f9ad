/* Seeded synthetic graph generators (host C ABI, libtcgen.so).
 *
 * Stand-ins for the graph files the reference drivers read (tests/cct.cpp:239-257,
 * tests/cct_upd.cpp:204-222). Every generator returns a symmetric CSR with self-loops and
 * duplicates removed and each adjacency list sorted ascending; a graph is a pure function of
 * its parameters (counter-based random draws), independent of the thread count.
 */
#ifndef TC_GEN_H_
#define TC_GEN_H_

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

enum { TCGEN_OK = 0, TCGEN_ERR_ARG = 1, TCGEN_ERR_OOM = 2, TCGEN_ERR_IO = 3, TCGEN_ERR_FORMAT = 4 };
enum { TCGEN_FMT_AUTO = 0, TCGEN_FMT_DIMACS = 1, TCGEN_FMT_SNAP = 2, TCGEN_FMT_MTX = 3, TCGEN_FMT_BINARY = 4 };

typedef struct tcgen_csr {
  int32_t n;    /* vertices */
  int64_t m;    /* directed edges (2x undirected) */
  int64_t* off; /* n+1 offsets, malloc'd; free with tcgen_free */
  int32_t* ind; /* m neighbour ids, malloc'd */
} tcgen_csr;

/* Raw R-MAT endpoint pairs (no symmetrization): pair e uses counter stream `stream`.
 * a/b/c are the quadrant weights (d = 1-a-b-c); noise=1 applies the per-level +/-5%
 * perturbation of the reference's noisy R-MAT (tests/cct_upd.cpp:67-112). */
int tcgen_rmat_pairs(int scale, int64_t num_pairs, double a, double b, double c, uint64_t seed,
                     int noise, uint64_t stream, int nthreads, int32_t* src, int32_t* dst);

/* R-MAT graph with 2^scale vertices and edge_factor * 2^scale generated pairs. */
int tcgen_rmat(int scale, int edge_factor, double a, double b, double c, uint64_t seed, int noise,
               int nthreads, tcgen_csr* out);

/* Erdos-Renyi G(n, p) (each unordered pair present with probability p). */
int tcgen_er(int32_t n, double p, uint64_t seed, int nthreads, tcgen_csr* out);

/* Barabasi-Albert preferential attachment, m0 edges per new vertex. */
int tcgen_ba(int32_t n, int m0, uint64_t seed, int nthreads, tcgen_csr* out);

/* side x side 4-neighbour grid, each edge rewired to a random endpoint with prob. `rewire`. */
int tcgen_grid(int32_t side, double rewire, uint64_t seed, int nthreads, tcgen_csr* out);

/* Symmetric sorted deduplicated CSR from k undirected pairs (self-loops dropped). */
int tcgen_from_pairs(int32_t n, int64_t k, const int32_t* src, const int32_t* dst, int nthreads,
                     tcgen_csr* out);

/* Read a graph file into the symmetric sorted deduplicated CSR (self-loops dropped; every input
 * edge contributes both directions). Replaces the absent cuStinger core's readers that the
 * reference drivers call (tests/cct.cpp:239-257):
 *   TCGEN_FMT_DIMACS  METIS / DIMACS-10 adjacency (.graph; weights skipped as its fmt says)
 *   TCGEN_FMT_SNAP    edge list "u v", '#' comments, 0-based ids (.txt)
 *   TCGEN_FMT_MTX     MatrixMarket coordinate, 1-based (.mtx)
 *   TCGEN_FMT_BINARY  the cache tcgen_write_binary writes (.tccsr), read back as is
 *   TCGEN_FMT_AUTO    by the file name, as the reference driver chooses. */
int tcgen_read(const char* path, int format, int nthreads, tcgen_csr* out);

/* Write g as a binary CSR cache ("TCCSRv1\0", int64 n, int64 m, int64 off[n+1], int32 ind[m]). */
int tcgen_write_binary(const char* path, const tcgen_csr* g);

void tcgen_free(tcgen_csr* g);

#ifdef __cplusplus
}
#endif
#endif /* TC_GEN_H_ */
