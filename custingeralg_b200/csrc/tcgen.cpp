// Seeded synthetic graph generators and CSR construction (host C++, OpenMP).
//
// The reference reads DIMACS / SNAP / MatrixMarket files (tests/cct.cpp:239-257) that are not
// shipped with it; these generators stand in for those inputs with the shapes the triangle
// counting workloads are quoted on: R-MAT (Graph500 a/b/c/d quadrant recursion, optional
// per-level noise as in tests/cct_upd.cpp:67-112), Erdos-Renyi G(n,p), Barabasi-Albert and a
// 2D grid with random rewiring.
//
// Every random draw comes from a counter-based generator (splitmix64 of seed, stream and
// counter), so a graph is a pure function of its parameters: the same on every machine and
// for every thread count. All graphs are returned symmetrized, with self-loops and duplicate
// edges removed and every adjacency list sorted ascending (the form the reference's readers
// hand to cuStinger's CSR initialisation, tests/cct.cpp:263-277).
#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstdint>
#include <cstdlib>
#include <cstring>
#include <vector>
#include <omp.h>

#include "../../include/tc_gen.h"

namespace {

inline uint64_t splitmix64(uint64_t x) {
  x += 0x9E3779B97F4A7C15ull;
  x = (x ^ (x >> 30)) * 0xBF58476D1CE4E5B9ull;
  x = (x ^ (x >> 27)) * 0x94D049BB133111EBull;
  return x ^ (x >> 31);
}

// One 64-bit draw for (seed, stream, counter).
inline uint64_t draw(uint64_t seed, uint64_t stream, uint64_t ctr) {
  uint64_t k = splitmix64(seed ^ 0x5851F42D4C957F2Dull) ^ splitmix64(stream * 0x2545F4914F6CDD1Dull + 1);
  return splitmix64(k + ctr * 0x9E3779B97F4A7C15ull);
}

// Uniform double in [0, 1) with 53 random bits.
inline double unif(uint64_t seed, uint64_t stream, uint64_t ctr) {
  return (double)(draw(seed, stream, ctr) >> 11) * (1.0 / 9007199254740992.0);
}

int nthreads_or_default(int nt) { return nt > 0 ? nt : omp_get_max_threads(); }

// Build a symmetric, sorted, deduplicated CSR without self-loops from k undirected pairs.
// Each pair (s[i], d[i]) contributes both directions.
int build_csr(int32_t n, int64_t k, const int32_t* s, const int32_t* d, int nt, tcgen_csr* out) {
  if (n < 0 || k < 0) return TCGEN_ERR_ARG;
  std::vector<std::atomic<int64_t>> cnt(n);
  for (int32_t v = 0; v < n; ++v) cnt[v].store(0, std::memory_order_relaxed);
#pragma omp parallel for num_threads(nt) schedule(static)
  for (int64_t i = 0; i < k; ++i) {
    int32_t a = s[i], b = d[i];
    if (a == b) continue;
    cnt[a].fetch_add(1, std::memory_order_relaxed);
    cnt[b].fetch_add(1, std::memory_order_relaxed);
  }
  std::vector<int64_t> start(n + 1);
  start[0] = 0;
  for (int32_t v = 0; v < n; ++v) start[v + 1] = start[v] + cnt[v].load(std::memory_order_relaxed);
  int64_t total = start[n];
  int32_t* tmp = (int32_t*)malloc(sizeof(int32_t) * (size_t)(total > 0 ? total : 1));
  if (!tmp) return TCGEN_ERR_OOM;
  std::vector<std::atomic<int64_t>> cur(n);
  for (int32_t v = 0; v < n; ++v) cur[v].store(start[v], std::memory_order_relaxed);
#pragma omp parallel for num_threads(nt) schedule(static)
  for (int64_t i = 0; i < k; ++i) {
    int32_t a = s[i], b = d[i];
    if (a == b) continue;
    tmp[cur[a].fetch_add(1, std::memory_order_relaxed)] = b;
    tmp[cur[b].fetch_add(1, std::memory_order_relaxed)] = a;
  }
  // Sort and deduplicate each list in place; record the deduplicated length.
  std::vector<int64_t> len(n);
#pragma omp parallel for num_threads(nt) schedule(dynamic, 1024)
  for (int32_t v = 0; v < n; ++v) {
    int32_t* b = tmp + start[v];
    int32_t* e = tmp + start[v + 1];
    std::sort(b, e);
    len[v] = std::unique(b, e) - b;
  }
  int64_t* off = (int64_t*)malloc(sizeof(int64_t) * ((size_t)n + 1));
  if (!off) { free(tmp); return TCGEN_ERR_OOM; }
  off[0] = 0;
  for (int32_t v = 0; v < n; ++v) off[v + 1] = off[v] + len[v];
  int64_t m = off[n];
  int32_t* ind = (int32_t*)malloc(sizeof(int32_t) * (size_t)(m > 0 ? m : 1));
  if (!ind) { free(tmp); free(off); return TCGEN_ERR_OOM; }
#pragma omp parallel for num_threads(nt) schedule(dynamic, 1024)
  for (int32_t v = 0; v < n; ++v) {
    if (len[v]) memcpy(ind + off[v], tmp + start[v], sizeof(int32_t) * (size_t)len[v]);
  }
  free(tmp);
  out->n = n;
  out->m = m;
  out->off = off;
  out->ind = ind;
  return TCGEN_OK;
}

}  // namespace

extern "C" {

int tcgen_rmat_pairs(int scale, int64_t num_pairs, double a, double b, double c, uint64_t seed,
                     int noise, uint64_t stream, int nthreads, int32_t* src, int32_t* dst) {
  if (scale < 1 || scale > 30 || num_pairs < 0) return TCGEN_ERR_ARG;
  double d = 1.0 - a - b - c;
  if (a < 0 || b < 0 || c < 0 || d < -1e-12) return TCGEN_ERR_ARG;
  int nt = nthreads_or_default(nthreads);
#pragma omp parallel for num_threads(nt) schedule(static)
  for (int64_t e = 0; e < num_pairs; ++e) {
    uint64_t ctr = (uint64_t)e * (uint64_t)(noise ? 5 * scale : scale);
    int64_t i = 0, j = 0;
    double A = a, B = b, C = c, D = d;
    for (int lvl = scale - 1; lvl >= 0; --lvl) {
      double r = unif(seed, stream, ctr++);
      int64_t bit = (int64_t)1 << lvl;
      if (r > A) {
        if (r <= A + B) j |= bit;
        else if (r <= A + B + C) i |= bit;
        else { i |= bit; j |= bit; }
      }
      if (noise) {
        // Per-level +/-5% perturbation of the quadrant weights, renormalised
        // (the noisy R-MAT of tests/cct_upd.cpp:87-105).
        A *= (9.5 + unif(seed, stream, ctr++)) / 10;
        B *= (9.5 + unif(seed, stream, ctr++)) / 10;
        C *= (9.5 + unif(seed, stream, ctr++)) / 10;
        D *= (9.5 + unif(seed, stream, ctr++)) / 10;
        double norm = 1.0 / (A + B + C + D);
        A *= norm; B *= norm; C *= norm;
        D = 1.0 - (A + B + C);
      }
    }
    src[e] = (int32_t)i;
    dst[e] = (int32_t)j;
  }
  return TCGEN_OK;
}

int tcgen_rmat(int scale, int edge_factor, double a, double b, double c, uint64_t seed, int noise,
               int nthreads, tcgen_csr* out) {
  if (scale < 1 || scale > 30 || edge_factor < 0) return TCGEN_ERR_ARG;
  int nt = nthreads_or_default(nthreads);
  int32_t n = (int32_t)((int64_t)1 << scale);
  int64_t k = (int64_t)edge_factor * (int64_t)n;
  std::vector<int32_t> s((size_t)k), d((size_t)k);
  int rc = tcgen_rmat_pairs(scale, k, a, b, c, seed, noise, 0, nt, s.data(), d.data());
  if (rc) return rc;
  return build_csr(n, k, s.data(), d.data(), nt, out);
}

int tcgen_er(int32_t n, double p, uint64_t seed, int nthreads, tcgen_csr* out) {
  if (n < 0 || !(p >= 0.0) || p > 1.0) return TCGEN_ERR_ARG;
  int nt = nthreads_or_default(nthreads);
  // Row i draws the pairs (i, j), j > i, by geometric skipping with its own stream.
  std::vector<std::vector<int32_t>> rows((size_t)n);
  if (p > 0.0) {
    double lq = std::log1p(-p);
#pragma omp parallel for num_threads(nt) schedule(dynamic, 256)
    for (int32_t i = 0; i < n; ++i) {
      uint64_t ctr = 0;
      int64_t j = i;
      while (true) {
        double r = unif(seed, (uint64_t)i, ctr++);
        int64_t skip = (p >= 1.0) ? 0 : (int64_t)std::floor(std::log1p(-r) / lq);
        j += skip + 1;
        if (j >= n) break;
        rows[i].push_back((int32_t)j);
      }
    }
  }
  int64_t k = 0;
  for (auto& r : rows) k += (int64_t)r.size();
  std::vector<int32_t> s((size_t)k), d((size_t)k);
  int64_t pos = 0;
  for (int32_t i = 0; i < n; ++i)
    for (int32_t j : rows[i]) { s[pos] = i; d[pos] = j; ++pos; }
  rows.clear();
  return build_csr(n, k, s.data(), d.data(), nt, out);
}

int tcgen_ba(int32_t n, int m0, uint64_t seed, int nthreads, tcgen_csr* out) {
  if (n < 2 || m0 < 1 || m0 >= n) return TCGEN_ERR_ARG;
  int nt = nthreads_or_default(nthreads);
  // Preferential attachment through the repeated-endpoint list: vertex t >= m0 + 1 joins
  // with m0 edges whose targets are uniform picks from all earlier endpoints (degree-
  // proportional). Vertices 0..m0 start as a clique.
  std::vector<int32_t> s, d, ends;
  s.reserve((size_t)n * m0);
  d.reserve((size_t)n * m0);
  ends.reserve((size_t)n * m0 * 2);
  for (int32_t i = 0; i <= m0; ++i)
    for (int32_t j = i + 1; j <= m0; ++j) {
      s.push_back(i); d.push_back(j);
      ends.push_back(i); ends.push_back(j);
    }
  uint64_t ctr = 0;
  for (int32_t t = m0 + 1; t < n; ++t) {
    size_t base = ends.size();
    for (int k2 = 0; k2 < m0; ++k2) {
      uint64_t r = draw(seed, 0, ctr++);
      int32_t tgt = ends[(size_t)(r % base)];
      s.push_back(t); d.push_back(tgt);
      ends.push_back(t); ends.push_back(tgt);
    }
  }
  return build_csr(n, (int64_t)s.size(), s.data(), d.data(), nt, out);
}

int tcgen_grid(int32_t side, double rewire, uint64_t seed, int nthreads, tcgen_csr* out) {
  if (side < 1 || rewire < 0 || rewire > 1) return TCGEN_ERR_ARG;
  int nt = nthreads_or_default(nthreads);
  int64_t n64 = (int64_t)side * side;
  if (n64 > INT32_MAX) return TCGEN_ERR_ARG;
  int32_t n = (int32_t)n64;
  // Right and down neighbours; each edge is rewired with probability `rewire` to a uniform
  // random endpoint (its source kept).
  int64_t k = 2 * n64;
  std::vector<int32_t> s((size_t)k), d((size_t)k);
#pragma omp parallel for num_threads(nt) schedule(static)
  for (int64_t v = 0; v < n64; ++v) {
    int64_t r = v / side, c = v % side;
    for (int dir = 0; dir < 2; ++dir) {
      int64_t e = 2 * v + dir;
      int64_t w;
      if (dir == 0) w = (c + 1 < side) ? v + 1 : v;
      else w = (r + 1 < side) ? v + side : v;
      if (unif(seed, 1, (uint64_t)e) < rewire) w = (int64_t)(draw(seed, 2, (uint64_t)e) % (uint64_t)n64);
      s[e] = (int32_t)v;
      d[e] = (int32_t)w;  // w == v (border or rewired onto itself) is dropped as a self-loop
    }
  }
  return build_csr(n, k, s.data(), d.data(), nt, out);
}

int tcgen_from_pairs(int32_t n, int64_t k, const int32_t* src, const int32_t* dst, int nthreads,
                     tcgen_csr* out) {
  for (int64_t i = 0; i < k; ++i)
    if (src[i] < 0 || src[i] >= n || dst[i] < 0 || dst[i] >= n) return TCGEN_ERR_ARG;
  return build_csr(n, k, src, dst, nthreads_or_default(nthreads), out);
}

void tcgen_free(tcgen_csr* g) {
  if (!g) return;
  free(g->off);
  free(g->ind);
  g->off = nullptr;
  g->ind = nullptr;
}

}  // extern "C"
