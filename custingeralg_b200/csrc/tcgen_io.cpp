// Graph file readers and a binary CSR cache (host C++, part of libtcgen.so).
//
// The reference's drivers read their inputs with readGraphDIMACS, readGraphSNAP and
// readGraphMatrixMarket (tests/cct.cpp:239-257, tests/cct_upd.cpp:204-222), which live in the
// absent cuStinger core. These readers give the triangle-counting path the form it needs:
// a symmetric CSR, 0-based ids, self-loops and duplicate edges removed, every list sorted
// ascending. Every input edge contributes both directions, whatever the file's own symmetry.
//
//   DIMACS (.graph)  the METIS / 10th DIMACS challenge adjacency format: '%' comments, a header
//                    "n m [fmt [ncon]]", then one line of 1-based neighbours per vertex (vertex
//                    sizes, vertex weights and edge weights skipped as fmt says).
//   SNAP (.txt)      '#' comments, one "u v" pair per line, 0-based ids; n = largest id + 1.
//   MatrixMarket (.mtx) "%%MatrixMarket matrix coordinate <field> <symmetry>", '%' comments, a
//                    size line "rows cols nnz", then nnz 1-based "i j [value...]" lines;
//                    n = max(rows, cols).
//   binary (.tccsr)  this library's cache: "TCCSRv1" and a zero byte, int64 n, int64 m,
//                    int64 off[n + 1], int32 ind[m] (little-endian), as tcgen_write_binary
//                    writes it; read back as is.
#include <algorithm>
#include <cctype>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include "../../include/cuStingerDefs.hpp"
#include "../../include/tc_gen.h"

extern "C" int tcgen_from_pairs(int32_t n, int64_t k, const int32_t* src, const int32_t* dst, int nthreads,
                                tcgen_csr* out);

namespace {

constexpr char kMagic[8] = {'T', 'C', 'C', 'S', 'R', 'v', '1', '\0'};

bool read_file(const char* path, std::string& buf) {
  FILE* f = fopen(path, "rb");
  if (!f) return false;
  if (fseek(f, 0, SEEK_END) != 0) {
    fclose(f);
    return false;
  }
  const long sz = ftell(f);
  if (sz < 0 || fseek(f, 0, SEEK_SET) != 0) {
    fclose(f);
    return false;
  }
  buf.resize((size_t)sz);
  const size_t got = sz > 0 ? fread(&buf[0], 1, (size_t)sz, f) : 0;
  fclose(f);
  return got == (size_t)sz;
}

// Line-by-line cursor over a text buffer with unsigned-integer token parsing.
struct Text {
  const char* p;
  const char* end;
  bool eof() const { return p >= end; }
  // [b, e) of the next line (without the newline); advances past it.
  void line(const char*& b, const char*& e) {
    b = p;
    while (p < end && *p != '\n') ++p;
    e = p;
    if (e > b && e[-1] == '\r') --e;
    if (p < end) ++p;
  }
};

// Parse an unsigned integer at s (after spaces); false at the end of the range or on junk.
bool next_uint(const char*& s, const char* e, uint64_t& v) {
  while (s < e && (*s == ' ' || *s == '\t')) ++s;
  if (s >= e || !isdigit((unsigned char)*s)) return false;
  uint64_t x = 0;
  while (s < e && isdigit((unsigned char)*s)) {
    x = x * 10 + (uint64_t)(*s - '0');
    if (x > (1ull << 40)) return false;
    ++s;
  }
  v = x;
  return true;
}

// Skip one whitespace-separated token of any kind (a weight, possibly real-valued).
bool skip_token(const char*& s, const char* e) {
  while (s < e && (*s == ' ' || *s == '\t')) ++s;
  if (s >= e) return false;
  while (s < e && *s != ' ' && *s != '\t') ++s;
  return true;
}

bool blank(const char* b, const char* e) {
  for (; b < e; ++b)
    if (*b != ' ' && *b != '\t') return false;
  return true;
}

int finish(int64_t n, std::vector<int32_t>& s, std::vector<int32_t>& d, int nthreads, tcgen_csr* out) {
  if (n > INT32_MAX) return TCGEN_ERR_FORMAT;
  return tcgen_from_pairs((int32_t)n, (int64_t)s.size(), s.data(), d.data(), nthreads, out);
}

int read_dimacs(const std::string& buf, int nthreads, tcgen_csr* out) {
  Text t{buf.data(), buf.data() + buf.size()};
  const char *b, *e;
  // header
  uint64_t n = 0, m = 0, fmt = 0;
  while (!t.eof()) {
    t.line(b, e);
    if (b < e && *b == '%') continue;
    if (blank(b, e)) continue;
    const char* s = b;
    if (!next_uint(s, e, n) || !next_uint(s, e, m)) return TCGEN_ERR_FORMAT;
    // fmt: up to three binary digits "abc": a = vertex sizes, b = vertex weights, c = edge weights
    next_uint(s, e, fmt);
    uint64_t ncon = 1;
    next_uint(s, e, ncon);
    const bool vsize = (fmt / 100) % 10 == 1, vwgt = (fmt / 10) % 10 == 1, ewgt = fmt % 10 == 1;
    std::vector<int32_t> src, dst;
    src.reserve((size_t)std::min<uint64_t>(2 * m, 1ull << 26));  // a hint only: the file may lie
    dst.reserve((size_t)std::min<uint64_t>(2 * m, 1ull << 26));
    uint64_t v = 0;
    while (v < n && !t.eof()) {
      t.line(b, e);
      if (b < e && *b == '%') continue;
      const char* q = b;
      if (vsize && !skip_token(q, e)) return TCGEN_ERR_FORMAT;
      if (vwgt)
        for (uint64_t c = 0; c < ncon; ++c)
          if (!skip_token(q, e)) return TCGEN_ERR_FORMAT;
      uint64_t u;
      while (next_uint(q, e, u)) {
        if (u < 1 || u > n) return TCGEN_ERR_FORMAT;
        src.push_back((int32_t)v);
        dst.push_back((int32_t)(u - 1));
        if (ewgt && !skip_token(q, e)) return TCGEN_ERR_FORMAT;
      }
      if (!blank(q, e)) return TCGEN_ERR_FORMAT;
      ++v;
    }
    // a file may end before its trailing isolated vertices' empty lines
    return finish((int64_t)n, src, dst, nthreads, out);
  }
  return TCGEN_ERR_FORMAT;
}

int read_snap(const std::string& buf, int nthreads, tcgen_csr* out) {
  Text t{buf.data(), buf.data() + buf.size()};
  const char *b, *e;
  std::vector<int32_t> src, dst;
  uint64_t mx = 0;
  bool any = false;
  while (!t.eof()) {
    t.line(b, e);
    if (b < e && (*b == '#' || *b == '%')) continue;
    if (blank(b, e)) continue;
    const char* q = b;
    uint64_t u, v;
    if (!next_uint(q, e, u) || !next_uint(q, e, v)) return TCGEN_ERR_FORMAT;
    if (u >= (uint64_t)INT32_MAX || v >= (uint64_t)INT32_MAX) return TCGEN_ERR_FORMAT;
    src.push_back((int32_t)u);
    dst.push_back((int32_t)v);
    mx = std::max(mx, std::max(u, v));
    any = true;
  }
  return finish(any ? (int64_t)mx + 1 : 0, src, dst, nthreads, out);
}

int read_mtx(const std::string& buf, int nthreads, tcgen_csr* out) {
  Text t{buf.data(), buf.data() + buf.size()};
  const char *b, *e;
  t.line(b, e);
  const std::string banner(b, e);
  std::string low(banner);
  for (auto& c : low) c = (char)tolower((unsigned char)c);
  if (low.rfind("%%matrixmarket", 0) != 0 || low.find("coordinate") == std::string::npos)
    return TCGEN_ERR_FORMAT;
  uint64_t rows = 0, cols = 0, nnz = 0;
  bool size_seen = false;
  std::vector<int32_t> src, dst;
  uint64_t got = 0;
  while (!t.eof()) {
    t.line(b, e);
    if (b < e && *b == '%') continue;
    if (blank(b, e)) continue;
    const char* q = b;
    if (!size_seen) {
      if (!next_uint(q, e, rows) || !next_uint(q, e, cols) || !next_uint(q, e, nnz)) return TCGEN_ERR_FORMAT;
      if (std::max(rows, cols) > (uint64_t)INT32_MAX) return TCGEN_ERR_FORMAT;
      src.reserve((size_t)std::min<uint64_t>(nnz, 1ull << 26));
      dst.reserve((size_t)std::min<uint64_t>(nnz, 1ull << 26));
      size_seen = true;
      continue;
    }
    uint64_t i, j;
    if (!next_uint(q, e, i) || !next_uint(q, e, j)) return TCGEN_ERR_FORMAT;
    if (i < 1 || j < 1 || i > rows || j > cols) return TCGEN_ERR_FORMAT;
    src.push_back((int32_t)(i - 1));
    dst.push_back((int32_t)(j - 1));
    ++got;
  }
  if (!size_seen || got != nnz) return TCGEN_ERR_FORMAT;
  return finish((int64_t)std::max(rows, cols), src, dst, nthreads, out);
}

int read_binary(const std::string& buf, tcgen_csr* out) {
  const size_t hdr = sizeof(kMagic) + 2 * sizeof(int64_t);
  if (buf.size() < hdr || memcmp(buf.data(), kMagic, sizeof(kMagic)) != 0) return TCGEN_ERR_FORMAT;
  int64_t n = 0, m = 0;
  memcpy(&n, buf.data() + sizeof(kMagic), sizeof(int64_t));
  memcpy(&m, buf.data() + sizeof(kMagic) + sizeof(int64_t), sizeof(int64_t));
  if (n < 0 || n > INT32_MAX || m < 0) return TCGEN_ERR_FORMAT;
  const size_t need = hdr + sizeof(int64_t) * ((size_t)n + 1) + sizeof(int32_t) * (size_t)m;
  if (buf.size() != need) return TCGEN_ERR_FORMAT;
  int64_t* off = (int64_t*)malloc(sizeof(int64_t) * ((size_t)n + 1));
  int32_t* ind = (int32_t*)malloc(sizeof(int32_t) * (size_t)(m > 0 ? m : 1));
  if (!off || !ind) {
    free(off);
    free(ind);
    return TCGEN_ERR_OOM;
  }
  memcpy(off, buf.data() + hdr, sizeof(int64_t) * ((size_t)n + 1));
  if (m) memcpy(ind, buf.data() + hdr + sizeof(int64_t) * ((size_t)n + 1), sizeof(int32_t) * (size_t)m);
  bool ok = off[0] == 0 && off[n] == m;
  for (int64_t v = 0; ok && v < n; ++v) ok = off[v] <= off[v + 1];
  for (int64_t k = 0; ok && k < m; ++k) ok = ind[k] >= 0 && ind[k] < n;
  if (!ok) {
    free(off);
    free(ind);
    return TCGEN_ERR_FORMAT;
  }
  out->n = (int32_t)n;
  out->m = m;
  out->off = off;
  out->ind = ind;
  return TCGEN_OK;
}

bool ends_with(const std::string& s, const char* suf) {
  const size_t k = strlen(suf);
  return s.size() >= k && s.compare(s.size() - k, k, suf) == 0;
}

}  // namespace

extern "C" int tcgen_read(const char* path, int format, int nthreads, tcgen_csr* out) {
  if (!path || !out) return TCGEN_ERR_ARG;
  out->n = 0;
  out->m = 0;
  out->off = nullptr;
  out->ind = nullptr;
  const std::string p(path);
  if (format == TCGEN_FMT_AUTO) {
    // by name, as the reference driver picks its reader (tests/cct.cpp:239-243)
    if (ends_with(p, ".tccsr")) format = TCGEN_FMT_BINARY;
    else if (p.find(".graph") != std::string::npos) format = TCGEN_FMT_DIMACS;
    else if (p.find(".txt") != std::string::npos) format = TCGEN_FMT_SNAP;
    else if (p.find(".mtx") != std::string::npos) format = TCGEN_FMT_MTX;
    else return TCGEN_ERR_ARG;
  }
  std::string buf;
  if (!read_file(path, buf)) return TCGEN_ERR_IO;
  switch (format) {
    case TCGEN_FMT_DIMACS: return read_dimacs(buf, nthreads, out);
    case TCGEN_FMT_SNAP: return read_snap(buf, nthreads, out);
    case TCGEN_FMT_MTX: return read_mtx(buf, nthreads, out);
    case TCGEN_FMT_BINARY: return read_binary(buf, out);
    default: return TCGEN_ERR_ARG;
  }
}

extern "C" int tcgen_write_binary(const char* path, const tcgen_csr* g) {
  if (!path || !g || g->n < 0 || g->m < 0 || (!g->off && g->n >= 0)) return TCGEN_ERR_ARG;
  FILE* f = fopen(path, "wb");
  if (!f) return TCGEN_ERR_IO;
  const int64_t n = g->n, m = g->m;
  bool ok = fwrite(kMagic, 1, sizeof(kMagic), f) == sizeof(kMagic) && fwrite(&n, sizeof(n), 1, f) == 1 &&
            fwrite(&m, sizeof(m), 1, f) == 1 &&
            fwrite(g->off, sizeof(int64_t), (size_t)n + 1, f) == (size_t)n + 1 &&
            (m == 0 || fwrite(g->ind, sizeof(int32_t), (size_t)m, f) == (size_t)m);
  ok = (fclose(f) == 0) && ok;
  return ok ? TCGEN_OK : TCGEN_ERR_IO;
}

// ---- the cuStinger core's reader entry points (drop-in for include/utils.hpp) -------------------
//
// Same call shape as the reference drivers use (tests/cct.cpp:245-254): the CSR comes back in
// malloc'd arrays (int32 offsets, nv + 1 of them, and ne neighbour ids) that the caller frees
// with free(). The flag argument (isRmat / undirected) is accepted and does not change the
// result: the triangle count needs the symmetric form, which every reader returns. A file that
// cannot be read or parsed leaves an empty graph and a message on stderr.
namespace {
void to_custinger(const char* path, int format, length_t** off, vertexId_t** adj, length_t* nv, length_t* ne) {
  tcgen_csr g{};
  int rc = tcgen_read(path, format, 0, &g);
  if (rc == TCGEN_OK && g.m > (int64_t)INT32_MAX) {
    tcgen_free(&g);
    rc = TCGEN_ERR_FORMAT;
    fprintf(stderr, "%s: more than 2^31-1 directed edges do not fit int32 offsets\n", path);
  }
  if (rc != TCGEN_OK) {
    fprintf(stderr, "%s: cannot read graph (error %d)\n", path, rc);
    *off = (length_t*)calloc(1, sizeof(length_t));
    *adj = nullptr;
    *nv = 0;
    *ne = 0;
    return;
  }
  length_t* o = (length_t*)malloc(sizeof(length_t) * ((size_t)g.n + 1));
  vertexId_t* a = (vertexId_t*)malloc(sizeof(vertexId_t) * (size_t)(g.m > 0 ? g.m : 1));
  for (int64_t v = 0; v <= g.n; ++v) o[v] = (length_t)g.off[v];
  if (g.m) memcpy(a, g.ind, sizeof(int32_t) * (size_t)g.m);
  *off = o;
  *adj = a;
  *nv = g.n;
  *ne = (length_t)g.m;
  tcgen_free(&g);
}
}  // namespace

void readGraphDIMACS(char* filePath, length_t** prmoff, vertexId_t** prmind, length_t* prmnv, length_t* prmne,
                     bool isRmat) {
  (void)isRmat;
  to_custinger(filePath, TCGEN_FMT_DIMACS, prmoff, prmind, prmnv, prmne);
}

void readGraphSNAP(char* filePath, length_t** prmoff, vertexId_t** prmind, length_t* prmnv, length_t* prmne,
                   bool undirected) {
  (void)undirected;
  to_custinger(filePath, TCGEN_FMT_SNAP, prmoff, prmind, prmnv, prmne);
}

void readGraphMatrixMarket(char* filePath, length_t** prmoff, vertexId_t** prmind, length_t* prmnv,
                           length_t* prmne, bool undirected) {
  (void)undirected;
  to_custinger(filePath, TCGEN_FMT_MTX, prmoff, prmind, prmnv, prmne);
}
