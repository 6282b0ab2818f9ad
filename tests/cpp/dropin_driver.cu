// Drop-in check: the reference drivers' call pattern (tests/cct.cpp:230-286 and the
// InsertionTest of tests/cct_upd.cpp:194-424) compiled against this library's cuStinger-compatible
// headers. Unlike the reference driver, which printed "should be" next to the result, every
// comparison here is asserted; the process exits non-zero on the first mismatch.
//
// usage: dropin_driver <scale> <numEdges>
#include <cstdio>
#include <cstdlib>
#include <vector>

#include <cuda_runtime.h>

#include "cuStinger.hpp"
#include "static_triangle_counting/cct.hpp"
#include "streaming_triangle_counting/cct_upd.hpp"
#include "tc_gen.h"
#include "update.hpp"

#define CHECK(cond, ...)                                  \
  do {                                                    \
    if (!(cond)) {                                        \
      fprintf(stderr, "FAIL %s:%d: ", __FILE__, __LINE__); \
      fprintf(stderr, __VA_ARGS__);                       \
      fprintf(stderr, "\n");                              \
      exit(1);                                            \
    }                                                     \
  } while (0)

// Lehmer generator (Park-Miller minimal standard), as the reference's driver draws its edges.
static int g_seed = 1;
static double lehmer() {
  const int a = 16807, m = 2147483647, q = 127773, r = 2836;
  int k = g_seed / q;
  g_seed = a * (g_seed - k * q) - k * r;
  if (g_seed < 0) g_seed += m;
  return g_seed * (1.0 / m);
}

static int64_t sum_array(const triangle_t* h, vertexId_t nv) {
  int64_t s = 0;
  for (vertexId_t v = 0; v < nv; ++v) s += h[v];
  return s;
}

// A user kernel written against the cuStinger device API: sums every adjacency entry.
__global__ void sum_adjacency(cuStinger* custing, unsigned long long* out) {
  const vertexId_t nv = custing->nv;
  for (vertexId_t v = blockIdx.x * blockDim.x + threadIdx.x; v < nv; v += gridDim.x * blockDim.x) {
    const length_t len = custing->dVD->getUsed()[v];
    const vertexId_t* dst = custing->dVD->getAdj()[v]->dst;
    unsigned long long s = 0;
    for (length_t k = 0; k < len; ++k) s += (unsigned long long)dst[k];
    atomicAdd(out, s);
  }
}

static int64_t count_static(cuStinger& custing, triangle_t* d_tri, std::vector<triangle_t>& h, vertexId_t nv) {
  std::fill(h.begin(), h.end(), 0);
  cudaMemcpy(d_tri, h.data(), sizeof(triangle_t) * (nv + 1), cudaMemcpyHostToDevice);
  callDeviceAllTriangles(custing, d_tri, 1, 128, 0, 16000, 128);
  cudaMemcpy(h.data(), d_tri, sizeof(triangle_t) * (nv + 1), cudaMemcpyDeviceToHost);
  CHECK(custing.lastStatus() == TC_OK, "callDeviceAllTriangles failed");
  return sum_array(h.data(), nv);
}

int main(int argc, char** argv) {
  const int scale = argc > 1 ? atoi(argv[1]) : 10;
  const int numEdges = argc > 2 ? atoi(argv[2]) : 200;
  cudaSetDevice(0);

  tcgen_csr g;
  CHECK(tcgen_rmat(scale, 16, 0.57, 0.19, 0.19, 11, 0, 0, &g) == TCGEN_OK, "generator");
  const length_t nv = g.n, ne = (length_t)g.m;
  std::vector<length_t> off(nv + 1);
  std::vector<vertexId_t> adj(g.ind, g.ind + ne);
  for (length_t i = 0; i <= nv; ++i) off[i] = (length_t)g.off[i];
  tcgen_free(&g);

  // ---- static: the cuStinger handle and the raw CSR entry point (tests/cct.cpp:127-226) ----
  cuStinger custing(defaultInitAllocater, defaultUpdateAllocater);
  cuStingerInitConfig cuInit;
  cuInit.initState = eInitStateCSR;
  cuInit.maxNV = nv + 1;
  cuInit.useVWeight = false;
  cuInit.isSemantic = false;
  cuInit.useEWeight = false;
  cuInit.csrNV = nv;
  cuInit.csrNE = ne;
  cuInit.csrOff = off.data();
  cuInit.csrAdj = adj.data();
  cuInit.csrVW = NULL;
  cuInit.csrEW = NULL;
  custing.initializeCuStinger(cuInit);
  CHECK(custing.lastStatus() == TC_OK, "initializeCuStinger");
  CHECK(custing.getNumberEdgesUsed() == ne, "edges used %d vs %d", custing.getNumberEdgesUsed(), ne);

  triangle_t* d_tri = nullptr;
  cudaMalloc(&d_tri, sizeof(triangle_t) * (nv + 1));
  std::vector<triangle_t> h(nv + 1);
  const int64_t sumDevice = count_static(custing, d_tri, h, nv);

  length_t* d_off = nullptr;
  vertexId_t* d_ind = nullptr;
  cudaMalloc(&d_off, sizeof(length_t) * (nv + 1));
  cudaMalloc(&d_ind, sizeof(vertexId_t) * ne);
  cudaMemcpy(d_off, off.data(), sizeof(length_t) * (nv + 1), cudaMemcpyHostToDevice);
  cudaMemcpy(d_ind, adj.data(), sizeof(vertexId_t) * ne, cudaMemcpyHostToDevice);
  const int sweep_bs[] = {32, 64, 96, 128, 192, 256};
  const int sweep_tsp[] = {1, 2, 4, 8, 16, 32};
  int64_t csr0 = -1;
  for (int bs : sweep_bs)
    for (int t = 0; t < 6; ++t) {
      std::fill(h.begin(), h.end(), 0);
      cudaMemcpy(d_tri, h.data(), sizeof(triangle_t) * (nv + 1), cudaMemcpyHostToDevice);
      callDeviceAllTrianglesCSR(nv, d_off, d_ind, d_tri, sweep_tsp[t], bs / sweep_tsp[t], t, 16000, bs);
      cudaMemcpy(h.data(), d_tri, sizeof(triangle_t) * (nv + 1), cudaMemcpyDeviceToHost);
      const int64_t s = sum_array(h.data(), nv);
      if (csr0 < 0) csr0 = s;
      CHECK(s == csr0, "CSR sum changed with the launch config");
    }
  CHECK(2 * csr0 == sumDevice, "CSR total 3T=%lld vs handle total 6T=%lld", (long long)csr0, (long long)sumDevice);
  printf("static: 6T=%lld 3T=%lld T=%lld\n", (long long)sumDevice, (long long)csr0, (long long)(sumDevice / 6));

  // ---- the device view for user kernels ----
  unsigned long long* d_sum = nullptr;
  cudaMalloc(&d_sum, sizeof(unsigned long long));
  cudaMemset(d_sum, 0, sizeof(unsigned long long));
  sum_adjacency<<<64, 256>>>(custing.devicePtr(), d_sum);
  unsigned long long dev_sum = 0;
  cudaMemcpy(&dev_sum, d_sum, sizeof(dev_sum), cudaMemcpyDeviceToHost);
  unsigned long long host_sum = 0;
  for (length_t i = 0; i < ne; ++i) host_sum += (unsigned long long)adj[i];
  CHECK(dev_sum == host_sum, "device view adjacency sum %llu vs %llu", dev_sum, host_sum);

  // ---- streaming: remove edges, recount, re-insert in batches (tests/cct_upd.cpp:267-414) ----
  std::vector<length_t> len(nv);
  for (length_t i = 0; i < nv; ++i) len[i] = off[i + 1] - off[i];
  const length_t dupEdges = 20, dupsFromCUS = 20;
  const length_t numTotalEdges = numEdges + dupEdges + dupsFromCUS;
  const int numBatches = 5;
  std::vector<BatchUpdateData*> buds(numBatches);
  std::vector<vertexId_t> work(adj);
  for (int bi = 0; bi < numBatches; ++bi) {
    buds[bi] = new BatchUpdateData(numTotalEdges * 2, true, nv);
    vertexId_t* src = buds[bi]->getSrc();
    vertexId_t* dst = buds[bi]->getDst();
    for (length_t i = 0; i < numEdges; ++i) {
      vertexId_t a, b;
      length_t lena;
      do {
        a = (vertexId_t)(lehmer() * nv);
        lena = off[a + 1] - off[a];
        if (!lena) continue;
        b = (vertexId_t)(lehmer() * lena);
      } while (!lena || work[off[a] + b] == -1);
      src[i] = a;
      dst[i] = work[off[a] + b];
      work[off[a] + b] = -1;
      for (length_t k = off[dst[i]]; k < off[dst[i] + 1]; ++k)
        if (work[k] == a) { work[k] = -1; break; }
      len[a]--;
      len[dst[i]]--;
    }
    for (length_t i = 0; i < dupEdges; ++i) {
      src[numEdges + i] = src[i];
      dst[numEdges + i] = dst[i];
    }
    for (length_t i = 0; i < dupsFromCUS; ++i) {
      vertexId_t a, b;
      length_t lena;
      do {
        a = (vertexId_t)(lehmer() * nv);
        lena = off[a + 1] - off[a];
        if (!lena) continue;
        b = (vertexId_t)(lehmer() * lena);
      } while (!lena || work[off[a] + b] == -1);
      src[numEdges + dupEdges + i] = a;
      dst[numEdges + dupEdges + i] = work[off[a] + b];
    }
    for (length_t i = 0; i < numTotalEdges; ++i) {
      dst[numTotalEdges + i] = src[i];
      src[numTotalEdges + i] = dst[i];
    }
  }
  std::vector<length_t> newOff(nv + 1);
  length_t acc = 0;
  for (length_t i = 0; i <= nv; ++i) {
    newOff[i] = acc;
    if (i < nv) acc += len[i];
  }
  std::vector<vertexId_t> newAdj;
  newAdj.reserve(acc);
  for (length_t i = 0; i < ne; ++i)
    if (work[i] != -1) newAdj.push_back(work[i]);
  cuInit.csrNE = newOff[nv];
  cuInit.csrOff = newOff.data();
  cuInit.csrAdj = newAdj.data();
  cuStinger custingTest(defaultInitAllocater, defaultUpdateAllocater);
  custingTest.initializeCuStinger(cuInit);
  CHECK(custingTest.lastStatus() == TC_OK, "initializeCuStinger (reduced)");
  const int64_t sumDevice_reduced = count_static(custingTest, d_tri, h, nv);

  triangle_t* d_new = nullptr;
  cudaMalloc(&d_new, sizeof(triangle_t) * (nv + 1));
  cudaMemset(d_new, 0, sizeof(triangle_t) * (nv + 1));
  for (int bi = 0; bi < numBatches; ++bi) {
    BatchUpdate bu1(*buds[bi]);
    length_t allocs = 0;
    bu1.sortDeviceBUD(128);
    custingTest.edgeInsertionsSorted(bu1, allocs);
    CHECK(custingTest.lastStatus() == TC_OK, "edgeInsertionsSorted");
    callDeviceNewTriangles(custingTest, bu1, d_new, 1, 128, 0, 16000, 128, h.data(), h.data());
    CHECK(custingTest.lastStatus() == TC_OK, "callDeviceNewTriangles");
  }
  cudaMemcpy(h.data(), d_new, sizeof(triangle_t) * (nv + 1), cudaMemcpyDeviceToHost);
  const int64_t sumDevice_new = sum_array(h.data(), nv);
  printf("streaming: created %lld, expected %lld (original %lld, reduced %lld)\n", (long long)sumDevice_new,
         (long long)(sumDevice - sumDevice_reduced), (long long)sumDevice, (long long)sumDevice_reduced);
  CHECK(sumDevice_new == sumDevice - sumDevice_reduced, "streaming delta mismatch");
  CHECK(custingTest.getNumberEdgesUsed() == ne, "edge count after re-insertion %d vs %d",
        custingTest.getNumberEdgesUsed(), ne);
  const int64_t sumAfter = count_static(custingTest, d_tri, h, nv);
  CHECK(sumAfter == sumDevice, "recount after re-insertion %lld vs %lld", (long long)sumAfter, (long long)sumDevice);

  for (auto* b : buds) delete b;
  custing.freecuStinger();
  custingTest.freecuStinger();
  cudaFree(d_tri);
  cudaFree(d_new);
  cudaFree(d_off);
  cudaFree(d_ind);
  cudaFree(d_sum);
  printf("dropin driver ok\n");
  return 0;
}
