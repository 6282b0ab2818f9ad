// Runs the reference's own graph algorithms (breadth-first search top-down, bottom-up and
// hybrid; connected components baseline, concurrent and load-balanced; PageRank), compiled
// unmodified from its src/ tree, on this repository's cuStinger handle and traversal operators
// (include/operators.cuh, include/load_balance.cuh, include/algs.cuh), and writes their outputs
// for the tests to check against CPU restatements.
//
//   ref_ops_driver <graph.graph> <bfs root> <out prefix>
// writes <prefix>.bfs_td, .bfs_bu, .bfs_hy (int32 levels, INT32_MAX = unreached), .cc_base,
// .cc_conc, .cc_lb (int32 labels), .pr (float32 scores) and prints one summary line per algorithm.
#include <cstdio>
#include <cstdlib>
#include <vector>

#include "cuStinger.hpp"
#include "operators.cuh"
#include "static_breadth_first_search/bfs_bottom_up.cuh"
#include "static_breadth_first_search/bfs_hybrid.cuh"
#include "static_breadth_first_search/bfs_top_down.cuh"
#include "static_connected_components/cc.cuh"
#include "static_page_rank/pr.cuh"
#include "utils.hpp"

using namespace cuStingerAlgs;

// The connected-component labels are protected members; these subclasses read them.
struct CcBase : ccBaseline {
  vertexId_t* labels() { return hostCCData.currState; }
};
struct CcConc : ccConcurrent {
  vertexId_t* labels() { return hostCCData.currState; }
};
struct CcLb : ccConcurrentLB {
  vertexId_t* labels() { return hostCCData.currState; }
};

static void dump(const char* prefix, const char* ext, const void* dev, size_t bytes) {
  std::vector<char> h(bytes);
  cudaMemcpy(h.data(), dev, bytes, cudaMemcpyDeviceToHost);
  char path[4096];
  snprintf(path, sizeof(path), "%s.%s", prefix, ext);
  FILE* f = fopen(path, "wb");
  if (!f) {
    fprintf(stderr, "cannot write %s\n", path);
    exit(2);
  }
  fwrite(h.data(), 1, bytes, f);
  fclose(f);
}

template <class Bfs>
static void run_bfs(cuStinger& cs, vertexId_t root, const char* prefix, const char* ext, const char* name) {
  Bfs b;
  b.Init(cs);
  b.setInputParameters(root);
  b.Run(cs);
  std::vector<vertexId_t> lv(cs.nv);
  b.getLevelArrayForHost(lv.data());
  char path[4096];
  snprintf(path, sizeof(path), "%s.%s", prefix, ext);
  FILE* f = fopen(path, "wb");
  fwrite(lv.data(), sizeof(vertexId_t), lv.size(), f);
  fclose(f);
  printf("%s levels %d\n", name, (int)b.getLevels());
  b.Release();
}

template <class Cc>
static void run_cc(cuStinger& cs, const char* prefix, const char* ext, const char* name) {
  Cc c;
  c.Init(cs);
  c.Run(cs);
  dump(prefix, ext, c.labels(), sizeof(vertexId_t) * cs.nv);
  const int iters = (int)c.GetIterationCount();
  const int comps_all = (int)c.CountConnectComponentsAll(cs);
  c.Reset();  // the count accumulates across calls; Reset zeroes it and keeps the labels
  const int comps = (int)c.CountConnectComponents(cs);
  printf("%s iterations %d components_all %d components %d\n", name, iters, comps_all, comps);
  c.Release();
}

int main(int argc, char** argv) {
  if (argc < 4) {
    fprintf(stderr, "usage: %s graph.graph root out_prefix\n", argv[0]);
    return 1;
  }
  length_t nv = 0, ne = 0, *off = nullptr;
  vertexId_t* adj = nullptr;
  readGraphDIMACS(argv[1], &off, &adj, &nv, &ne, false);
  const vertexId_t root = (vertexId_t)atoi(argv[2]);
  const char* prefix = argv[3];

  cuStinger cs(defaultInitAllocater, defaultUpdateAllocater);
  cuStingerInitConfig cfg;
  cfg.initState = eInitStateCSR;
  cfg.maxNV = nv + 1;
  cfg.csrNV = nv;
  cfg.csrNE = ne;
  cfg.csrOff = off;
  cfg.csrAdj = adj;
  cs.initializeCuStinger(cfg);

  run_bfs<bfsTD>(cs, root, prefix, "bfs_td", "bfs_top_down");
  run_bfs<bfsBU>(cs, root, prefix, "bfs_bu", "bfs_bottom_up");
  run_bfs<bfsHybrid>(cs, root, prefix, "bfs_hy", "bfs_hybrid");
  run_cc<CcBase>(cs, prefix, "cc_base", "cc_baseline");
  run_cc<CcConc>(cs, prefix, "cc_conc", "cc_concurrent");
  run_cc<CcLb>(cs, prefix, "cc_lb", "cc_load_balanced");

  StaticPageRank pr;
  pr.Init(cs);
  pr.setInputParameters(20, 0.001f, 0.85f);
  pr.Run(cs);
  prType* scores = pr.getPageRankScoresHost();
  char path[4096];
  snprintf(path, sizeof(path), "%s.pr", prefix);
  FILE* f = fopen(path, "wb");
  fwrite(scores, sizeof(prType), nv, f);
  fclose(f);
  freeHostArray(scores);
  printf("pagerank iterations %d\n", (int)pr.getIterationCount());
  pr.Release();

  const cudaError_t e = cudaDeviceSynchronize();
  printf("status %s\n", cudaGetErrorString(e));
  cs.freecuStinger();
  free(off);
  free(adj);
  return e == cudaSuccess ? 0 : 3;
}
