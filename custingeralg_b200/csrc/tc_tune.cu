// Autotuner for the static count: times candidate scheduler settings on the graph with CUDA
// events and keeps the fastest. Results are cached per graph-statistics bucket
// (log2 n, log2 m, log2 of the largest out-degree) so similar graphs reuse them; the cache can be
// saved to and loaded from a small text file.
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <map>
#include <mutex>
#include <string>
#include <tuple>
#include <vector>

#include "tc_graph.cuh"

namespace tc {
namespace {

using Key = std::tuple<int, int, int>;

struct TuneCache {
  std::mutex mu;
  std::map<Key, tc_sched> entries;
};

TuneCache& cache() {
  static TuneCache* c = new TuneCache();
  return *c;
}

int ilog2(int64_t x) {
  int r = 0;
  while (x > 1) {
    x >>= 1;
    ++r;
  }
  return r;
}

std::vector<tc_sched> candidates() {
  std::vector<tc_sched> out;
  const int warp_max[] = {32, 64, 128};
  // (lane_max, packed_max): lists up to lane_max walked by a lane, up to packed_max packed
  const int list_rule[][2] = {{8, 0}, {0, 64}, {4, 32}, {8, 32}, {16, 128}};
  const int chunk[] = {32, 128};
  const int bps[] = {0, 6};
  for (int w : warp_max)
    for (const auto& r : list_rule)
      for (int c : chunk)
        for (int b : bps) {
          tc_sched s;
          tc_sched_default(&s);
          s.warp_max_deg = w;
          s.lane_max_deg = r[0];
          s.packed_max_deg = r[1];
          s.chunk = c;
          s.blocks_per_sm = b;
          out.push_back(s);
        }
  return out;
}

}  // namespace
}  // namespace tc

using namespace tc;

extern "C" {

tc_status tc_autotune_static(tc_graph* g, int pv_mode, int32_t* per_vertex, int32_t reps, tc_sched* best,
                             float* best_ms, void* stream) {
  if (!g || !best || reps < 1) return fail(TC_ERR_INVALID_ARG, "invalid autotune arguments");
  if (pv_mode != TC_PV_NONE && g->n > 0 && !per_vertex) return fail(TC_ERR_INVALID_ARG, "per_vertex required");
  cudaStream_t s = (cudaStream_t)stream;
  tc_count_info info;
  TC_TRY(tc_count_static(g, pv_mode, per_vertex, nullptr, &info, nullptr, stream));
  const Key key{ilog2(std::max(g->n, 1)), ilog2(std::max<int64_t>(g->m, 1)), ilog2(std::max(info.max_out_degree, 1))};
  cudaEvent_t e0, e1;
  TC_CUDA_TRY(cudaEventCreate(&e0));
  TC_CUDA_TRY(cudaEventCreate(&e1));
  float bestt = 1e30f;
  tc_sched bests;
  tc_sched_default(&bests);
  for (const tc_sched& c : candidates()) {
    std::vector<float> t;
    for (int r = 0; r < reps + 1; ++r) {
      cudaEventRecord(e0, s);
      tc_status st = tc_count_static(g, pv_mode, per_vertex, nullptr, nullptr, &c, stream);
      cudaEventRecord(e1, s);
      if (st != TC_OK) {
        cudaEventDestroy(e0);
        cudaEventDestroy(e1);
        return st;
      }
      TC_CUDA_TRY(cudaEventSynchronize(e1));
      float ms = 0.f;
      cudaEventElapsedTime(&ms, e0, e1);
      if (r > 0) t.push_back(ms);  // first run warms the caches
    }
    std::sort(t.begin(), t.end());
    const float med = t[t.size() / 2];
    if (med < bestt) {
      bestt = med;
      bests = c;
    }
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  *best = bests;
  if (best_ms) *best_ms = bestt;
  {
    std::lock_guard<std::mutex> lk(cache().mu);
    cache().entries[key] = bests;
  }
  return TC_OK;
}

tc_status tc_autotune_lookup(int32_t nv, int64_t edges, int32_t max_out_degree, tc_sched* out) {
  if (!out) return fail(TC_ERR_INVALID_ARG, "out is NULL");
  const Key key{ilog2(std::max(nv, 1)), ilog2(std::max<int64_t>(edges, 1)), ilog2(std::max(max_out_degree, 1))};
  std::lock_guard<std::mutex> lk(cache().mu);
  auto it = cache().entries.find(key);
  if (it == cache().entries.end()) {
    tc_sched_default(out);
    return fail(TC_ERR_STATE, "no tuned entry for this graph bucket");
  }
  *out = it->second;
  return TC_OK;
}

tc_status tc_autotune_save(const char* path) {
  if (!path) return fail(TC_ERR_INVALID_ARG, "path is NULL");
  FILE* f = fopen(path, "w");
  if (!f) return fail(TC_ERR_INVALID_ARG, "cannot write %s", path);
  std::lock_guard<std::mutex> lk(cache().mu);
  fprintf(f, "# tc autotune v3: log2n log2m log2maxdplus warp_max lane_max chunk blocks_per_sm packed_max\n");
  for (const auto& kv : cache().entries) {
    const tc_sched& s = kv.second;
    fprintf(f, "%d %d %d %d %d %d %d %d\n", std::get<0>(kv.first), std::get<1>(kv.first), std::get<2>(kv.first),
            s.warp_max_deg, s.lane_max_deg, s.chunk, s.blocks_per_sm, s.packed_max_deg);
  }
  fclose(f);
  return TC_OK;
}

tc_status tc_autotune_load(const char* path) {
  if (!path) return fail(TC_ERR_INVALID_ARG, "path is NULL");
  FILE* f = fopen(path, "r");
  if (!f) return fail(TC_ERR_INVALID_ARG, "cannot read %s", path);
  char line[512];
  int loaded = 0;
  std::lock_guard<std::mutex> lk(cache().mu);
  while (fgets(line, sizeof(line), f)) {
    if (line[0] == '#') continue;
    int a, b, c, w, r, ch, bp, pk = 0;
    // v3 lines carry packed_max last; v2 lines (7 fields) get no packed walks
    const int got = sscanf(line, "%d %d %d %d %d %d %d %d", &a, &b, &c, &w, &r, &ch, &bp, &pk);
    if (got == 7 || got == 8) {
      tc_sched s;
      tc_sched_default(&s);
      s.warp_max_deg = w;
      s.lane_max_deg = r;
      s.packed_max_deg = got == 8 ? pk : 0;
      s.chunk = ch;
      s.blocks_per_sm = bp;
      cache().entries[Key{a, b, c}] = s;
      ++loaded;
    }
  }
  fclose(f);
  return loaded > 0 ? TC_OK : fail(TC_ERR_INVALID_ARG, "no entries in %s", path);
}

}  // extern "C"
