// Graph handle: creation from a CSR, export, validation and the static count entry point.
#include <algorithm>
#include <cmath>
#include <cstring>

#include "tc_graph.cuh"

namespace tc {
namespace {

__global__ void k_init_caps(const int32_t n, const int64_t* __restrict__ off, int32_t* __restrict__ used,
                            int32_t* __restrict__ cap, const int32_t slack_q10, unsigned* __restrict__ bad) {
  for (int64_t v = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; v < n; v += (int64_t)gridDim.x * blockDim.x) {
    const int64_t len = off[v + 1] - off[v];
    if (len < 0 || len > INT32_MAX / 2) {
      atomicOr(bad, 1u);
      used[v] = 0;
      cap[v] = 0;
      continue;
    }
    used[v] = (int32_t)len;
    cap[v] = slack_capacity((int32_t)len, slack_q10);
  }
}

// One warp per vertex: copy its list from the CSR into its pool slot.
__global__ void k_copy_lists(const int32_t n, const int64_t* __restrict__ off, const int32_t* __restrict__ ind,
                             const int64_t* __restrict__ start, const int32_t* __restrict__ used,
                             int32_t* __restrict__ pool) {
  const int lane = threadIdx.x & 31;
  const int64_t gw = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int64_t nw = ((int64_t)gridDim.x * blockDim.x) >> 5;
  for (int64_t v = gw; v < n; v += nw) {
    const int64_t s = off[v], d = start[v];
    const int32_t len = used[v];
    for (int32_t k = lane; k < len; k += 32) pool[d + k] = ind[s + k];
  }
}

// One warp per vertex: gather the used prefix of each list into a compact CSR.
__global__ void k_gather_lists(const int32_t n, const int64_t* __restrict__ start, const int32_t* __restrict__ used,
                               const int32_t* __restrict__ pool, const int64_t* __restrict__ coff,
                               int32_t* __restrict__ cind) {
  const int lane = threadIdx.x & 31;
  const int64_t gw = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int64_t nw = ((int64_t)gridDim.x * blockDim.x) >> 5;
  for (int64_t v = gw; v < n; v += nw) {
    const int64_t s = start[v], d = coff[v];
    const int32_t len = used[v];
    for (int32_t k = lane; k < len; k += 32) cind[d + k] = pool[s + k];
  }
}

int warp_grid(int64_t n) {
  const int64_t want = (n + 7) / 8;
  return (int)std::max<int64_t>(1, std::min<int64_t>(want, (int64_t)device_info().sms * 16));
}

void free_graph(tc_graph* g) {
  if (!g) return;
  cudaFree(g->start);
  cudaFree(g->used);
  cudaFree(g->cap);
  cudaFree(g->pool);
  cudaFree(g->d_pool_top);
  cudaFree(g->mark);
  cudaFree(g->pv_scratch);
  release_stream_ws(g->sw);
  g->sw = nullptr;
  g->ws.release();
}

}  // namespace
}  // namespace tc

using namespace tc;

extern "C" {

tc_status tc_graph_create(int32_t nv, const int64_t* off, const int32_t* ind, int mem, double slack, int validate,
                          void* stream, tc_graph** out) {
  if (!out) return fail(TC_ERR_INVALID_ARG, "out is NULL");
  *out = nullptr;
  if (nv < 0 || !off || (mem != TC_MEM_HOST && mem != TC_MEM_DEVICE) || !(slack >= 0.0) || slack > 64.0)
    return fail(TC_ERR_INVALID_ARG, "invalid graph arguments");
  cudaStream_t s = (cudaStream_t)stream;
  int64_t m = 0;
  if (mem == TC_MEM_HOST) {
    m = off[nv];
    if (off[0] != 0) return fail(TC_ERR_INVALID_ARG, "off[0] must be 0");
  } else {
    int64_t h[2] = {0, 0};
    TC_CUDA_TRY(cudaMemcpyAsync(&h[0], off, sizeof(int64_t), cudaMemcpyDeviceToHost, s));
    TC_CUDA_TRY(cudaMemcpyAsync(&h[1], off + nv, sizeof(int64_t), cudaMemcpyDeviceToHost, s));
    TC_CUDA_TRY(cudaStreamSynchronize(s));
    if (h[0] != 0) return fail(TC_ERR_INVALID_ARG, "off[0] must be 0");
    m = h[1];
  }
  if (m < 0 || (m > 0 && !ind)) return fail(TC_ERR_INVALID_ARG, "invalid edge array");

  tc_graph* g = new tc_graph();
  int64_t* t_off = nullptr;
  int32_t* t_ind = nullptr;
  unsigned* d_bad = nullptr;
  int64_t* tiles = nullptr;
  auto free_tmp = [&]() {
    cudaFree(t_off);
    cudaFree(t_ind);
    cudaFree(d_bad);
    cudaFree(tiles);
    t_off = nullptr;
    t_ind = nullptr;
    d_bad = nullptr;
    tiles = nullptr;
  };
  auto bail = [&](tc_status st) {
    free_tmp();
    free_graph(g);
    delete g;
    return st;
  };
#define G_TRY(call)                                                                                          \
  do {                                                                                                       \
    cudaError_t _e = (call);                                                                                 \
    if (_e != cudaSuccess) {                                                                                 \
      fail(_e == cudaErrorMemoryAllocation ? TC_ERR_OOM : TC_ERR_CUDA, "%s: %s", #call, cudaGetErrorString(_e)); \
      return bail(_e == cudaErrorMemoryAllocation ? TC_ERR_OOM : TC_ERR_CUDA);                               \
    }                                                                                                        \
  } while (0)
  G_TRY(cudaGetDevice(&g->device));
  g->n = nv;
  g->m = m;
  g->slack_q10 = (int32_t)std::lround(slack * 1024.0);

  const int64_t* d_off = off;
  const int32_t* d_ind = ind;
  if (mem == TC_MEM_HOST) {
    G_TRY(::tc::dev_malloc(&t_off, sizeof(int64_t) * ((size_t)nv + 1)));
    G_TRY(::tc::dev_malloc(&t_ind, sizeof(int32_t) * (size_t)std::max<int64_t>(m, 1)));
    G_TRY(cudaMemcpyAsync(t_off, off, sizeof(int64_t) * ((size_t)nv + 1), cudaMemcpyHostToDevice, s));
    if (m) G_TRY(cudaMemcpyAsync(t_ind, ind, sizeof(int32_t) * (size_t)m, cudaMemcpyHostToDevice, s));
    d_off = t_off;
    d_ind = t_ind;
  }
  G_TRY(::tc::dev_malloc(&g->start, sizeof(int64_t) * ((size_t)nv + 1)));
  G_TRY(::tc::dev_malloc(&g->used, sizeof(int32_t) * (size_t)std::max(nv, 1)));
  G_TRY(::tc::dev_malloc(&g->cap, sizeof(int32_t) * (size_t)std::max(nv, 1)));
  G_TRY(::tc::dev_malloc(&d_bad, sizeof(unsigned)));
  G_TRY(::tc::dev_malloc(&tiles, sizeof(int64_t) * (size_t)(scan_tiles(nv) + 1)));
  G_TRY(cudaMemsetAsync(d_bad, 0, sizeof(unsigned), s));
  if (nv > 0) {
    k_init_caps<<<warp_grid(nv), 256, 0, s>>>(nv, d_off, g->used, g->cap, g->slack_q10, d_bad);
    G_TRY(cudaGetLastError());
  }
  {
    tc_status st = scan_counts(g->cap, nv, g->start, tiles, s);
    if (st != TC_OK) {
      free_tmp();
      return bail(st);
    }
  }
  int64_t top = 0;
  unsigned bad = 0;
  G_TRY(cudaMemcpyAsync(&top, g->start + nv, sizeof(int64_t), cudaMemcpyDeviceToHost, s));
  G_TRY(cudaMemcpyAsync(&bad, d_bad, sizeof(unsigned), cudaMemcpyDeviceToHost, s));
  G_TRY(cudaStreamSynchronize(s));
  if (bad) {
    free_tmp();
    fail(TC_ERR_BAD_GRAPH, "offsets not non-decreasing or a list too long");
    return bail(TC_ERR_BAD_GRAPH);
  }
  g->pool_top = top;
  // Headroom for lists that move when they outgrow their slack.
  g->pool_cap = top + (g->slack_q10 > 0 ? std::max<int64_t>(top / 4, 1 << 16) : 0);
  G_TRY(::tc::dev_malloc(&g->pool, sizeof(int32_t) * (size_t)std::max<int64_t>(g->pool_cap, 1)));
  G_TRY(::tc::dev_malloc(&g->d_pool_top, sizeof(unsigned long long)));
  G_TRY(cudaMemcpyAsync(g->d_pool_top, &g->pool_top, sizeof(unsigned long long), cudaMemcpyHostToDevice, s));
  if (nv > 0) {
    k_copy_lists<<<warp_grid(nv), 256, 0, s>>>(nv, d_off, d_ind, g->start, g->used, g->pool);
    G_TRY(cudaGetLastError());
  }
  G_TRY(cudaStreamSynchronize(s));
  free_tmp();
#undef G_TRY
  if (validate) {
    tc_status st = tc_graph_validate(g, stream);
    if (st != TC_OK) {
      std::string msg = tc_last_error();
      free_graph(g);
      delete g;
      fail(st, "%s", msg.c_str());
      return st;
    }
  }
  *out = g;
  return TC_OK;
}

tc_status tc_graph_destroy(tc_graph* g) {
  if (!g) return TC_OK;
  int cur = 0;
  cudaGetDevice(&cur);
  if (g->device >= 0 && g->device != cur) cudaSetDevice(g->device);
  free_graph(g);
  if (g->device >= 0 && g->device != cur) cudaSetDevice(cur);
  delete g;
  return TC_OK;
}

tc_status tc_graph_info(const tc_graph* g, int32_t* nv, int64_t* edges_used, int64_t* edges_alloc) {
  if (!g) return fail(TC_ERR_INVALID_ARG, "graph is NULL");
  if (nv) *nv = g->n;
  if (edges_used) *edges_used = g->m;
  if (edges_alloc) *edges_alloc = g->pool_top;
  return TC_OK;
}

tc_status tc_graph_device_view(tc_graph* g, const int64_t** start, const int32_t** used, const int32_t** pool) {
  if (!g) return fail(TC_ERR_INVALID_ARG, "graph is NULL");
  if (start) *start = g->start;
  if (used) *used = g->used;
  if (pool) *pool = g->pool;
  return TC_OK;
}

tc_status tc_graph_export(tc_graph* g, int64_t* off_host, int32_t* ind_host) {
  if (!g || !off_host) return fail(TC_ERR_INVALID_ARG, "invalid export arguments");
  const int32_t n = g->n;
  int64_t* coff = nullptr;
  int32_t* cind = nullptr;
  int64_t* tiles = nullptr;
  tc_status rc = TC_OK;
  do {
    if (::tc::dev_malloc(&coff, sizeof(int64_t) * ((size_t)n + 1)) != cudaSuccess ||
        ::tc::dev_malloc(&cind, sizeof(int32_t) * (size_t)std::max<int64_t>(g->m, 1)) != cudaSuccess ||
        ::tc::dev_malloc(&tiles, sizeof(int64_t) * (size_t)(scan_tiles(n) + 1)) != cudaSuccess) {
      rc = fail(TC_ERR_OOM, "export: allocation failed");
      break;
    }
    rc = scan_counts(g->used, n, coff, tiles, 0);
    if (rc != TC_OK) break;
    if (n > 0) k_gather_lists<<<warp_grid(n), 256>>>(n, g->start, g->used, g->pool, coff, cind);
    if (cudaMemcpy(off_host, coff, sizeof(int64_t) * ((size_t)n + 1), cudaMemcpyDeviceToHost) != cudaSuccess) {
      rc = fail(TC_ERR_CUDA, "export: copy failed: %s", cudaGetErrorString(cudaGetLastError()));
      break;
    }
    if (off_host[n] != g->m) {
      rc = fail(TC_ERR_STATE, "export: edge count mismatch (%lld vs %lld)", (long long)off_host[n], (long long)g->m);
      break;
    }
    if (ind_host && g->m &&
        cudaMemcpy(ind_host, cind, sizeof(int32_t) * (size_t)g->m, cudaMemcpyDeviceToHost) != cudaSuccess) {
      rc = fail(TC_ERR_CUDA, "export: copy failed");
      break;
    }
  } while (0);
  cudaFree(coff);
  cudaFree(cind);
  cudaFree(tiles);
  return rc;
}

tc_status tc_graph_validate(tc_graph* g, void* stream) {
  if (!g) return fail(TC_ERR_INVALID_ARG, "graph is NULL");
  cudaStream_t s = (cudaStream_t)stream;
  TC_TRY(g->ws.ensure(g->n, g->m, g->pool_cap));
  SlackView view{g->start, g->used, g->pool};
  TC_TRY(validate_view(view, g->n, g->ws, s));
  tc_count_info info;
  return read_info(g->ws, s, &info);
}

tc_status tc_count_static(tc_graph* g, int pv_mode, int32_t* per_vertex, int64_t* triangles_dev, tc_count_info* info,
                          const tc_sched* sched, void* stream) {
  tc::TraceRange trace_range("tc_count_static");
  if (!g) return fail(TC_ERR_INVALID_ARG, "graph is NULL");
  if (pv_mode < TC_PV_NONE || pv_mode > TC_PV_HANDLE64) return fail(TC_ERR_INVALID_ARG, "unknown per-vertex mode %d", pv_mode);
  if (pv_mode != TC_PV_NONE && g->n > 0 && !per_vertex)
    return fail(TC_ERR_INVALID_ARG, "per_vertex output required for mode %d", pv_mode);
  cudaStream_t s = (cudaStream_t)stream;
#ifdef TC_DEBUG_PROGRESS
  extern volatile int tc_dbg_host_stage;
  tc_dbg_host_stage = 201;
#endif
  TC_TRY(g->ws.ensure(g->n, g->m, g->pool_cap));
  SlackView view{g->start, g->used, g->pool};
  TC_TRY(static_count(view, g->n, g->m, g->ws, pv_mode, per_vertex, triangles_dev, to_params(sched), s));
#ifdef TC_DEBUG_PROGRESS
  tc_dbg_host_stage = 202;
#endif
  if (info) return read_info(g->ws, s, info);
  return TC_OK;
}

}  // extern "C"

extern "C" tc_status tc_cell_stats(tc_graph* g, double* out_host, void* stream) {
  if (!g || !out_host) return fail(TC_ERR_INVALID_ARG, "invalid arguments");
  tc_sched none;
  tc_sched_default(&none);
  none.cell_filter = -2;  // build the orientation, intersect nothing
  TC_TRY(tc_count_static(g, TC_PV_NONE, nullptr, nullptr, nullptr, &none, stream));
  return cell_stats(g->n, g->ws, out_host, (cudaStream_t)stream);
}
