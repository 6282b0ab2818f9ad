// C ABI (include/custinger_tc.h): graph handle, workspaces and static counts.
#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstdarg>
#include <cstring>
#include <mutex>
#include <string>

#include "tc_graph.cuh"
#include "tc_internal.cuh"

namespace tc {

namespace {
thread_local std::string g_last_error;

struct Prof {
  bool on = false;
  bool valid = false;
  int launches = 0;
  cudaEvent_t ev[3] = {nullptr, nullptr, nullptr};
};
thread_local Prof g_prof;
}  // namespace

namespace {
std::atomic<long long> g_alloc_cap{0};  // 0 = no cap
}  // namespace

cudaError_t dev_malloc_bytes(void** p, size_t bytes) {
  const long long cap = g_alloc_cap.load(std::memory_order_relaxed);
  if (cap > 0 && (long long)bytes > cap) {
    *p = nullptr;
    return cudaErrorMemoryAllocation;
  }
  return cudaMalloc(p, bytes);
}

void prof_mark(int point, cudaStream_t stream) {
  if (!g_prof.on || point < 0 || point > 2) return;
  if (!g_prof.ev[point] && cudaEventCreate(&g_prof.ev[point]) != cudaSuccess) return;
  cudaEventRecord(g_prof.ev[point], stream);
  g_prof.valid = (point == 2);
}

void prof_launches(int n) {
  if (g_prof.on) g_prof.launches = n;
}

void set_error(const char* fmt, ...) {
  char buf[1024];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(buf, sizeof(buf), fmt, ap);
  va_end(ap);
  g_last_error = buf;
}

tc_status fail(tc_status s, const char* fmt, ...) {
  char buf[1024];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(buf, sizeof(buf), fmt, ap);
  va_end(ap);
  g_last_error = buf;
  return s;
}

const DeviceInfo& device_info() {
  constexpr int kMaxDev = 64;
  static DeviceInfo infos[kMaxDev];
  static bool init[kMaxDev] = {};
  static std::mutex mu;
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDev) dev = 0;
  std::lock_guard<std::mutex> lk(mu);
  if (!init[dev]) {
    int sms = 0;
    if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) == cudaSuccess && sms > 0)
      infos[dev].sms = sms;
    init[dev] = true;
  }
  return infos[dev];
}

namespace {
template <typename T>
tc_status grow(T*& p, int64_t& cap, int64_t want) {
  if (p && cap >= want) return TC_OK;
  if (p) cudaFree(p);
  p = nullptr;
  cap = 0;
  const int64_t n = std::max<int64_t>(want, 1);
  const cudaError_t e = ::tc::dev_malloc(&p, sizeof(T) * (size_t)n);
  if (e != cudaSuccess) {
    p = nullptr;
    return fail(e == cudaErrorMemoryAllocation ? TC_ERR_OOM : TC_ERR_CUDA, "device allocation of %lld bytes: %s",
                (long long)(sizeof(T) * (size_t)n), cudaGetErrorString(e));
  }
  cap = n;
  return TC_OK;
}
}  // namespace

// Each group of arrays is (re)allocated together; a failed allocation leaves the group's
// capacity at 0 (every array of it freed or null), so the next call allocates it again and no
// kernel ever sees a freed or missing array.
tc_status Workspace::ensure(int64_t n, int64_t m, int64_t extent) {
  int dev = 0;
  TC_CUDA_TRY(cudaGetDevice(&dev));
  if (device >= 0 && device != dev) return fail(TC_ERR_INVALID_ARG, "workspace used on device %d, created on %d", dev, device);
  device = dev;
  if (n + 1 > n_cap) {
    n_cap = 0;
    int64_t c1 = 0, c2 = 0, c3 = 0;
    if (dplus) { cudaFree(dplus); dplus = nullptr; }
    if (offp) { cudaFree(offp); offp = nullptr; }
    if (degv) { cudaFree(degv); degv = nullptr; }
    TC_TRY(grow(dplus, c1, n + 1));
    TC_TRY(grow(offp, c2, n + 1));
    TC_TRY(grow(degv, c3, n + 1));
    n_cap = n + 1;
  }
  if (items_for(n, m) > item_cap) {
    item_cap = 0;
    int64_t c1 = 0, c2 = 0;
    if (medium) { cudaFree(medium); medium = nullptr; }
    if (large) { cudaFree(large); large = nullptr; }
    TC_TRY(grow(medium, c1, items_for(n, m)));
    TC_TRY(grow(large, c2, items_for(n, m)));
    item_cap = items_for(n, m);
  }
  TC_TRY(grow(indp, e_cap, std::max(m, extent) + kIndpPad));
  if (hubs_for(m) > hub_cap) {
    hub_cap = 0;
    int64_t c1 = 0, c2 = 0, c3 = 0;
    if (hub_base) { cudaFree(hub_base); hub_base = nullptr; }
    if (hub_done) { cudaFree(hub_done); hub_done = nullptr; }
    if (hub_u) { cudaFree(hub_u); hub_u = nullptr; }
    TC_TRY(grow(hub_base, c1, hubs_for(m)));
    TC_TRY(grow(hub_done, c2, hubs_for(m)));
    TC_TRY(grow(hub_u, c3, hubs_for(m)));
    hub_cap = hubs_for(m);
  }
  if (chunks_for(m) > chunk_cap) {
    chunk_cap = 0;
    int64_t c1 = 0, c2 = 0;
    if (chunk_hub) { cudaFree(chunk_hub); chunk_hub = nullptr; }
    if (hub_cnt) { cudaFree(hub_cnt); hub_cnt = nullptr; }
    TC_TRY(grow(hub_cnt, c1, chunks_for(m)));
    TC_TRY(grow(chunk_hub, c2, chunks_for(m)));
    chunk_cap = chunks_for(m);
  }
  if (!st && ::tc::dev_malloc(&st, sizeof(DevStatus)) != cudaSuccess) {
    st = nullptr;
    return fail(TC_ERR_OOM, "workspace status: device allocation failed");
  }
  return TC_OK;
}

tc_status Workspace::ensure_shards(int64_t n) {
  if (n + 1 <= shard_cap) return TC_OK;
  cudaFree(shard_cost);
  cudaFree(shard_prefix);
  cudaFree(shard_tiles);
  shard_cost = nullptr;
  shard_prefix = nullptr;
  shard_tiles = nullptr;
  shard_cap = 0;
  if (::tc::dev_malloc(&shard_cost, sizeof(int32_t) * (size_t)(n + 1)) != cudaSuccess ||
      ::tc::dev_malloc(&shard_prefix, sizeof(int64_t) * (size_t)(n + 2)) != cudaSuccess ||
      ::tc::dev_malloc(&shard_tiles, sizeof(int64_t) * (size_t)(scan_tiles(n + 1) + 1)) != cudaSuccess) {
    cudaFree(shard_cost);
    cudaFree(shard_prefix);
    cudaFree(shard_tiles);
    shard_cost = nullptr;
    shard_prefix = nullptr;
    shard_tiles = nullptr;
    return fail(TC_ERR_OOM, "shard workspace: device allocation failed");
  }
  shard_cap = n + 1;
  return TC_OK;
}

void Workspace::release() {
  cudaFree(shard_cost);
  cudaFree(shard_prefix);
  cudaFree(shard_tiles);
  cudaFree(dplus);
  cudaFree(offp);
  cudaFree(indp);
  cudaFree(degv);
  cudaFree(large);
  cudaFree(medium);
  cudaFree(hub_u);
  cudaFree(hub_base);
  cudaFree(hub_cnt);
  cudaFree(hub_done);
  cudaFree(chunk_hub);
  cudaFree(st);
  *this = Workspace();
}

namespace {
// Library-owned workspace for the stateless CSR entry points, one per device.
struct GlobalWs {
  std::mutex mu;
  Workspace ws[64];
};
GlobalWs& global_ws() {
  static GlobalWs* g = new GlobalWs();  // intentionally leaked: outlives CUDA teardown
  return *g;
}

#ifdef TC_DEBUG_PROGRESS
extern "C" volatile int tc_dbg_host_stage;
#define TC_DBG_STAGE(x) (tc_dbg_host_stage = (x))
#else
#define TC_DBG_STAGE(x) ((void)0)
#endif

template <class View, typename OffT>
tc_status count_csr(int32_t nv, const OffT* d_off, const int32_t* d_ind, int pv_mode, int32_t* per_vertex,
                    int64_t* triangles_dev, tc_count_info* info, const tc_sched* sched, void* stream) {
  if (nv < 0 || (nv > 0 && (!d_off || !d_ind)))
    return fail(TC_ERR_INVALID_ARG, "invalid CSR (nv=%d)", nv);
  if (pv_mode != TC_PV_NONE && nv > 0 && !per_vertex)
    return fail(TC_ERR_INVALID_ARG, "per_vertex output required for mode %d", pv_mode);
  if (pv_mode < TC_PV_NONE || pv_mode > TC_PV_HANDLE64) return fail(TC_ERR_INVALID_ARG, "unknown per-vertex mode %d", pv_mode);
  cudaStream_t s = (cudaStream_t)stream;
  int dev = 0;
  TC_CUDA_TRY(cudaGetDevice(&dev));
  if (dev < 0 || dev >= 64) return fail(TC_ERR_INVALID_ARG, "device %d out of range", dev);
  OffT m_h = 0;
  TC_DBG_STAGE(101);
  if (nv > 0) {
    TC_CUDA_TRY(cudaMemcpyAsync(&m_h, d_off + nv, sizeof(OffT), cudaMemcpyDeviceToHost, s));
    TC_CUDA_TRY(cudaStreamSynchronize(s));
  }
  TC_DBG_STAGE(102);
  if (m_h < 0) return fail(TC_ERR_BAD_GRAPH, "negative edge count");
  GlobalWs& g = global_ws();
  std::lock_guard<std::mutex> lk(g.mu);
  Workspace& ws = g.ws[dev];
  TC_TRY(ws.ensure(nv, (int64_t)m_h));
  View view{d_off, d_ind};
  TC_DBG_STAGE(103);
  TC_TRY(static_count(view, nv, (int64_t)m_h, ws, pv_mode, per_vertex, triangles_dev, to_params(sched), s));
  TC_DBG_STAGE(104);
  if (info) {
    tc_status r = read_info(ws, s, info);
    TC_DBG_STAGE(105);
    return r;
  }
  return TC_OK;
}
}  // namespace

}  // namespace tc

// ============================================================================================
// C ABI
// ============================================================================================

using namespace tc;

extern "C" {

const char* tc_last_error(void) { return g_last_error.c_str(); }

const char* tc_status_string(tc_status s) {
  switch (s) {
    case TC_OK: return "ok";
    case TC_ERR_INVALID_ARG: return "invalid argument";
    case TC_ERR_CUDA: return "CUDA error";
    case TC_ERR_OOM: return "out of device memory";
    case TC_ERR_BAD_GRAPH: return "graph not sorted/deduplicated, has self-loops or ids out of range";
    case TC_ERR_NOT_SYMMETRIC: return "graph not symmetric";
    case TC_ERR_CAPACITY: return "capacity exceeded";
    case TC_ERR_TIMEOUT: return "device wait timed out";
    case TC_ERR_STATE: return "call out of order";
    default: return "unknown status";
  }
}

void tc_sched_default(tc_sched* s) {
  if (!s) return;
  memset(s, 0, sizeof(*s));
  s->warp_max_deg = 64;      // centre out-degree up to which one warp counts it alone
  s->search_ratio_x16 = 16;  // streaming: search when d_long > d_short (log2 d_long + 1)
  s->lane_max_deg = 8;       // static: one lane walks each list of at most 8 entries
  s->packed_max_deg = 32;    // static: longer lists up to 32 entries walked packed
  s->blocks_per_sm = 0;
  s->chunk = 64;
  s->use_table = 0;
  s->shard = 0;
  s->nshards = 1;
  s->cell_filter = -1;
  s->stream_hub_min = 8;     // streaming: count at an endpoint holding >= 8 of a phase's changed edges
}

tc_status tc_count_csr32(int32_t nv, const int32_t* d_off, const int32_t* d_ind, int pv_mode, int32_t* per_vertex,
                         int64_t* triangles_dev, tc_count_info* info, const tc_sched* sched, void* stream) {
  tc::TraceRange trace_range("tc_count_csr32");
  return count_csr<Csr32View>(nv, d_off, d_ind, pv_mode, per_vertex, triangles_dev, info, sched, stream);
}

tc_status tc_count_csr64(int32_t nv, const int64_t* d_off, const int32_t* d_ind, int pv_mode, int32_t* per_vertex,
                         int64_t* triangles_dev, tc_count_info* info, const tc_sched* sched, void* stream) {
  tc::TraceRange trace_range("tc_count_csr64");
  return count_csr<Csr64View>(nv, d_off, d_ind, pv_mode, per_vertex, triangles_dev, info, sched, stream);
}

tc_status tc_debug_alloc_cap(int64_t bytes) {
  if (bytes < 0) return fail(TC_ERR_INVALID_ARG, "negative allocation cap");
  g_alloc_cap.store((long long)bytes, std::memory_order_relaxed);
  return TC_OK;
}

tc_status tc_shard_ranges(const int64_t* prefix_host, int32_t n, int32_t nshards, int32_t* lo_host) {
  if (!prefix_host || !lo_host || n < 0 || nshards < 1) return fail(TC_ERR_INVALID_ARG, "invalid shard arguments");
  for (int32_t r = 0; r <= nshards; ++r) lo_host[r] = shard_start(prefix_host, n, r, nshards);
  return TC_OK;
}

tc_status tc_profile_enable(int on) {
  g_prof.on = on != 0;
  g_prof.valid = false;
  return TC_OK;
}

tc_status tc_profile_last(tc_phase_times* t) {
  if (!t) return fail(TC_ERR_INVALID_ARG, "t is NULL");
  if (!g_prof.valid) return fail(TC_ERR_STATE, "no profiled count on this thread");
  TC_CUDA_TRY(cudaEventSynchronize(g_prof.ev[2]));
  TC_CUDA_TRY(cudaEventElapsedTime(&t->orient_ms, g_prof.ev[0], g_prof.ev[1]));
  TC_CUDA_TRY(cudaEventElapsedTime(&t->count_ms, g_prof.ev[1], g_prof.ev[2]));
  t->launches = g_prof.launches;
  return TC_OK;
}

tc_status tc_workspace_release(void) {
  int dev = 0;
  TC_CUDA_TRY(cudaGetDevice(&dev));
  if (dev < 0 || dev >= 64) return fail(TC_ERR_INVALID_ARG, "device %d out of range", dev);
  GlobalWs& g = global_ws();
  std::lock_guard<std::mutex> lk(g.mu);
  TC_CUDA_TRY(cudaDeviceSynchronize());  // no count may still use it
  g.ws[dev].release();
  return TC_OK;
}

tc_status tc_workspace_status(void* stream, tc_count_info* info) {
  if (!info) return fail(TC_ERR_INVALID_ARG, "info is NULL");
  int dev = 0;
  TC_CUDA_TRY(cudaGetDevice(&dev));
  if (dev < 0 || dev >= 64) return fail(TC_ERR_INVALID_ARG, "device %d out of range", dev);
  GlobalWs& g = global_ws();
  std::lock_guard<std::mutex> lk(g.mu);
  if (!g.ws[dev].st) return fail(TC_ERR_STATE, "no count has run on device %d", dev);
  return read_info(g.ws[dev], (cudaStream_t)stream, info);
}

}  // extern "C"
