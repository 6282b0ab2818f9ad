// The graph handle behind tc_graph* (the cuStinger-compatible dynamic graph).
#pragma once

#include "tc_internal.cuh"

namespace tc {
struct StreamWs;
void release_stream_ws(StreamWs* w);
}  // namespace tc

// Slack-managed adjacency: vertex v owns pool[start[v] .. start[v] + cap[v]); its first used[v]
// entries are its neighbours, strictly ascending. Capacities are multiples of 4 entries so
// every list starts on a 16-byte boundary. Lists that outgrow their capacity move to fresh
// space at the pool's top (pool_top); the pool is compacted when it runs out.
struct tc_graph {
  int device = -1;
  int32_t n = 0;
  int64_t m = 0;          // directed edges in use
  int64_t pool_cap = 0;   // slots allocated in pool
  int64_t pool_top = 0;   // first slot past every list's capacity
  int32_t slack_q10 = 0;  // per-list slack as a fraction of its degree, in 1/1024
  int64_t* start = nullptr;
  int32_t* used = nullptr;
  int32_t* cap = nullptr;
  int32_t* pool = nullptr;
  tc::Workspace ws;       // static-count workspace (oriented CSR etc.)
  unsigned long long* d_pool_top = nullptr;  // device bump pointer (authoritative)
  uint8_t* mark = nullptr;        // per-slot change marks, parallel to pool (streaming)
  tc::StreamWs* sw = nullptr;     // streaming workspace
  void* pv_scratch = nullptr;     // per-vertex sink when a batch call passes none
  uint64_t view_version = 0;      // bumped by every structural update
};

namespace tc {
// Slack capacity for a list of `len` entries.
__host__ __device__ inline int32_t slack_capacity(int32_t len, int32_t slack_q10) {
  int64_t c = (int64_t)len + (((int64_t)len * slack_q10 + 1023) >> 10);
  if (slack_q10 > 0 && c < 4) c = 4;
  c = (c + 3) & ~(int64_t)3;
  return (int32_t)c;
}
}  // namespace tc
