// Internal declarations shared by the library's translation units.
#pragma once

#include <cuda_runtime.h>
#include <cstdint>
#include <cstdio>
#include <string>

#include <nvtx3/nvToolsExt.h>

#include "../../include/custinger_tc.h"

namespace tc {

// A named NVTX range over a scope: the public entry points mark themselves on the timelines of
// tools such as Nsight Systems; with no tool attached the calls return at once.
struct TraceRange {
  explicit TraceRange(const char* name) { nvtxRangePushA(name); }
  ~TraceRange() { nvtxRangePop(); }
  TraceRange(const TraceRange&) = delete;
  TraceRange& operator=(const TraceRange&) = delete;
};

constexpr int kWarp = 32;
constexpr unsigned kFull = 0xffffffffu;
constexpr int kHubChunk = 2048;     // orientation: list entries per warp work item of a hub
constexpr int kHubMin = 256;        // orientation: lists longer than this are oriented as hubs
static_assert(kHubMin <= kHubChunk, "a hub has at least one chunk");
constexpr int kWarpTierMax = 128;   // largest out-degree a single warp counts on its own
constexpr int kItemRangeMin = 256;  // fewest neighbours of a count work item (queue sizing)
// The count reads oriented lists in aligned 16-byte units, up to 3 entries past a list's end:
// every oriented-list array holds this many entries past its capacity.
constexpr int kIndpPad = 4;

// ---- error reporting -------------------------------------------------------------------

void set_error(const char* fmt, ...);
tc_status fail(tc_status s, const char* fmt, ...);

#define TC_CUDA_TRY(call)                                                                  \
  do {                                                                                     \
    cudaError_t _e = (call);                                                               \
    if (_e != cudaSuccess) {                                                               \
      return ::tc::fail(_e == cudaErrorMemoryAllocation ? TC_ERR_OOM : TC_ERR_CUDA,        \
                        "%s failed: %s (%s:%d)", #call, cudaGetErrorString(_e), __FILE__,  \
                        __LINE__);                                                         \
    }                                                                                      \
  } while (0)

// Every device allocation of the library goes through dev_malloc. A test hook
// (tc_debug_alloc_cap) makes allocations above a size fail the way cudaMalloc fails when device
// memory runs out (cudaErrorMemoryAllocation, nothing allocated), so the out-of-memory paths can
// be tested without exhausting a GPU.
cudaError_t dev_malloc_bytes(void** p, size_t bytes);
template <typename T>
inline cudaError_t dev_malloc(T** p, size_t bytes) {
  return dev_malloc_bytes(reinterpret_cast<void**>(p), bytes);
}

#define TC_TRY(expr)                  \
  do {                                \
    tc_status _s = (expr);            \
    if (_s != TC_OK) return _s;       \
  } while (0)

// ---- adjacency views -------------------------------------------------------------------
// The orientation kernels read the input graph through one of these: a compact CSR with
// int32 or int64 offsets (the reference's raw-CSR path) or the slack-managed handle storage
// (per-vertex start + used length into a pool, the cuStinger layout).

struct Csr32View {
  const int32_t* off;
  const int32_t* ind;
  __device__ __forceinline__ int64_t start(int32_t v) const { return off[v]; }
  __device__ __forceinline__ int32_t len(int32_t v) const { return off[v + 1] - off[v]; }
};

struct Csr64View {
  const int64_t* off;
  const int32_t* ind;
  __device__ __forceinline__ int64_t start(int32_t v) const { return off[v]; }
  __device__ __forceinline__ int32_t len(int32_t v) const { return (int32_t)(off[v + 1] - off[v]); }
};

struct SlackView {
  const int64_t* st;
  const int32_t* used;
  const int32_t* ind;
  __device__ __forceinline__ int64_t start(int32_t v) const { return st[v]; }
  __device__ __forceinline__ int32_t len(int32_t v) const { return used[v]; }
};

// ---- device-side status of one count ---------------------------------------------------

enum : unsigned { kBadRange = 1u, kBadOrder = 2u, kBadSelfLoop = 4u, kBadCapacity = 8u, kBadTimeout = 16u };

struct DevStatus {
  unsigned long long triangles;          // T
  unsigned long long edges_intersected;  // oriented edges with deg(u) >= 2
  unsigned long long oriented_work;      // sum over u->v with d+(u) >= 2 of d+(u) + d+(v)
  unsigned long long sym_checksum;       // signed edge checksum, 0 when symmetric
  unsigned long long q_small;            // work-queue head over vertex ids
  unsigned int bad_flags;
  unsigned int max_dplus;
  unsigned int n_large;                  // vertices on the CTA (large out-degree) queue
  unsigned int q_large;                  // work-queue head over the large list
  unsigned int n_medium;                 // vertices on the warp (medium out-degree) queue
  unsigned int q_medium;
  unsigned int n_hubs;                   // vertices whose list is split into chunks
  unsigned int n_hub_chunks;
  unsigned int q_orient_hub;             // orientation work-queue heads: hub chunks,
  unsigned int q_orient_vtx;             // vertex ids
  unsigned int cls_cnt[32];              // CTA-queue items per work class
  unsigned int cls_pos[32];              // and their fill cursors
  unsigned int sharded;                  // 1: count only centres in [shard_lo, shard_hi)
  unsigned int shard_lo, shard_hi;
  unsigned int pad0;
  unsigned long long shard_work;         // predicted work of this shard's centres (units of 16)
  unsigned long long total_work;         // and of all centres
};

// Multi-GPU split of the static count: shard r of N counts the edge centres c in
// [shard_start(r), shard_start(r + 1)), where prefix[c] is the exclusive prefix over the centres
// of their predicted work; shard r starts at the first centre whose prefix reaches r/N of the
// total. Host and device use this one function, so every rank derives the same ranges.
__host__ __device__ inline int32_t shard_start(const int64_t* prefix, int32_t n, int32_t r, int32_t nshards) {
  if (r <= 0) return 0;
  if (r >= nshards) return n;
  const int64_t total = prefix[n];
  const int64_t target = (total / nshards) * r + ((total % nshards) * r) / nshards;
  int32_t lo = 0, hi = n;  // first c in [0, n] with prefix[c] >= target
  while (lo < hi) {
    const int32_t mid = lo + (hi - lo) / 2;
    if (prefix[mid] < target) lo = mid + 1;
    else hi = mid;
  }
  return lo;
}

// ---- scheduler parameters as the kernels see them --------------------------------------

struct SchedParams {
  int32_t warp_max;        // <= kWarpTierMax
  int32_t search_ratio_x16;
  int32_t use_table;
  int32_t chunk;
  int32_t blocks_per_sm;   // 0 = occupancy limit
  int32_t shard;           // static: count the centres of range `shard` of `nshards` (shard_start);
  int32_t nshards;         // streaming: the changed edges whose key hashes to `shard` (edge_shard)
  int32_t cell_filter;     // -1 all edges, -2 none, >= 0 only that degree cell
  int32_t lane_max;        // static: lists of at most this many entries are walked by one lane
  int32_t packed_max;      // static: longer lists up to this many entries are walked packed
  int32_t hub_min;         // streaming: changed edges per longer endpoint for the hub count (0 = off)
  uint8_t table[16][16];
};

SchedParams to_params(const tc_sched* s);

// ---- workspace for one static count ----------------------------------------------------

struct Workspace {
  int device = -1;
  int64_t n_cap = 0;       // vertices
  int64_t e_cap = 0;       // oriented edge slots
  int32_t* dplus = nullptr;      // [n]
  int64_t* offp = nullptr;       // [n+1]
  int32_t* indp = nullptr;       // [e_cap] N+(u) at indp[start(u) ...] (the input's own index space)
  int32_t* degv = nullptr;       // [n] deg(u)
  unsigned long long* large = nullptr;   // [item_cap] count work items (centre << 32 | first neighbour)
  unsigned long long* medium = nullptr;  // [item_cap]
  int64_t item_cap = 0;
  int32_t* hub_u = nullptr;      // [hub_cap] vertices split into chunks
  int32_t* hub_base = nullptr;   // [hub_cap] their first chunk index
  int32_t* hub_cnt = nullptr;    // [chunk_cap] out-neighbours found per chunk
  int32_t* hub_done = nullptr;   // [hub_cap] chunks of each hub oriented so far
  int32_t* chunk_hub = nullptr;  // [chunk_cap] hub of each chunk
  int64_t hub_cap = 0;
  int64_t chunk_cap = 0;
  DevStatus* st = nullptr;       // [1]
  // multi-GPU split (allocated on the first sharded count): predicted work per centre (units of
  // 16 probes), its exclusive prefix and the scan's tile sums
  int32_t* shard_cost = nullptr;   // [shard_cap]
  int64_t* shard_prefix = nullptr; // [shard_cap + 1]
  int64_t* shard_tiles = nullptr;
  int64_t shard_cap = 0;
  // n vertices, m directed edges, lists inside [0, extent) of the input's index space.
  tc_status ensure(int64_t n, int64_t m_directed, int64_t extent = -1);
  tc_status ensure_shards(int64_t n);
  void release();
  // Hub arrays needed for a graph of m directed edges.
  static int64_t hubs_for(int64_t m) { return m / kHubMin + 1; }
  static int64_t chunks_for(int64_t m) { return m / kHubMin + m / kHubChunk + 2; }
  // Count work items of one queue: at most one per vertex plus one per kItemRangeMin neighbours.
  static constexpr int64_t items_for(int64_t n, int64_t m) { return n + m / kItemRangeMin + 1; }
};

// Device properties cached per device.
struct DeviceInfo {
  int sms = 148;
  int count_blocks_per_sm = 1;
};
const DeviceInfo& device_info();

// Static count over any view. `ws` must be sized for (n, m). Stream-ordered.
template <class View>
tc_status static_count(const View& view, int32_t n, int64_t m, Workspace& ws, int pv_mode,
                       int32_t* per_vertex, int64_t* triangles_dev, const SchedParams& sp,
                       cudaStream_t stream);

// Structural check only (the first orientation pass). Stream-ordered; read with read_info.
template <class View>
tc_status validate_view(const View& view, int32_t n, Workspace& ws, cudaStream_t stream);

// Phase events of the calling thread (tc_profile_enable). Each is a no-op when disabled.
void prof_mark(int point, cudaStream_t stream);   // 0 = start, 1 = orientation done, 2 = count done
void prof_launches(int n);

// Oriented-edge statistics per degree cell (needs the orientation in ws): 256 x 4 doubles.
tc_status cell_stats(int32_t n, Workspace& ws, double* out_host, cudaStream_t stream);

// Read back a count's info (syncs the stream).
tc_status read_info(const Workspace& ws, cudaStream_t stream, tc_count_info* info);

// Exclusive scan of int32 counts into int64 offsets: out[0..n] (out[n] = total).
tc_status scan_counts(const int32_t* in, int64_t n, int64_t* out, int64_t* tile_sums,
                      cudaStream_t stream);
int64_t scan_tiles(int64_t n);

}  // namespace tc
