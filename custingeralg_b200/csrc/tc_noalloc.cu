// Static triangle count with no device allocation: the stateless raw-CSR count
// (tc_count_csr32) with its working memory in a fixed array of this library's own device
// memory instead of cudaMalloc'd buffers.
//
// Who needs it: callers that must not allocate device memory when they count. A process whose
// memory is owned by another allocator (a framework's caching pool that has taken the free
// device memory, so a cudaMalloc of its own would fail) or a service that reserves every byte of
// device memory at start-up; and latency-sensitive loops, where cudaMalloc and cudaFree can
// synchronise the device and stall the work of other streams. They still pass their own input
// CSR and output buffers.
//
// The array is sized for graphs of up to TC_NOALLOC_MAX_NV vertices and TC_NOALLOC_MAX_EDGES
// directed edges: about 48.6 MiB (51 MB, checked below), which every GPU that loads the library
// holds until the process exits. Larger graphs are rejected with TC_ERR_CAPACITY. All calls
// share the array and each starts by clearing the part that must start at zero (the status
// block); two calls that overlap on the GPU race and corrupt each other, so serialise them (one
// stream, or events). The first call on a device looks up the array's device address
// (cudaGetSymbolAddress) with that device current and keeps it for later calls. The edge count
// d_off[nv] is read back to the host, so every call synchronises `stream` once.
#include <cstring>
#include <mutex>

#include "tc_internal.cuh"

namespace tc {
namespace {

constexpr int64_t kMaxNv = TC_NOALLOC_MAX_NV;
constexpr int64_t kMaxEdges = TC_NOALLOC_MAX_EDGES;

constexpr int64_t kMaxHubs = kMaxEdges / kHubMin + 1;
constexpr int64_t kMaxChunks = kMaxEdges / kHubMin + kMaxEdges / kHubChunk + 2;

// Layout (bytes, each part 256-aligned): DevStatus | offp int64[maxnv+1] | dplus, degv
// int32[maxnv+1] | large, medium uint64[items] | hub_u, hub_base, hub_done int32[hubs]
// | hub_cnt, chunk_hub int32[chunks] | indp int32[max_edges + kIndpPad]
constexpr size_t align256(size_t x) { return (x + 255) & ~size_t(255); }
constexpr size_t kOffStatus = 0;
constexpr size_t kOffOffp = align256(kOffStatus + sizeof(DevStatus));
constexpr size_t kOffDplus = align256(kOffOffp + sizeof(int64_t) * (kMaxNv + 1));
constexpr int64_t kMaxItems = Workspace::items_for(kMaxNv, kMaxEdges);
constexpr size_t kOffDegv = align256(kOffDplus + sizeof(int32_t) * (kMaxNv + 1));
constexpr size_t kOffLarge = align256(kOffDegv + sizeof(int32_t) * (kMaxNv + 1));
constexpr size_t kOffMedium = align256(kOffLarge + sizeof(unsigned long long) * kMaxItems);
constexpr size_t kOffHubU = align256(kOffMedium + sizeof(unsigned long long) * kMaxItems);
constexpr size_t kOffHubBase = align256(kOffHubU + sizeof(int32_t) * kMaxHubs);
constexpr size_t kOffHubDone = align256(kOffHubBase + sizeof(int32_t) * kMaxHubs);
constexpr size_t kOffHubCnt = align256(kOffHubDone + sizeof(int32_t) * kMaxHubs);
constexpr size_t kOffChunkHub = align256(kOffHubCnt + sizeof(int32_t) * kMaxChunks);
constexpr size_t kOffIndp = align256(kOffChunkHub + sizeof(int32_t) * kMaxChunks);
constexpr size_t kScratchBytes = align256(kOffIndp + sizeof(int32_t) * (kMaxEdges + kIndpPad));
static_assert(kScratchBytes > (size_t(48) << 20) && kScratchBytes < (size_t(49) << 20),
              "the documented size of the no-alloc scratch (about 48.6 MiB) no longer holds");

static __device__ __align__(256) unsigned char g_noalloc_scratch[kScratchBytes];

struct DevScratch {
  std::mutex mu;
  unsigned char* ptr[64] = {};
};
DevScratch& dev_scratch() {
  static DevScratch* d = new DevScratch();
  return *d;
}

// Device address of the scratch array on the current device (looked up once per device).
tc_status scratch_address(unsigned char** out) {
  int dev = 0;
  TC_CUDA_TRY(cudaGetDevice(&dev));
  if (dev < 0 || dev >= 64) return fail(TC_ERR_INVALID_ARG, "device %d out of range", dev);
  DevScratch& d = dev_scratch();
  std::lock_guard<std::mutex> lk(d.mu);
  if (!d.ptr[dev]) {
    void* p = nullptr;
    const cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess || !p)
      return fail(TC_ERR_CUDA, "cudaGetSymbolAddress of the no-alloc scratch failed: %s", cudaGetErrorString(e));
    d.ptr[dev] = static_cast<unsigned char*>(p);
  }
  *out = d.ptr[dev];
  return TC_OK;
}

}  // namespace
}  // namespace tc

using namespace tc;

extern "C" tc_status tc_count_csr32_noalloc(int32_t nv, const int32_t* d_off, const int32_t* d_ind, int pv_mode,
                                            int32_t* per_vertex, int64_t* triangles_dev, tc_count_info* info,
                                            const tc_sched* sched, void* stream) {
  tc::TraceRange trace_range("tc_count_csr32_noalloc");
  if (nv < 0 || (nv > 0 && (!d_off || !d_ind))) return fail(TC_ERR_INVALID_ARG, "invalid CSR (nv=%d)", nv);
  if (sched && sched->nshards > 1)
    return fail(TC_ERR_INVALID_ARG, "no-alloc count: a sharded count needs working memory this entry point does not hold");
  if (pv_mode < TC_PV_NONE || pv_mode > TC_PV_HANDLE64) return fail(TC_ERR_INVALID_ARG, "unknown per-vertex mode %d", pv_mode);
  if (pv_mode != TC_PV_NONE && nv > 0 && !per_vertex)
    return fail(TC_ERR_INVALID_ARG, "per_vertex output required for mode %d", pv_mode);
  if ((int64_t)nv > kMaxNv)
    return fail(TC_ERR_CAPACITY, "no-alloc count: %d vertices exceed the fixed limit of %lld", nv, (long long)kMaxNv);
  cudaStream_t s = (cudaStream_t)stream;
  int32_t m = 0;
  if (nv > 0) {
    TC_CUDA_TRY(cudaMemcpyAsync(&m, d_off + nv, sizeof(int32_t), cudaMemcpyDeviceToHost, s));
    TC_CUDA_TRY(cudaStreamSynchronize(s));
  }
  if (m < 0) return fail(TC_ERR_BAD_GRAPH, "negative edge count");
  if ((int64_t)m > kMaxEdges)
    return fail(TC_ERR_CAPACITY, "no-alloc count: %d directed edges exceed the fixed limit of %lld", m,
                (long long)kMaxEdges);
  unsigned char* base = nullptr;
  TC_TRY(scratch_address(&base));
  // A workspace view onto the fixed array; nothing is allocated or freed.
  Workspace ws;
  ws.device = -1;
  ws.n_cap = kMaxNv + 1;
  ws.e_cap = kMaxEdges;
  ws.st = reinterpret_cast<DevStatus*>(base + kOffStatus);
  ws.offp = reinterpret_cast<int64_t*>(base + kOffOffp);
  ws.dplus = reinterpret_cast<int32_t*>(base + kOffDplus);
  ws.degv = reinterpret_cast<int32_t*>(base + kOffDegv);
  ws.large = reinterpret_cast<unsigned long long*>(base + kOffLarge);
  ws.medium = reinterpret_cast<unsigned long long*>(base + kOffMedium);
  ws.item_cap = kMaxItems;
  ws.hub_u = reinterpret_cast<int32_t*>(base + kOffHubU);
  ws.hub_base = reinterpret_cast<int32_t*>(base + kOffHubBase);
  ws.hub_done = reinterpret_cast<int32_t*>(base + kOffHubDone);
  ws.hub_cnt = reinterpret_cast<int32_t*>(base + kOffHubCnt);
  ws.chunk_hub = reinterpret_cast<int32_t*>(base + kOffChunkHub);
  ws.hub_cap = kMaxHubs;
  ws.chunk_cap = kMaxChunks;
  ws.indp = reinterpret_cast<int32_t*>(base + kOffIndp);
  Csr32View view{d_off, d_ind};
  // static_count clears the status word (the only scratch that must start at zero) itself.
  TC_TRY(static_count(view, nv, (int64_t)m, ws, pv_mode, per_vertex, triangles_dev, to_params(sched), s));
  if (info) return read_info(ws, s, info);
  return TC_OK;
}
