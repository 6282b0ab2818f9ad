// load_balance.cuh - edge-balanced traversal for the operator library (the reference's
// include/load_balance.cuh, class cusLoadBalance: a vertex array, its work estimate and a
// partition of that work; built there on ModernGPU's scan and sorted search).
//
// Here the partition is per edge: the lengths of the lists of the vertices in the array are
// scanned (CUB) into an int64 prefix, and one thread takes each edge slot j of the concatenated
// lists; the slot's owner is the last vertex whose prefix is <= j (a binary search), so a
// 64k-entry hub list is spread over 64k threads instead of being one warp's serial loop. The
// total comes from the device; no host synchronisation happens inside a traversal.
#ifndef CUSTINGER_LOAD_BALANCE_CUH_
#define CUSTINGER_LOAD_BALANCE_CUH_

#include <cub/cub.cuh>

#include "algs.cuh"

namespace cuStingerAlgs {

namespace lb_detail {

constexpr int kThreads = 256;

inline int resident_blocks() {
  int dev = 0, sms = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  return (sms > 0 ? sms : 1) * 8;
}

inline int blocks_for(long long n) {
  const long long want = (n + kThreads - 1) / kThreads;
  const long long cap = resident_blocks();
  return (int)(want < 1 ? 1 : want < cap ? want : cap);
}

// len[i] = list length of arr[i] (of vertex i when arr is NULL); len[n] = 0 so that the scan
// leaves the total in prefix[n].
static __global__ void k_lengths(const cuStinger* cs, const vertexId_t* arr, length_t n, long long* len) {
  const length_t* used = cs->dVD->used;
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i <= n; i += (long long)gridDim.x * blockDim.x)
    len[i] = i < n ? (long long)used[arr ? arr[i] : (vertexId_t)i] : 0;
}

static __global__ void k_iota(vertexId_t* out, length_t n) {
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
    out[i] = (vertexId_t)i;
}

// The vertices with a non-empty list, in arrival order (one atomic per warp).
static __global__ void k_nonzero(const cuStinger* cs, length_t nv, vertexId_t* out, length_t* count) {
  const length_t* used = cs->dVD->used;
  const int lane = threadIdx.x & 31;
  for (long long b = (long long)blockIdx.x * blockDim.x; b < nv; b += (long long)gridDim.x * blockDim.x) {
    const long long v = b + threadIdx.x;
    const bool keep = v < nv && used[v] > 0;
    const unsigned m = __ballot_sync(0xffffffffu, keep);
    length_t at = 0;
    if (lane == 0 && m) at = atomicAdd(count, (length_t)__popc(m));
    at = __shfl_sync(0xffffffffu, at, 0);
    if (keep) out[at + __popc(m & ((1u << lane) - 1u))] = (vertexId_t)v;
  }
}

// One thread per edge slot j < prefix[n] of the concatenated lists of arr[0 .. n).
template <cusSubKernelEdge F>
static __global__ void k_edges(cuStinger* cs, void* metadata, const vertexId_t* arr, length_t n,
                               const long long* __restrict__ prefix) {
  const long long total = prefix[n];
  cusEdgeData** adj = cs->dVD->adj;
  for (long long j = (long long)blockIdx.x * blockDim.x + threadIdx.x; j < total;
       j += (long long)gridDim.x * blockDim.x) {
    long long lo = 0, hi = n;  // owner: the largest i with prefix[i] <= j (its list is non-empty)
    while (hi - lo > 1) {
      const long long mid = (lo + hi) >> 1;
      if (prefix[mid] <= j) lo = mid;
      else hi = mid;
    }
    const vertexId_t src = arr ? arr[lo] : (vertexId_t)lo;
    const vertexId_t dst = adj[src]->dst[j - prefix[lo]];
    (F)(cs, src, dst, metadata);
  }
}

}  // namespace lb_detail

class cusLoadBalance {
 public:
  // Workspace for traversals of arrays of up to maxArrayLen vertices (currArray left empty).
  explicit cusLoadBalance(length_t maxArrayLen) { reserve(maxArrayLen); }

  // currArray = every vertex (queueZeros) or the vertices with a non-empty list; the order of
  // the array does not change any traversal's result, so queueRandomly is accepted and ignored.
  cusLoadBalance(cuStinger& custing, bool queueZeros = true, bool queueRandomly = false) {
    (void)queueRandomly;
    const length_t nv = custing.nv;
    reserve(nv);
    internalAlloc_ = true;
    currArray = static_cast<vertexId_t*>(allocDeviceArray(nv + 1, sizeof(vertexId_t)));
    if (queueZeros) {
      lb_detail::k_iota<<<lb_detail::blocks_for(nv), lb_detail::kThreads>>>(currArray, nv);
      currArrayLen = nv;
    } else {
      length_t* d_count = static_cast<length_t*>(allocDeviceArray(1, sizeof(length_t)));
      cudaMemset(d_count, 0, sizeof(length_t));
      lb_detail::k_nonzero<<<lb_detail::blocks_for(nv), lb_detail::kThreads>>>(custing.devicePtr(), nv, currArray,
                                                                                  d_count);
      copyArrayDeviceToHost(d_count, &currArrayLen, 1, sizeof(length_t));
      freeDeviceArray(d_count);
    }
  }

  ~cusLoadBalance() {
    if (internalAlloc_) freeDeviceArray(currArray);
    freeDeviceArray(len_);
    freeDeviceArray(prefix_);
    freeDeviceArray(cubTmp_);
  }

  cusLoadBalance(const cusLoadBalance&) = delete;
  cusLoadBalance& operator=(const cusLoadBalance&) = delete;

  // Kept for the reference interface: the partition is computed inside every traversal.
  void LoadBalanceArray(cuStinger& custing) { (void)custing; }

  // F(src, dst) for every entry dst of the list of every src in arr[0 .. len) (every vertex
  // when arr is NULL), one thread per edge.
  template <cusSubKernelEdge F>
  void traverseEdges(cuStinger& custing, void* metadata, const vertexId_t* arr, length_t len) {
    if (len <= 0) return;
    reserve(len);
    cuStinger* cs = custing.devicePtr();
    lb_detail::k_lengths<<<lb_detail::blocks_for((long long)len + 1), lb_detail::kThreads>>>(cs, arr, len, len_);
    size_t bytes = cubBytes_;
    cub::DeviceScan::ExclusiveSum(cubTmp_, bytes, len_, prefix_, (int)len + 1);
    // a thread per edge up to the resident grid; the kernel strides over the rest
    lb_detail::k_edges<F><<<lb_detail::resident_blocks(), lb_detail::kThreads>>>(cs, metadata, arr, len, prefix_);
  }

  vertexId_t* currArray = nullptr;
  length_t currArrayLen = 0;

 private:
  void reserve(length_t n) {
    if (n <= cap_ && prefix_) return;
    freeDeviceArray(len_);
    freeDeviceArray(prefix_);
    freeDeviceArray(cubTmp_);
    cap_ = n > 0 ? n : 1;
    len_ = static_cast<long long*>(allocDeviceArray(cap_ + 1, sizeof(long long)));
    prefix_ = static_cast<long long*>(allocDeviceArray(cap_ + 1, sizeof(long long)));
    cubBytes_ = 0;
    cub::DeviceScan::ExclusiveSum(nullptr, cubBytes_, len_, prefix_, (int)cap_ + 1);
    cubTmp_ = allocDeviceArray((length_t)((cubBytes_ + 15) / 16), 16);
  }

  long long* len_ = nullptr;     // list lengths of the array, then 0
  long long* prefix_ = nullptr;  // their exclusive prefix (prefix_[n] = total)
  void* cubTmp_ = nullptr;
  size_t cubBytes_ = 0;
  length_t cap_ = 0;
  bool internalAlloc_ = false;
};

}  // namespace cuStingerAlgs

#endif
