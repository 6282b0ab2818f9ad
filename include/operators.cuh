// operators.cuh - traversal operators of the cuStinger algorithm library, with the names and
// call forms of the reference's include/operators.cuh (allVinG_TraverseVertices,
// allEinG_TraverseEdges, allVinA_TraverseVertices, allVinA_TraverseEdges,
// allVinA_TraverseEdges_LB, allEinA_TraverseEdges), so algorithms written against them (the
// reference's BFS, connected components and PageRank) build on this library unchanged.
//
// Each operator launches one kernel on the default stream and calls a __device__ function,
// given as a template argument, per vertex or per edge:
//   - vertex operators: one thread per vertex, grid-strided;
//   - edge operators over all vertices or a vertex array: edge-balanced through cusLoadBalance
//     (one thread per edge slot of the concatenated lists; load_balance.cuh), so power-law hubs
//     do not serialise a warp;
//   - batch edges: one thread per batch entry.
// The device view of the graph (cuStinger::devicePtr()) is refreshed by the handle after
// structural updates.
#ifndef CUSTINGER_OPERATORS_CUH_
#define CUSTINGER_OPERATORS_CUH_

#include "algs.cuh"
#include "load_balance.cuh"
#include "update.hpp"

namespace cuStingerAlgs {

namespace ops_detail {

template <cusSubKernelVertex F>
static __global__ void k_all_vertices(cuStinger* cs, void* metadata, length_t nv) {
  for (long long v = (long long)blockIdx.x * blockDim.x + threadIdx.x; v < nv; v += (long long)gridDim.x * blockDim.x)
    (F)(cs, (vertexId_t)v, metadata);
}

template <cusSubKernelVertex F>
static __global__ void k_array_vertices(cuStinger* cs, void* metadata, const vertexId_t* arr, length_t len) {
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < len; i += (long long)gridDim.x * blockDim.x)
    (F)(cs, arr[i], metadata);
}

// One warp per vertex of the array (lists read with coalesced loads); no workspace.
template <cusSubKernelEdge F>
static __global__ void k_array_edges_warp(cuStinger* cs, void* metadata, const vertexId_t* arr, length_t len) {
  const int lane = threadIdx.x & 31;
  const long long w0 = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const long long nw = ((long long)gridDim.x * blockDim.x) >> 5;
  for (long long i = w0; i < len; i += nw) {
    const vertexId_t src = arr[i];
    const length_t d = cs->dVD->used[src];
    const vertexId_t* lst = cs->dVD->adj[src]->dst;
    for (length_t k = lane; k < d; k += 32) (F)(cs, src, lst[k], metadata);
  }
}

template <cusSubKernelEdge F>
static __global__ void k_batch_edges(cuStinger* cs, void* metadata, const vertexId_t* src, const vertexId_t* dst,
                                     length_t b) {
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < b; i += (long long)gridDim.x * blockDim.x)
    (F)(cs, src[i], dst[i], metadata);
}

}  // namespace ops_detail

// F(v) for every vertex of the graph.
template <cusSubKernelVertex cusSK>
static void allVinG_TraverseVertices(cuStinger& custing, void* metadata) {
  const length_t nv = custing.nv;
  if (nv <= 0) return;
  ops_detail::k_all_vertices<cusSK><<<lb_detail::blocks_for(nv), lb_detail::kThreads>>>(custing.devicePtr(), metadata,
                                                                                          nv);
}

// F(src, dst) for every directed edge of the graph (both directions of an undirected edge),
// edge-balanced. Allocates its scan workspace for the call.
template <cusSubKernelEdge cusSK>
static void allEinG_TraverseEdges(cuStinger& custing, void* metadata) {
  if (custing.nv <= 0) return;
  cusLoadBalance lb(custing.nv);
  lb.traverseEdges<cusSK>(custing, metadata, nullptr, custing.nv);
}

// F(v) for every vertex of a device array.
template <cusSubKernelVertex cusSK>
static void allVinA_TraverseVertices(cuStinger& custing, void* metadata, vertexId_t* verArray, length_t len) {
  if (len <= 0) return;
  ops_detail::k_array_vertices<cusSK><<<lb_detail::blocks_for(len), lb_detail::kThreads>>>(custing.devicePtr(),
                                                                                             metadata, verArray, len);
}

template <cusSubKernelVertex cusSK>
static void allVinA_TraverseVertices(cuStinger& custing, void* metadata, cusLoadBalance& cusLB) {
  allVinA_TraverseVertices<cusSK>(custing, metadata, cusLB.currArray, cusLB.currArrayLen);
}

// F(src, dst) for the lists of a device array of vertices, one warp per vertex.
template <cusSubKernelEdge cusSK>
static void allVinA_TraverseEdges(cuStinger& custing, void* metadata, vertexId_t* verArray, length_t len) {
  if (len <= 0) return;
  ops_detail::k_array_edges_warp<cusSK><<<lb_detail::blocks_for((long long)len * 32), lb_detail::kThreads>>>(
      custing.devicePtr(), metadata, verArray, len);
}

// Edge-balanced: the lists of the active part of a vertex queue (a frontier) ...
template <cusSubKernelEdge cusSK>
static void allVinA_TraverseEdges_LB(cuStinger& custing, void* metadata, cusLoadBalance& cusLB, vertexQueue& vQueue,
                                     bool needLoadBalance = true) {
  (void)needLoadBalance;  // the partition is always per edge
  cusLB.traverseEdges<cusSK>(custing, metadata, vQueue.getQueueAtCurr(), vQueue.getActiveQueueSize());
}

// ... or of the load balancer's own vertex array.
template <cusSubKernelEdge cusSK>
static void allVinA_TraverseEdges_LB(cuStinger& custing, void* metadata, cusLoadBalance& cusLB) {
  cusLB.traverseEdges<cusSK>(custing, metadata, cusLB.currArray, cusLB.currArrayLen);
}

// F(src, dst) for every entry of a batch (its device copy).
template <cusSubKernelEdge cusSK>
static void allEinA_TraverseEdges(cuStinger& custing, void* metadata, BatchUpdate& bu) {
  const length_t b = *bu.getHostBUD()->getBatchSize();
  if (b <= 0) return;
  BatchUpdateData* d = bu.getDeviceBUD();
  ops_detail::k_batch_edges<cusSK><<<lb_detail::blocks_for(b), lb_detail::kThreads>>>(
      custing.devicePtr(), metadata, d->getSrc(), d->getDst(), b);
}

}  // namespace cuStingerAlgs

#endif
