// The cuStinger-compatible C++ layer (include/cuStinger.hpp, update.hpp,
// static_triangle_counting/cct.hpp, streaming_triangle_counting/cct_upd.hpp): thin wrappers over
// the C ABI that keep the reference's call pattern and signatures.
#include <algorithm>
#include <cstdio>
#include <cstring>
#include <vector>

#include "cuStinger.hpp"
#include "static_triangle_counting/cct.hpp"
#include "streaming_triangle_counting/cct_upd.hpp"
#include "update.hpp"

namespace {

void report(const char* where, tc_status s) {
  if (s != TC_OK) fprintf(stderr, "%s: %s (%s)\n", where, tc_status_string(s), tc_last_error());
}

// Slack fraction implied by an initial-capacity policy at large degree.
double slack_of(initAllocator ia) {
  if (!ia) return 0.0;
  const length_t probe = 1 << 16;
  const double r = (double)ia(probe) / (double)probe - 1.0;
  return std::min(8.0, std::max(0.0, r));
}

__global__ void k_fill_view(const int32_t n, const int64_t* __restrict__ start, int32_t* __restrict__ pool,
                            cusEdgeData* __restrict__ edges, cusEdgeData** __restrict__ adj) {
  for (int64_t v = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; v < n; v += (int64_t)gridDim.x * blockDim.x) {
    edges[v].dst = pool + start[v];
    adj[v] = &edges[v];
  }
}

}  // namespace

length_t defaultInitAllocater(length_t elements) { return elements + elements / 2 + 4; }
length_t defaultUpdateAllocater(length_t elements, length_t overLimit) {
  const length_t need = elements + overLimit;
  return need + need / 2 + 4;
}
length_t exactInitAllocater(length_t elements) { return elements; }
length_t exactUpdateAllocater(length_t elements, length_t overLimit) { return elements + overLimit; }

// ---- cuStinger ---------------------------------------------------------------------------------

cuStinger::cuStinger(initAllocator ia, updateAllocator ua) : ia_(ia), ua_(ua) {}

cuStinger::cuStinger(const cuStinger& other)
    : nv(other.nv), g_(other.g_), ia_(other.ia_), ua_(other.ua_), owns_graph_(false), status_(other.status_) {}

cuStinger::~cuStinger() {
  if (owns_graph_) freecuStinger();
  else releaseView();
}

void cuStinger::releaseView() {
  cudaFree(d_self_);
  cudaFree(d_vd_);
  cudaFree(d_edges_);
  cudaFree(d_adj_);
  d_self_ = nullptr;
  d_vd_ = nullptr;
  d_edges_ = nullptr;
  d_adj_ = nullptr;
  dVD = nullptr;
  view_stale_ = true;
}

void cuStinger::initializeCuStinger(cuStingerInitConfig& cfg) {
  freecuStinger();
  if (cfg.initState != eInitStateCSR || cfg.csrVW || cfg.csrEW || cfg.useVWeight || cfg.useEWeight || cfg.isSemantic) {
    status_ = TC_ERR_INVALID_ARG;
    fprintf(stderr, "initializeCuStinger: only eInitStateCSR without weights or types is supported\n");
    return;
  }
  const length_t nvv = cfg.csrNV;
  // The reference stores int32 offsets; the library takes int64.
  int64_t* off = new int64_t[(size_t)nvv + 1];
  for (length_t i = 0; i <= nvv; ++i) off[i] = cfg.csrOff[i];
  status_ = tc_graph_create(nvv, off, cfg.csrAdj, TC_MEM_HOST, slack_of(ia_), 1, nullptr, &g_);
  delete[] off;
  report("initializeCuStinger", status_);
  if (status_ == TC_OK) nv = nvv;
  view_stale_ = true;
}

void cuStinger::freecuStinger() {
  if (g_ && owns_graph_) tc_graph_destroy(g_);
  g_ = nullptr;
  releaseView();
  nv = 0;
}

void cuStinger::refreshDeviceView() {
  if (!g_) return;
  const int64_t* start = nullptr;
  const int32_t* used = nullptr;
  const int32_t* pool = nullptr;
  tc_graph_device_view(g_, &start, &used, &pool);
  if (!d_vd_) {
    cudaMalloc(&d_vd_, sizeof(cusVertexData));
    cudaMalloc(&d_edges_, sizeof(cusEdgeData) * std::max(nv, 1));
    cudaMalloc(&d_adj_, sizeof(cusEdgeData*) * std::max(nv, 1));
    cudaMalloc(&d_self_, sizeof(cuStinger));
  }
  if (nv > 0) {
    k_fill_view<<<std::min(4096, (nv + 255) / 256), 256>>>(nv, start, const_cast<int32_t*>(pool), d_edges_, d_adj_);
  }
  cusVertexData h;
  h.used = const_cast<length_t*>(used);
  h.max = nullptr;
  h.adj = d_adj_;
  cudaMemcpy(d_vd_, &h, sizeof(h), cudaMemcpyHostToDevice);
  dVD = d_vd_;
  // Only the leading {nv, dVD} members are meaningful on the device.
  cudaMemcpy(d_self_, this, sizeof(cuStinger), cudaMemcpyHostToDevice);
  view_stale_ = false;
}

cuStinger* cuStinger::devicePtr() {
  if (view_stale_) refreshDeviceView();
  return d_self_;
}

length_t cuStinger::getNumberEdgesUsed() const {
  int64_t used = 0;
  if (g_) tc_graph_info(g_, nullptr, &used, nullptr);
  return (length_t)used;
}

length_t cuStinger::getNumberEdgesAllocated() const {
  int64_t alloc = 0;
  if (g_) tc_graph_info(g_, nullptr, nullptr, &alloc);
  return (length_t)alloc;
}

void cuStinger::edgeInsertionsSorted(BatchUpdate& bu, length_t& requireAllocation) {
  requireAllocation = 0;
  BatchUpdateData* d = bu.getDeviceBUD();
  if (!g_ || !bu.isSorted()) {
    status_ = TC_ERR_STATE;
    fprintf(stderr, "edgeInsertionsSorted: %s\n", g_ ? "batch not sorted (call sortDeviceBUD)" : "no graph");
    return;
  }
  int64_t moved = 0;
  status_ = tc_insert_sorted(g_, d->getSrc(), d->getDst(), *bu.getHostBUD()->getBatchSize(), d->getIndDuplicate(),
                             &moved, nullptr);
  report("edgeInsertionsSorted", status_);
  requireAllocation = (length_t)moved;
  view_stale_ = true;
}

void cuStinger::edgeDeletionsSorted(BatchUpdate& bu) {
  BatchUpdateData* d = bu.getDeviceBUD();
  if (!g_ || !bu.isSorted()) {
    status_ = TC_ERR_STATE;
    fprintf(stderr, "edgeDeletionsSorted: %s\n", g_ ? "batch not sorted (call sortDeviceBUD)" : "no graph");
    return;
  }
  status_ = tc_delete_sorted(g_, d->getSrc(), d->getDst(), d->getIndDuplicate(), *bu.getHostBUD()->getBatchSize(),
                             nullptr);
  report("edgeDeletionsSorted", status_);
  view_stale_ = true;
}

// ---- batches -----------------------------------------------------------------------------------

BatchUpdateData::BatchUpdateData(length_t batchSize, bool isHost, length_t nv) : isHost_(isHost), capacity_(batchSize), nv_(nv) {
  const size_t b = (size_t)std::max(batchSize, 1);
  const size_t n1 = (size_t)std::max(nv, 0) + 1;
  if (isHost) {
    src_ = new vertexId_t[b]();
    dst_ = new vertexId_t[b]();
    indDuplicate_ = new length_t[b]();
    offsets_ = new length_t[n1]();
    vNumDuplicates_ = new length_t[n1]();
    batchSize_ = new length_t[1];
    numVertices_ = new length_t[1];
    batchSize_[0] = batchSize;
    numVertices_[0] = nv;
  } else {
    cudaMalloc(&src_, sizeof(vertexId_t) * b);
    cudaMalloc(&dst_, sizeof(vertexId_t) * b);
    cudaMalloc(&indDuplicate_, sizeof(length_t) * b);
    cudaMalloc(&offsets_, sizeof(length_t) * n1);
    cudaMalloc(&vNumDuplicates_, sizeof(length_t) * n1);
    cudaMalloc(&batchSize_, sizeof(length_t));
    cudaMalloc(&numVertices_, sizeof(length_t));
    cudaMemset(indDuplicate_, 0, sizeof(length_t) * b);
    cudaMemset(offsets_, 0, sizeof(length_t) * n1);
    cudaMemset(vNumDuplicates_, 0, sizeof(length_t) * n1);
    cudaMemcpy(batchSize_, &batchSize, sizeof(length_t), cudaMemcpyHostToDevice);
    cudaMemcpy(numVertices_, &nv, sizeof(length_t), cudaMemcpyHostToDevice);
  }
}

BatchUpdateData::~BatchUpdateData() {
  if (isHost_) {
    delete[] src_;
    delete[] dst_;
    delete[] indDuplicate_;
    delete[] offsets_;
    delete[] vNumDuplicates_;
    delete[] batchSize_;
    delete[] numVertices_;
  } else {
    cudaFree(src_);
    cudaFree(dst_);
    cudaFree(indDuplicate_);
    cudaFree(offsets_);
    cudaFree(vNumDuplicates_);
    cudaFree(batchSize_);
    cudaFree(numVertices_);
    cudaFree(d_self_);
  }
}

BatchUpdateData* BatchUpdateData::devicePtr() {
  if (isHost_) return nullptr;
  if (!d_self_) cudaMalloc(&d_self_, sizeof(BatchUpdateData));
  cudaMemcpy(d_self_, this, sizeof(BatchUpdateData), cudaMemcpyHostToDevice);
  return d_self_;
}

BatchUpdate::BatchUpdate(BatchUpdateData& hostBatch) : host_(&hostBatch) {
  const length_t b = hostBatch.capacity_;
  dev_ = new BatchUpdateData(b, false, hostBatch.nv_);
  if (hostBatch.isHost_) {
    cudaMemcpy(dev_->src_, hostBatch.src_, sizeof(vertexId_t) * (size_t)b, cudaMemcpyHostToDevice);
    cudaMemcpy(dev_->dst_, hostBatch.dst_, sizeof(vertexId_t) * (size_t)b, cudaMemcpyHostToDevice);
  }
}

BatchUpdate::~BatchUpdate() { delete dev_; }

void BatchUpdate::sortDeviceBUD(const int blockdim) {
  (void)blockdim;
  const tc_status s = tc_batch_sort(dev_->nv_, dev_->src_, dev_->dst_, dev_->capacity_, dev_->offsets_,
                                    dev_->indDuplicate_, nullptr);
  report("sortDeviceBUD", s);
  sorted_ = s == TC_OK;
  if (sorted_ && host_ && host_->isHost_) {
    // mirror the sorted batch back like the reference's host copy
    const size_t b = (size_t)dev_->capacity_;
    cudaMemcpy(host_->src_, dev_->src_, sizeof(vertexId_t) * b, cudaMemcpyDeviceToHost);
    cudaMemcpy(host_->dst_, dev_->dst_, sizeof(vertexId_t) * b, cudaMemcpyDeviceToHost);
    cudaMemcpy(host_->indDuplicate_, dev_->indDuplicate_, sizeof(length_t) * b, cudaMemcpyDeviceToHost);
    cudaMemcpy(host_->offsets_, dev_->offsets_, sizeof(length_t) * ((size_t)dev_->nv_ + 1), cudaMemcpyDeviceToHost);
  }
}

// Sort check of the reference's sort test (declared and called at tests/cct_upd.cpp:30,173; its
// definition is not in the reference tree): sort the batch on the device, then verify on the
// host that the entries are ordered by (src, dst), that the batch CSR offsets over src match
// them, and that exactly the self-loops and repeats are flagged. Prints one line.
void testSort(length_t nv, BatchUpdate& bu, const int blockdim) {
  bu.sortDeviceBUD(blockdim);
  BatchUpdateData* d = bu.getDeviceBUD();
  const length_t b = *bu.getHostBUD()->getBatchSize();
  std::vector<vertexId_t> src((size_t)std::max(b, 1)), dst(src.size());
  std::vector<length_t> dup(src.size()), off((size_t)nv + 1);
  cudaMemcpy(src.data(), d->getSrc(), sizeof(vertexId_t) * (size_t)b, cudaMemcpyDeviceToHost);
  cudaMemcpy(dst.data(), d->getDst(), sizeof(vertexId_t) * (size_t)b, cudaMemcpyDeviceToHost);
  cudaMemcpy(dup.data(), d->getIndDuplicate(), sizeof(length_t) * (size_t)b, cudaMemcpyDeviceToHost);
  cudaMemcpy(off.data(), d->getOffsets(), sizeof(length_t) * ((size_t)nv + 1), cudaMemcpyDeviceToHost);
  length_t bad = 0, dups = 0;
  for (length_t i = 0; i < b; ++i) {
    const bool repeat = i > 0 && src[i] == src[i - 1] && dst[i] == dst[i - 1];
    const bool expect_dup = src[i] == dst[i] || repeat;
    if (i > 0 && (src[i] < src[i - 1] || (src[i] == src[i - 1] && dst[i] < dst[i - 1]))) ++bad;
    if ((dup[i] != 0) != expect_dup) ++bad;
    dups += dup[i] != 0;
  }
  for (vertexId_t v = 0; v < nv; ++v)
    for (length_t k = off[v]; k < off[v + 1]; ++k)
      if (k < 0 || k >= b || src[k] != v) ++bad;
  if (off[0] != 0 || off[nv] != b) ++bad;
  printf("testSort: %d entries, %d flagged as duplicates, %s\n", b, dups, bad ? "NOT SORTED" : "sorted");
}

// ---- triangle counting entry points --------------------------------------------------------------

void callDeviceAllTriangles(cuStinger& custing, triangle_t* const __restrict__ outPutTriangles,
                            const int threads_per_block, const int number_blocks, const int shifter,
                            const int thread_blocks, const int blockdim) {
  (void)threads_per_block; (void)number_blocks; (void)shifter; (void)thread_blocks; (void)blockdim;
  const tc_status s = tc_count_static(custing.graph(), TC_PV_HANDLE, outPutTriangles, nullptr, nullptr, nullptr, nullptr);
  custing.setLastStatus(s);
  report("callDeviceAllTriangles", s);
}

void callDeviceAllTrianglesCSR(const vertexId_t nv, length_t const* const __restrict__ d_off,
                               vertexId_t const* const __restrict__ d_ind, int* const __restrict__ outPutTriangles,
                               const int threads_per_block, const int number_blocks, const int shifter,
                               const int thread_blocks, const int blockdim) {
  (void)threads_per_block; (void)number_blocks; (void)shifter; (void)thread_blocks; (void)blockdim;
  const tc_status s = tc_count_csr32(nv, d_off, d_ind, TC_PV_CSR, outPutTriangles, nullptr, nullptr, nullptr, nullptr);
  report("callDeviceAllTrianglesCSR", s);
}

void callDeviceNewTriangles(cuStinger& custing, BatchUpdate& bu, triangle_t* const __restrict__ outPutTriangles,
                            const int threads_per_block, const int number_blocks, const int shifter,
                            const int thread_blocks, const int blockdim, triangle_t* const __restrict__ h_triangles,
                            triangle_t* const __restrict__ h_triangles_t) {
  (void)threads_per_block; (void)number_blocks; (void)shifter; (void)thread_blocks; (void)blockdim;
  (void)h_triangles; (void)h_triangles_t;
  BatchUpdateData* d = bu.getDeviceBUD();
  const tc_status s = tc_count_batch(custing.graph(), d->getSrc(), d->getDst(), d->getOffsets(), d->getIndDuplicate(),
                                     *bu.getHostBUD()->getBatchSize(), +1, outPutTriangles, nullptr, nullptr, nullptr);
  custing.setLastStatus(s);
  report("callDeviceNewTriangles", s);
}

void callDeviceDeletedTriangles(cuStinger& custing, BatchUpdate& bu, triangle_t* const __restrict__ outPutTriangles) {
  BatchUpdateData* d = bu.getDeviceBUD();
  const tc_status s = tc_count_batch(custing.graph(), d->getSrc(), d->getDst(), d->getOffsets(), d->getIndDuplicate(),
                                     *bu.getHostBUD()->getBatchSize(), -1, outPutTriangles, nullptr, nullptr, nullptr);
  custing.setLastStatus(s);
  report("callDeviceDeletedTriangles", s);
}
