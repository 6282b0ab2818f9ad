// cuStinger.hpp - the subset of the cuStinger dynamic-graph handle that the triangle-counting
// entry points take (cuStinger core, externals/cuStinger in the reference, absent from its tree;
// used at tests/cct.cpp:261-281 and tests/cct_upd.cpp:227-244,364-398).
//
// The graph lives in the B200 library (libcustinger_tc.so) behind the C ABI tc_graph*. This class
// keeps the reference's call pattern:
//     cuStinger custing(defaultInitAllocater, defaultUpdateAllocater);
//     cuStingerInitConfig cfg; cfg.initState = eInitStateCSR; cfg.csrNV = nv; ... ;
//     custing.initializeCuStinger(cfg);
//     callDeviceAllTriangles(custing, d_out, ...);
//     custing.freecuStinger();
// and a device-side view in the cuStinger style for user kernels: on the pointer returned by
// devicePtr(), custing->nv, custing->dVD->getUsed()[v] and custing->dVD->getAdj()[v]->dst.
#ifndef CUSTINGER_HPP_
#define CUSTINGER_HPP_

#include <stddef.h>

#include "cuStingerDefs.hpp"
#include "custinger_tc.h"

class BatchUpdate;

// Capacity policies: list capacity for `elements` entries at initialisation, and after an
// update that needs `overLimit` more entries than a list holds. Only their ratio at large
// degrees is used (it becomes the per-list slack of the device storage).
typedef length_t (*initAllocator)(length_t elements);
typedef length_t (*updateAllocator)(length_t elements, length_t overLimit);
length_t defaultInitAllocater(length_t elements);
length_t defaultUpdateAllocater(length_t elements, length_t overLimit);
length_t exactInitAllocater(length_t elements);
length_t exactUpdateAllocater(length_t elements, length_t overLimit);

enum cuStingerInitState { eInitStateEmpty = 0, eInitStateCSR = 1, eInitStateEdgeList = 2 };

struct cuStingerInitConfig {
  cuStingerInitState initState = eInitStateCSR;
  length_t maxNV = 0;
  bool useVWeight = false;
  bool isSemantic = false;
  bool useEWeight = false;
  length_t csrNV = 0;
  length_t csrNE = 0;
  length_t* csrOff = nullptr;   // host, csrNV+1 offsets
  vertexId_t* csrAdj = nullptr; // host, csrNE ids, each list sorted ascending
  void* csrVW = nullptr;        // vertex/edge weights are not supported (must be NULL)
  void* csrEW = nullptr;
};

// Device-side adjacency view in the cuStinger layout.
struct cusEdgeData {
  vertexId_t* dst;
};

struct cusVertexData {
  length_t* used;
  length_t* max;
  cusEdgeData** adj;
  CUS_HD length_t* getUsed() const { return used; }
  CUS_HD length_t* getMax() const { return max; }
  CUS_HD cusEdgeData** getAdj() const { return adj; }
};

class cuStinger {
 public:
  // The first two members form the device-visible part (copied by devicePtr()).
  vertexId_t nv = 0;
  cusVertexData* dVD = nullptr;  // device pointer, valid after devicePtr()

  explicit cuStinger(initAllocator ia = defaultInitAllocater, updateAllocator ua = defaultUpdateAllocater);
  ~cuStinger();
  // A copy (the reference drivers pass cuStinger by value, tests/cct_upd.cpp:124) is a view of
  // the same graph: it reads and updates it, but freeing stays with the original.
  cuStinger(const cuStinger& other);
  cuStinger& operator=(const cuStinger&) = delete;

  // Vertex count, readable on the device copy (devicePtr()) by traversal kernels.
  CUS_HD length_t getMaxNV() const { return nv; }

  void initializeCuStinger(cuStingerInitConfig& cfg);
  void freecuStinger();

  // Device copy of {nv, dVD} for kernels written against the cuStinger device API. Rebuilt
  // after structural updates.
  cuStinger* devicePtr();

  length_t getNumberEdgesUsed() const;
  length_t getNumberEdgesAllocated() const;

  // Sorted batch insertion / deletion (the batch must have gone through sortDeviceBUD).
  // Insertion flags entries already present in the graph as duplicates; requireAllocation
  // returns how many entries did not fit their list's capacity.
  void edgeInsertionsSorted(BatchUpdate& bu, length_t& requireAllocation);
  void edgeDeletionsSorted(BatchUpdate& bu);

  // The underlying library handle (C ABI).
  tc_graph* graph() const { return g_; }
  // Status of the last operation on this handle (TC_OK or a tc_status code).
  tc_status lastStatus() const { return status_; }
  void setLastStatus(tc_status s) { status_ = s; }

 private:
  void refreshDeviceView();
  tc_graph* g_ = nullptr;
  initAllocator ia_;
  updateAllocator ua_;
  cuStinger* d_self_ = nullptr;
  cusVertexData* d_vd_ = nullptr;
  cusEdgeData* d_edges_ = nullptr;
  cusEdgeData** d_adj_ = nullptr;
  bool view_stale_ = true;
  bool owns_graph_ = true;
  tc_status status_ = TC_OK;
  void releaseView();
  friend class BatchUpdate;
};

#endif
