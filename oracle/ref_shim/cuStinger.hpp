// Compile-only stand-in for the absent cuStinger core header (externals/cuStinger is an empty
// submodule in the reference). It declares just enough for the reference's tests/cct.cpp to
// compile so that its CPU counter (hostSingleIntersection / hostCountTriangles) can be built
// from the reference source as an oracle. Every stub aborts if reached: only the CPU counter
// is ever called.
#ifndef REF_SHIM_CUSTINGER_HPP_
#define REF_SHIM_CUSTINGER_HPP_
#include <cstdint>
#include <cstdlib>
#include <cstdio>
#include <iostream>
#include <string>
#include <cuda_runtime.h>

using namespace std;

typedef int32_t vertexId_t;  // the int32 typedefs the reference's kernels assume
typedef int32_t length_t;

enum cuStingerInitState { eInitStateEmpty, eInitStateCSR, eInitStateEdgeList };

struct cuStingerInitConfig {
  cuStingerInitState initState;
  length_t maxNV;
  bool useVWeight, isSemantic, useEWeight;
  length_t csrNV, csrNE;
  length_t* csrOff;
  vertexId_t* csrAdj;
  void* csrVW;
  void* csrEW;
};

inline void ref_shim_unreachable(const char* what) {
  fprintf(stderr, "reference shim: %s is not available\n", what);
  abort();
}

inline void defaultInitAllocater() {}
inline void defaultUpdateAllocater() {}

class cuStinger {
 public:
  template <typename A, typename B>
  cuStinger(A, B) {}
  void initializeCuStinger(cuStingerInitConfig&) { ref_shim_unreachable("initializeCuStinger"); }
  void freecuStinger() {}
  cuStinger* devicePtr() { return this; }
};
#endif
