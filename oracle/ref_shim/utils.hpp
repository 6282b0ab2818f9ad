// Compile-only stand-in for the absent cuStinger utils header (see cuStinger.hpp here).
#ifndef REF_SHIM_UTILS_HPP_
#define REF_SHIM_UTILS_HPP_
#include "cuStinger.hpp"

inline void readGraphDIMACS(char*, length_t**, vertexId_t**, length_t*, length_t*, bool) {
  ref_shim_unreachable("readGraphDIMACS");
}
inline void readGraphSNAP(char*, length_t**, vertexId_t**, length_t*, length_t*, bool) {
  ref_shim_unreachable("readGraphSNAP");
}
inline void readGraphMatrixMarket(char*, length_t**, vertexId_t**, length_t*, length_t*, bool) {
  ref_shim_unreachable("readGraphMatrixMarket");
}
inline void start_clock(cudaEvent_t&, cudaEvent_t&) { ref_shim_unreachable("start_clock"); }
inline float end_clock(cudaEvent_t&, cudaEvent_t&) {
  ref_shim_unreachable("end_clock");
  return 0.f;
}
#endif
