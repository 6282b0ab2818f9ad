// utils.hpp - the graph readers, event timers and array helpers the reference drivers and
// algorithms take from the cuStinger core (tests/cct.cpp:9, 239-257, 189-201;
// src/static_breadth_first_search/bfs_top_down.cu:26-31), which is absent from the reference
// tree. The readers live in libtcgen.so (custingeralg_b200/csrc/tcgen_io.cpp) and return the symmetric, sorted,
// deduplicated CSR without self-loops in malloc'd arrays the caller frees with free().
#ifndef CUSTINGER_UTILS_HPP_
#define CUSTINGER_UTILS_HPP_

#include <cuda_runtime.h>

#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <iostream>
#include <string>

#include "cuStingerDefs.hpp"

// The reference drivers use cout, endl and string unqualified (tests/cct.cpp:216, 240), relying
// on the cuStinger core headers to open namespace std for them; this header does the same so
// that they compile unchanged.
using namespace std;

void readGraphDIMACS(char* filePath, length_t** prmoff, vertexId_t** prmind, length_t* prmnv, length_t* prmne,
                     bool isRmat);
void readGraphSNAP(char* filePath, length_t** prmoff, vertexId_t** prmind, length_t* prmnv, length_t* prmne,
                   bool undirected);
void readGraphMatrixMarket(char* filePath, length_t** prmoff, vertexId_t** prmind, length_t* prmnv,
                           length_t* prmne, bool undirected);

// Event timing on the default stream: start_clock creates and records the pair's start,
// end_clock records the stop, waits for it and returns the elapsed milliseconds.
inline void start_clock(cudaEvent_t& start, cudaEvent_t& stop) {
  cudaEventCreate(&start);
  cudaEventCreate(&stop);
  cudaEventRecord(start, 0);
}

inline float end_clock(cudaEvent_t& start, cudaEvent_t& stop) {
  float ms = 0.f;
  cudaEventRecord(stop, 0);
  cudaEventSynchronize(stop);
  cudaEventElapsedTime(&ms, start, stop);
  cudaEventDestroy(start);
  cudaEventDestroy(stop);
  return ms;
}

// Array helpers of the cuStinger core that algorithms and the operator library call
// (allocDeviceArray(hostBfsData.nv, sizeof(vertexId_t)), copyArrayHostToDevice(&host, dev, 1,
// sizeof(T)), ...: source first, destination second, then element count and size). Blocking
// copies on the default stream; a failed CUDA call is reported on stderr.
inline void cus_report(cudaError_t e, const char* what) {
  if (e != cudaSuccess) fprintf(stderr, "%s: %s\n", what, cudaGetErrorString(e));
}
inline void* allocDeviceArray(length_t elements, int32_t eleSize) {
  void* p = nullptr;
  cus_report(cudaMalloc(&p, (size_t)elements * (size_t)eleSize), "allocDeviceArray");
  return p;
}
inline void freeDeviceArray(void* p) { cus_report(cudaFree(p), "freeDeviceArray"); }
inline void* allocHostArray(length_t elements, int32_t eleSize) { return malloc((size_t)elements * (size_t)eleSize); }
inline void freeHostArray(void* p) { free(p); }
inline void copyArrayHostToDevice(const void* hostSrc, void* devDst, length_t elements, int32_t eleSize) {
  cus_report(cudaMemcpy(devDst, hostSrc, (size_t)elements * (size_t)eleSize, cudaMemcpyHostToDevice),
             "copyArrayHostToDevice");
}
inline void copyArrayDeviceToHost(const void* devSrc, void* hostDst, length_t elements, int32_t eleSize) {
  cus_report(cudaMemcpy(hostDst, devSrc, (size_t)elements * (size_t)eleSize, cudaMemcpyDeviceToHost),
             "copyArrayDeviceToHost");
}
inline void copyArrayHostToHost(const void* hostSrc, void* hostDst, length_t elements, int32_t eleSize) {
  memcpy(hostDst, hostSrc, (size_t)elements * (size_t)eleSize);
}
inline void copyArrayDeviceToDevice(const void* devSrc, void* devDst, length_t elements, int32_t eleSize) {
  cus_report(cudaMemcpy(devDst, devSrc, (size_t)elements * (size_t)eleSize, cudaMemcpyDeviceToDevice),
             "copyArrayDeviceToDevice");
}

#endif
