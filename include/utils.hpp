// utils.hpp - the graph readers and event timers the reference drivers take from the cuStinger
// core (tests/cct.cpp:9, 239-257, 189-201), which is absent from the reference tree. The readers
// live in libtcgen.so (custingeralg_b200/csrc/tcgen_io.cpp) and return the symmetric, sorted,
// deduplicated CSR without self-loops in malloc'd arrays the caller frees with free().
#ifndef CUSTINGER_UTILS_HPP_
#define CUSTINGER_UTILS_HPP_

#include <cuda_runtime.h>

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

#endif
