// C-ABI wrapper around the reference's own raw-CSR GPU triangle counter, compiled for sm_100a
// together with the reference source tests/cct_csr.cu (see oracle/Makefile). COMPARISON
// INFRASTRUCTURE ONLY: tests time it beside this library's kernels and check its per-vertex
// output (forward convention: out[src] = sum over dest > src of |N(src) ∩ N(dest)|,
// tests/cct_csr.cu:228-276) against them.
//
// The reference's merge-path search reads one entry before and one past a list
// (tests/cct_csr.cu:110-112), so callers pass d_ind with guard entries on both sides of the
// allocation.
#include <cstdint>
#include <cuda_runtime.h>
#include "cuStingerDefs.hpp"
#include "static_triangle_counting/cct.hpp"

void callDeviceAllTrianglesCSR(const vertexId_t nv, length_t const* const __restrict__ d_off,
                               vertexId_t const* const __restrict__ d_ind, int* const __restrict__ outPutTriangles,
                               const int threads_per_block, const int number_blocks, const int shifter,
                               const int thread_blocks, const int blockdim);

extern "C" int ref_gpu_count_csr(int32_t nv, const int32_t* d_off, const int32_t* d_ind, int32_t* d_out,
                                 int32_t threads_per_intersection, int32_t shifter, int32_t blocks,
                                 int32_t block_size) {
  const int nbl = block_size / threads_per_intersection;
  callDeviceAllTrianglesCSR(nv, d_off, d_ind, d_out, threads_per_intersection, nbl, shifter, blocks, block_size);
  return (int)cudaGetLastError();
}
