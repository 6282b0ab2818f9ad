// Streaming triangle counting entry point with the reference's signature
// (src/streaming_triangle_counting/cct_upd.cu:412-415, redeclared tests/cct_upd.cpp:31-34).
#ifndef CUSTINGER_TC_STREAMING_CCT_UPD_HPP_
#define CUSTINGER_TC_STREAMING_CCT_UPD_HPP_

#include "static_triangle_counting/cct.hpp"

// After custing.edgeInsertionsSorted(bu, ...): add to outPutTriangles[v] (device int32[nv+1])
// the change of 2 t(v) caused by the batch's new edges, i.e. +2 for every vertex of every new
// triangle (the net of the reference's three kernels K1 + K2 - K3 on a symmetric batch).
// h_triangles / h_triangles_t are unused, as in the reference.
void callDeviceNewTriangles(cuStinger& custing, BatchUpdate& bu, triangle_t* const __restrict__ outPutTriangles,
                            const int threads_per_block, const int number_blocks, const int shifter,
                            const int thread_blocks, const int blockdim, triangle_t* const __restrict__ h_triangles,
                            triangle_t* const __restrict__ h_triangles_t);

// Deletion counterpart (no reference kernel exists): BEFORE custing.edgeDeletionsSorted(bu),
// subtract 2 from outPutTriangles[v] for every vertex of every triangle the batch destroys.
void callDeviceDeletedTriangles(cuStinger& custing, BatchUpdate& bu, triangle_t* const __restrict__ outPutTriangles);

#endif
