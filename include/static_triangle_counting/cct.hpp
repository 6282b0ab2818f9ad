// Static triangle counting entry points with the reference's signatures
// (include/static_triangle_counting/cct.hpp:15-17, tests/cct_csr.cu:279-282).
#ifndef CUSTINGER_TC_STATIC_CCT_HPP_
#define CUSTINGER_TC_STATIC_CCT_HPP_

#include "cuStinger.hpp"
#include "update.hpp"

typedef int32_t triangle_t;

// outPutTriangles: device int32[nv+1]; entries [0, nv) are overwritten with 2 t(v) (their sum
// is 6T, hostCountTriangles' total). The launch-shape arguments are accepted as hints; the
// library's scheduler picks the strategy and grid. Stream-ordered on the legacy default stream
// like the reference launch; errors are kept in custing.lastStatus() / tc_last_error().
void callDeviceAllTriangles(cuStinger& custing, triangle_t* const __restrict__ outPutTriangles,
                            const int threads_per_block, const int number_blocks, const int shifter,
                            const int thread_blocks, const int blockdim);

// Raw CSR (device d_off int32[nv+1], d_ind): outPutTriangles[v] = sum over w in N(v), w > v of
// |N(v) ∩ N(w)| (their sum is 3T), entries [0, nv) overwritten.
void callDeviceAllTrianglesCSR(const vertexId_t nv, length_t const* const __restrict__ d_off,
                               vertexId_t const* const __restrict__ d_ind, int* const __restrict__ outPutTriangles,
                               const int threads_per_block, const int number_blocks, const int shifter,
                               const int thread_blocks, const int blockdim);

#endif
