// cuStingerDefs.hpp - the integer types of the cuStinger API (int32 ids and lengths), as the
// reference's triangle-counting code assumes them (include/static_triangle_counting/cct.hpp:12
// and its use of vertexId_t / length_t from the cuStinger core).
#ifndef CUSTINGER_DEFS_HPP_
#define CUSTINGER_DEFS_HPP_

#include <stdint.h>

typedef int32_t vertexId_t;
typedef int32_t length_t;

#if defined(__CUDACC__)
#define CUS_HD __host__ __device__
#else
#define CUS_HD
#endif

#endif
