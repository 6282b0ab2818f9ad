// Compile-only stand-in for the absent cuStinger definitions header: the int32 id and length
// types the reference's kernels assume (they live in the shim's cuStinger.hpp).
#ifndef REF_SHIM_CUSTINGERDEFS_HPP_
#define REF_SHIM_CUSTINGERDEFS_HPP_
#include "cuStinger.hpp"
#endif
