// Compile-only stand-in for the absent cuStinger update header (see cuStinger.hpp here).
#ifndef REF_SHIM_UPDATE_HPP_
#define REF_SHIM_UPDATE_HPP_
#include "cuStinger.hpp"
#endif
