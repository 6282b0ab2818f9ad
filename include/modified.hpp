// modified.hpp - compatibility header: the reference's streaming driver includes it
// (tests/cct_upd.cpp:14) from the absent cuStinger core. Everything the driver uses from the
// core is declared in cuStinger.hpp, update.hpp, utils.hpp and timer.h.
#ifndef CUSTINGER_MODIFIED_HPP_
#define CUSTINGER_MODIFIED_HPP_

#include "cuStinger.hpp"
#include "update.hpp"

#endif
