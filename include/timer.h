// timer.h - the host wall-clock timer of the cuStinger utilities that the reference's streaming
// driver calls (init_timer / tic / toc, tests/cct_upd.cpp:259-264,374-404,432; part of the absent
// cuStinger core). toc() returns the seconds since the last tic() (or init_timer()); it does not
// synchronise the device, so it times what the host waited for.
#ifndef CUSTINGER_TIMER_H_
#define CUSTINGER_TIMER_H_

#include <chrono>

namespace custinger_timer {
inline std::chrono::steady_clock::time_point& mark() {
  static std::chrono::steady_clock::time_point t = std::chrono::steady_clock::now();
  return t;
}
}  // namespace custinger_timer

inline void init_timer() { custinger_timer::mark() = std::chrono::steady_clock::now(); }
inline void tic() { custinger_timer::mark() = std::chrono::steady_clock::now(); }
inline double toc() {
  return std::chrono::duration<double>(std::chrono::steady_clock::now() - custinger_timer::mark()).count();
}

#endif
