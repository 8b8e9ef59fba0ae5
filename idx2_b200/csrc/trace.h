// Host stage timers. With IDX2G_TRACE set in the environment, every stage of encode, pack,
// write and dataset open prints one line "idx2g <stage> <ms>" to stderr; otherwise a lap
// costs one branch. The timers measure host wall time (device work is timed with events).
#pragma once

#include <chrono>
#include <cstdio>
#include <cstdlib>

namespace idx2g
{

inline bool trace_on()
{
  static const bool on = std::getenv("IDX2G_TRACE") != nullptr;
  return on;
}

struct stage_timer
{
  double t = 0;
  stage_timer()
  {
    if (trace_on())
      t = now();
  }
  static double now()
  {
    return std::chrono::duration<double>(std::chrono::steady_clock::now().time_since_epoch()).count();
  }
  // prints the time since the previous lap (or construction) under `stage`
  void lap(const char* stage)
  {
    if (!trace_on())
      return;
    double n = now();
    std::fprintf(stderr, "idx2g %s %.3f\n", stage, 1e3 * (n - t));
    t = n;
  }
};

} // namespace idx2g
