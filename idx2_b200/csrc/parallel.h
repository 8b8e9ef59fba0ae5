// Host thread pool for the pack, write and open stages: f(i) for i in [0, n) on up to 32
// threads (the calling thread included), items handed out one at a time.
#pragma once

#include <atomic>
#include <cstddef>
#include <thread>
#include <vector>

namespace idx2g
{

template <typename F>
void parallel_for(size_t n, F&& f)
{
  unsigned nt = std::thread::hardware_concurrency();
  nt = nt ? (nt > 32 ? 32 : nt) : 4;
  if (nt > n)
    nt = (unsigned)(n ? n : 1);
  std::atomic<size_t> next{ 0 };
  auto work = [&]() {
    for (size_t i; (i = next.fetch_add(1)) < n;)
      f(i);
  };
  std::vector<std::thread> th;
  for (unsigned t = 1; t < nt; ++t)
    th.emplace_back(work);
  work();
  for (auto& t : th)
    t.join();
}

// f(i0, i1) over [0, n) cut into about 8 ranges per thread
template <typename F>
void parallel_ranges(size_t n, F&& f)
{
  unsigned nt = std::thread::hardware_concurrency();
  nt = nt ? (nt > 32 ? 32 : nt) : 4;
  const size_t nr = (size_t)nt * 8;
  const size_t step = (n + nr - 1) / nr;
  if (!step)
    return;
  parallel_for((n + step - 1) / step, [&](size_t r) {
    const size_t i0 = r * step;
    f(i0, i0 + step < n ? i0 + step : n);
  });
}

} // namespace idx2g
