// Test infrastructure: oneTBB parallel_for stand-in (see tbb_shim_pool.h).
// The range is cut into one contiguous chunk per worker; a body that pulls work from a
// shared counter (Tasking::run) load-balances by itself.
#pragma once
#include "blocked_range.h"
#include "blocked_range2d.h"

namespace tbb {

template <typename Value, typename Body>
void parallel_for(const blocked_range<Value>& range, const Body& body)
{
  const long long n = (long long)(range.end() - range.begin());
  if (n <= 0) return;
  const int workers = (int)std::min<long long>(shim::maxThreads(), n);
  shim::runWorkers(workers, [&](int w) {
    const long long lo = n * w / workers;
    const long long hi = n * (w + 1) / workers;
    if (hi > lo)
      body(blocked_range<Value>(Value(range.begin() + lo), Value(range.begin() + hi)));
  });
}

template <typename Value, typename Body, typename Partitioner>
void parallel_for(const blocked_range<Value>& range, const Body& body, const Partitioner&)
{
  parallel_for(range, body);
}

template <typename Index, typename Func>
void parallel_for(Index first, Index last, const Func& f)
{
  parallel_for(blocked_range<Index>(first, last), [&](const blocked_range<Index>& r) {
    for (Index i = r.begin(); i != r.end(); ++i) f(i);
  });
}

} // namespace tbb
