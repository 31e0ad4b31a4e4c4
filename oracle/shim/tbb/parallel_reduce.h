// Test infrastructure: oneTBB parallel_reduce / parallel_deterministic_reduce stand-ins
// (see tbb_shim_pool.h). Partial results are combined in worker order, so both forms
// are deterministic for a fixed thread count.
#pragma once
#include <mutex>
#include <vector>
#include "blocked_range.h"
#include "blocked_range2d.h"

namespace tbb {

template <typename Value, typename T, typename Body, typename Reduction>
T parallel_reduce(const blocked_range<Value>& range, const T& identity, const Body& body,
                  const Reduction& reduction)
{
  const long long n = (long long)(range.end() - range.begin());
  if (n <= 0) return identity;
  const int workers = (int)std::min<long long>(shim::maxThreads(), n);
  std::vector<T> partial(workers, identity);
  shim::runWorkers(workers, [&](int w) {
    const long long lo = n * w / workers;
    const long long hi = n * (w + 1) / workers;
    if (hi > lo)
      partial[w] = body(blocked_range<Value>(Value(range.begin() + lo), Value(range.begin() + hi)), identity);
  });
  T result = identity;
  for (const T& p : partial) result = reduction(result, p);
  return result;
}

template <typename RowValue, typename ColValue, typename T, typename Body, typename Reduction>
T parallel_reduce(const blocked_range2d<RowValue, ColValue>& range, const T& identity,
                  const Body& body, const Reduction& reduction)
{
  const long long n = (long long)(range.rows().end() - range.rows().begin());
  if (n <= 0) return identity;
  const int workers = (int)std::min<long long>(shim::maxThreads(), n);
  std::vector<T> partial(workers, identity);
  shim::runWorkers(workers, [&](int w) {
    const long long lo = n * w / workers;
    const long long hi = n * (w + 1) / workers;
    if (hi > lo)
      partial[w] = body(blocked_range2d<RowValue, ColValue>(
                          RowValue(range.rows().begin() + lo), RowValue(range.rows().begin() + hi),
                          range.cols().begin(), range.cols().end()),
                        identity);
  });
  T result = identity;
  for (const T& p : partial) result = reduction(result, p);
  return result;
}

template <typename Range, typename T, typename Body, typename Reduction>
T parallel_deterministic_reduce(const Range& range, const T& identity, const Body& body,
                                const Reduction& reduction)
{
  return parallel_reduce(range, identity, body, reduction);
}

} // namespace tbb
