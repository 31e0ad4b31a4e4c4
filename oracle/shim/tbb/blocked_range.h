// Test infrastructure: oneTBB blocked_range stand-in (see tbb_shim_pool.h).
#pragma once
#include "tbb_shim_pool.h"

namespace tbb {

template <typename Value>
class blocked_range
{
public:
  blocked_range() = default;
  blocked_range(Value b, Value e, size_t grain = 1) : b_(b), e_(e), grain_(grain) {}
  Value begin() const { return b_; }
  Value end() const { return e_; }
  size_t size() const { return size_t(e_ - b_); }
  bool empty() const { return !(b_ < e_); }
  size_t grainsize() const { return grain_; }

private:
  Value b_{}, e_{};
  size_t grain_ = 1;
};

class static_partitioner {};
class simple_partitioner {};
class auto_partitioner {};

} // namespace tbb
