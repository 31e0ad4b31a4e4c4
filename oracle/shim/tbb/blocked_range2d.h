// Test infrastructure: oneTBB blocked_range2d stand-in (see tbb_shim_pool.h).
#pragma once
#include "blocked_range.h"

namespace tbb {

template <typename RowValue, typename ColValue = RowValue>
class blocked_range2d
{
public:
  blocked_range2d(RowValue rb, RowValue re, ColValue cb, ColValue ce)
    : rows_(rb, re), cols_(cb, ce) {}
  blocked_range2d(const blocked_range<RowValue>& r, const blocked_range<ColValue>& c)
    : rows_(r), cols_(c) {}
  const blocked_range<RowValue>& rows() const { return rows_; }
  const blocked_range<ColValue>& cols() const { return cols_; }
  bool empty() const { return rows_.empty() || cols_.empty(); }

private:
  blocked_range<RowValue> rows_;
  blocked_range<ColValue> cols_;
};

} // namespace tbb
