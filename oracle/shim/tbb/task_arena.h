// Test infrastructure: oneTBB this_task_arena stand-in (see tbb_shim_pool.h).
#pragma once
#include "tbb_shim_pool.h"

namespace tbb {
namespace this_task_arena {

inline int max_concurrency() { return shim::maxThreads(); }
inline int current_thread_index() { return shim::threadIndexRef(); }

} // namespace this_task_arena
} // namespace tbb
