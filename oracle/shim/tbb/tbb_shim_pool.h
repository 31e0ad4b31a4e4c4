// Test infrastructure: a std::thread stand-in for the few oneTBB entry points the
// reference uses (sys/tasking.h:23-51, image/accum_buffer.h, material/material_param.h).
// It exists only so the reference's own sources compile here without oneTBB; it is linked
// into the oracle library and never into the product.
//
// Semantics kept from oneTBB that the reference relies on:
//   * this_task_arena::current_thread_index() is unique among threads running a
//     parallel region and lies in [0, max_concurrency()); PathRendererStream indexes its
//     per-thread state array with it (render/path_renderer_stream.h:205).
//   * parallel_for with static_partitioner splits the range into contiguous chunks, one
//     per worker; Tasking::run relies only on every index being visited once.
#pragma once

#include <algorithm>
#include <immintrin.h> // oneTBB pulls this in; sys/atomic.h relies on _mm_pause
#include <atomic>
#include <cstdlib>
#include <functional>
#include <thread>
#include <vector>

namespace tbb {
namespace shim {

inline int& threadIndexRef()
{
  static thread_local int index = 0;
  return index;
}

inline int maxThreads()
{
  static int n = []() {
    const char* env = std::getenv("PRT_ORACLE_THREADS");
    int v = env ? std::atoi(env) : 0;
    if (v <= 0) v = (int)std::thread::hardware_concurrency();
    return std::max(v, 1);
  }();
  return n;
}

inline bool& inParallelRef()
{
  static thread_local bool inside = false;
  return inside;
}

// Runs fn(workerIndex) on `count` threads (the calling thread is worker 0) and joins.
inline void runWorkers(int count, const std::function<void(int)>& fn)
{
  if (count <= 1 || inParallelRef())
  {
    // Nested regions run inline on the calling thread, keeping its index.
    bool saved = inParallelRef();
    inParallelRef() = true;
    fn(threadIndexRef());
    inParallelRef() = saved;
    return;
  }
  std::vector<std::thread> threads;
  threads.reserve(count - 1);
  for (int w = 1; w < count; ++w)
  {
    threads.emplace_back([w, &fn]() {
      threadIndexRef() = w;
      inParallelRef() = true;
      fn(w);
    });
  }
  int savedIndex = threadIndexRef();
  threadIndexRef() = 0;
  inParallelRef() = true;
  fn(0);
  inParallelRef() = false;
  threadIndexRef() = savedIndex;
  for (auto& t : threads) t.join();
}

} // namespace shim
} // namespace tbb
