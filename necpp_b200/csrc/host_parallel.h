// Host-side data parallelism for the per-segment and per-direction loops of
// card processing: a range split into contiguous chunks, one std::thread per
// chunk.  Results must not depend on the split: callers write disjoint
// outputs per index and do any reduction serially afterwards.
#pragma once

#include <algorithm>
#include <cstdint>
#include <exception>
#include <thread>
#include <vector>

namespace necb {

// Worker count for a loop of `count` items where one worker should get at
// least `min_per_worker` of them (1 for small loops; at most 8 threads).
inline int host_workers(int64_t count, int64_t min_per_worker) {
  const int hw = std::max(1, std::min(8, (int)std::thread::hardware_concurrency()));
  return (int)std::max<int64_t>(1, std::min<int64_t>(hw, count / std::max<int64_t>(1, min_per_worker)));
}

// f(worker, begin, end) over [0, count) split into `workers` contiguous
// chunks; worker 0 runs on the calling thread.  An exception thrown by f is
// rethrown after all workers finish: the one of the lowest chunk, which is
// the one a serial loop over [0, count) would have met first.
template <typename F>
void parallel_chunks(int64_t count, int workers, F f) {
  if (workers <= 1 || count <= 1) {
    f(0, (int64_t)0, count);
    return;
  }
  const int64_t chunk = (count + workers - 1) / workers;
  std::vector<std::exception_ptr> errs(workers);
  auto run = [&](int w) {
    try {
      f(w, std::min(count, w * chunk), std::min(count, (w + 1) * chunk));
    } catch (...) {
      errs[w] = std::current_exception();
    }
  };
  std::vector<std::thread> pool;
  pool.reserve(workers - 1);
  for (int w = 1; w < workers; w++) pool.emplace_back(run, w);
  run(0);
  for (auto& th : pool) th.join();
  for (auto& ep : errs)
    if (ep) std::rethrow_exception(ep);
}

}  // namespace necb
