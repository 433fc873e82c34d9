// Minimal fork-join helper for the host-side passes (format conversion, value
// refresh maps).  Work is split into contiguous index ranges, one per thread.
#ifndef ISPM_HOST_POOL_H
#define ISPM_HOST_POOL_H

#include <algorithm>
#include <thread>
#include <vector>

#include "ispm_internal.h"

namespace ispm {

template <class F> void parallel_for(long long n, F fn)
{
  if (n <= 0)
    return;
  long long nt = host_threads();
  // Below a few thousand items the thread start-up costs more than it saves.
  if (nt > n / 2048)
    nt = std::max(1LL, n / 2048);
  if (nt <= 1) {
    fn(0LL, n);
    return;
  }
  std::vector<std::thread> pool;
  pool.reserve(nt - 1);
  long long step = (n + nt - 1) / nt;
  for (long long t = 1; t < nt; t++) {
    long long lo = t * step, hi = std::min(n, lo + step);
    if (lo >= hi)
      break;
    pool.emplace_back([=] { fn(lo, hi); });
  }
  fn(0LL, std::min(n, step));
  for (auto &th : pool)
    th.join();
}

}  // namespace ispm

#endif
