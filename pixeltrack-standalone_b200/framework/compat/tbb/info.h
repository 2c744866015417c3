// oneTBB info::default_concurrency
#pragma once

#include <thread>

namespace tbb {
  namespace info {
    inline int default_concurrency() {
      unsigned n = std::thread::hardware_concurrency();
      return n ? int(n) : 1;
    }
  }  // namespace info
}  // namespace tbb
