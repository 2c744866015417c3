// oneTBB global_control: accepted and ignored (the compat scheduler runs the
// tasks on the threads that wait for them)
#pragma once

#include <cstddef>

namespace tbb {

  class global_control {
  public:
    enum parameter { max_allowed_parallelism, thread_stack_size };
    global_control(parameter, std::size_t) {}
  };

}  // namespace tbb
