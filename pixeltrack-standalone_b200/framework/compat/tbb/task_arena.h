// oneTBB task_arena (see detail_scheduler.h): one arena for the process
#pragma once

#include <utility>

#include "tbb/detail_scheduler.h"

namespace tbb {

  class task_arena {
  public:
    struct attach {};
    explicit task_arena(int max_concurrency = -1) : concurrency_(max_concurrency) {}
    explicit task_arena(attach) {}

    template <typename F>
    void enqueue(F&& f) {
      detail_compat::Scheduler::instance().push(std::function<void()>(std::forward<F>(f)));
    }

    template <typename F>
    auto execute(F&& f) -> decltype(f()) {
      return f();
    }

    int max_concurrency() const { return concurrency_; }

  private:
    int concurrency_ = -1;
  };

}  // namespace tbb
