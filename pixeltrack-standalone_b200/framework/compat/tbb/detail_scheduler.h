// The part of oneTBB's task API that the reference framework uses
// (task_group, task_handle, task_arena, global_control, info,
// concurrent_queue), for building the framework and its plugins where oneTBB
// is not installed.  Every task of the process goes through one queue; a
// thread that waits on a task_group runs queued tasks (of any group) until
// its group has none left, so an event loop run from one thread interleaves
// the events of all its streams, and threads outside the loop (completion
// callbacks of device work) hand tasks back through task_arena::enqueue.
// oneTBB itself runs the same task graph on a thread pool.
#pragma once

#include <atomic>
#include <chrono>
#include <condition_variable>
#include <deque>
#include <functional>
#include <mutex>

namespace tbb {
  namespace detail_compat {

    class Scheduler {
    public:
      static Scheduler& instance() {
        static Scheduler s;
        return s;
      }
      void push(std::function<void()> f) {
        {
          std::lock_guard<std::mutex> lk(mu_);
          queue_.push_back(std::move(f));
        }
        cv_.notify_all();
      }
      // runs one queued task, or waits a little for one; false when none ran
      bool runOne() {
        std::function<void()> f;
        {
          std::unique_lock<std::mutex> lk(mu_);
          if (queue_.empty()) cv_.wait_for(lk, std::chrono::milliseconds(1));
          if (queue_.empty()) return false;
          f = std::move(queue_.front());
          queue_.pop_front();
        }
        f();
        return true;
      }
      bool empty() {
        std::lock_guard<std::mutex> lk(mu_);
        return queue_.empty();
      }
      void notify() { cv_.notify_all(); }

    private:
      std::mutex mu_;
      std::condition_variable cv_;
      std::deque<std::function<void()>> queue_;
    };

  }  // namespace detail_compat
}  // namespace tbb
