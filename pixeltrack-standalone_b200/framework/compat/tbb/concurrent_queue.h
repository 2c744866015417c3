// oneTBB concurrent_queue: push and try_pop under a mutex
#pragma once

#include <deque>
#include <mutex>
#include <utility>

namespace tbb {

  template <typename T>
  class concurrent_queue {
  public:
    void push(T const& v) {
      std::lock_guard<std::mutex> lk(mu_);
      q_.push_back(v);
    }
    void push(T&& v) {
      std::lock_guard<std::mutex> lk(mu_);
      q_.push_back(std::move(v));
    }
    bool try_pop(T& out) {
      std::lock_guard<std::mutex> lk(mu_);
      if (q_.empty()) return false;
      out = std::move(q_.front());
      q_.pop_front();
      return true;
    }
    bool empty() const {
      std::lock_guard<std::mutex> lk(mu_);
      return q_.empty();
    }

  private:
    mutable std::mutex mu_;
    std::deque<T> q_;
  };

}  // namespace tbb
