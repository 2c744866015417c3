// oneTBB task_group and task_handle (see detail_scheduler.h)
#pragma once

#include <memory>
#include <utility>

#include "tbb/detail_scheduler.h"

namespace tbb {

  class task_group;

  // A deferred task of a group: counted by the group from defer() until it
  // has run, or until the handle is dropped unrun.
  class task_handle {
  public:
    task_handle() = default;
    task_handle(task_handle&& o) noexcept : group_(o.group_), fn_(std::move(o.fn_)) { o.group_ = nullptr; }
    task_handle& operator=(task_handle&& o) noexcept {
      release();
      group_ = o.group_;
      fn_ = std::move(o.fn_);
      o.group_ = nullptr;
      return *this;
    }
    task_handle(task_handle const&) = delete;
    task_handle& operator=(task_handle const&) = delete;
    ~task_handle() { release(); }
    explicit operator bool() const noexcept { return group_ != nullptr; }

  private:
    friend class task_group;
    task_handle(task_group* g, std::function<void()> f) : group_(g), fn_(std::move(f)) {}
    inline void release();
    task_group* group_ = nullptr;
    std::function<void()> fn_;
  };

  class task_group {
  public:
    task_group() = default;
    task_group(task_group const&) = delete;
    task_group& operator=(task_group const&) = delete;
    ~task_group() { wait(); }

    template <typename F>
    void run(F&& f) {
      pending_.fetch_add(1);
      detail_compat::Scheduler::instance().push([this, fn = std::function<void()>(std::forward<F>(f))]() {
        fn();
        done();
      });
    }

    void run(task_handle&& h) {
      if (!h.group_) return;
      std::function<void()> fn = std::move(h.fn_);
      h.group_ = nullptr;  // the count taken by defer() moves to the queued task
      detail_compat::Scheduler::instance().push([this, fn = std::move(fn)]() {
        fn();
        done();
      });
    }

    template <typename F>
    task_handle defer(F&& f) {
      pending_.fetch_add(1);
      return task_handle(this, std::function<void()>(std::forward<F>(f)));
    }

    // runs queued tasks until this group has none pending
    void wait() {
      auto& s = detail_compat::Scheduler::instance();
      while (pending_.load() > 0) s.runOne();
    }

  private:
    friend class task_handle;
    void done() {
      pending_.fetch_sub(1);
      detail_compat::Scheduler::instance().notify();
    }
    std::atomic<long> pending_{0};
  };

  inline void task_handle::release() {
    if (group_) {
      task_group* g = group_;
      group_ = nullptr;
      g->done();
    }
  }

}  // namespace tbb
