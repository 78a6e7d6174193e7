// A pool of host threads that live for the whole process (host code).
#pragma once
#include <condition_variable>
#include <cstdint>
#include <functional>
#include <mutex>
#include <thread>

namespace qed {

// Worker threads kept for the life of the process, so that each keeps its
// Workspace (stream, reduction buffers, pinned staging) from one batch call to
// the next. A batch call hands the pool one work loop that `extra` workers and
// the calling thread run; batch calls from different host threads take turns.
// Its threads are detached and wait on its members for the rest of the
// process, so a pool is never destroyed (the library's pools are leaked
// singletons).
class WorkerPool {
 public:
  void run(int extra, const std::function<void()> &work) {
    std::lock_guard<std::mutex> serial(run_mtx_);
    {
      std::lock_guard<std::mutex> l(m_);
      while ((int)threads_ < extra) {
        const int idx = (int)threads_++;
        std::thread([this, idx] { loop(idx); }).detach();
      }
      job_ = work;
      wanted_ = extra;
      active_ = extra;
      ++gen_;
    }
    cv_.notify_all();
    work();
    std::unique_lock<std::mutex> l(m_);
    done_.wait(l, [&] { return active_ == 0; });
    job_ = nullptr;
  }

 private:
  void loop(int idx) {
    uint64_t seen = 0;
    std::unique_lock<std::mutex> l(m_);
    for (;;) {
      cv_.wait(l, [&] { return gen_ != seen; });
      seen = gen_;
      if (idx >= wanted_) continue;
      std::function<void()> w = job_;
      l.unlock();
      w();
      l.lock();
      if (--active_ == 0) done_.notify_all();
    }
  }
  std::mutex run_mtx_, m_;
  std::condition_variable cv_, done_;
  std::function<void()> job_;
  size_t threads_ = 0;
  int wanted_ = 0, active_ = 0;
  uint64_t gen_ = 0;
};

}  // namespace qed
