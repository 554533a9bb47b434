// Minimal persistent thread pool for the oracle's outer loops (test infrastructure).
// par_for(lo, hi, f) calls f(v) for v = lo..hi (inclusive) split in contiguous chunks over
// ORACLE_THREADS threads (default: all hardware threads).  Each chunk runs its indices in
// ascending order, so per-index results never depend on the thread count.
#pragma once

#include <algorithm>
#include <condition_variable>
#include <cstdlib>
#include <functional>
#include <mutex>
#include <thread>
#include <vector>

namespace streams_oracle {

class ThreadPool {
 public:
  static ThreadPool& instance() {
    static ThreadPool pool;
    return pool;
  }
  int size() const { return nthreads_; }

  void run(int lo, int hi, const std::function<void(int)>& f) {
    const int n = hi - lo + 1;
    if (n <= 0) return;
    if (nthreads_ <= 1 || n == 1) {
      for (int v = lo; v <= hi; ++v) f(v);
      return;
    }
    std::unique_lock<std::mutex> lk(m_);
    job_ = &f;
    lo_ = lo;
    hi_ = hi;
    pending_ = nthreads_ - 1;
    ++gen_;
    cv_.notify_all();
    lk.unlock();
    chunk(0, f);  // the caller takes chunk 0
    lk.lock();
    done_cv_.wait(lk, [&] { return pending_ == 0; });
    job_ = nullptr;
  }

  ~ThreadPool() {
    {
      std::lock_guard<std::mutex> lk(m_);
      stop_ = true;
      ++gen_;
    }
    cv_.notify_all();
    for (auto& t : workers_) t.join();
  }

 private:
  ThreadPool() {
    const char* e = std::getenv("ORACLE_THREADS");
    int n = e ? std::atoi(e) : static_cast<int>(std::thread::hardware_concurrency());
    nthreads_ = std::max(1, n);
    for (int t = 1; t < nthreads_; ++t) workers_.emplace_back([this, t] { loop(t); });
  }

  void chunk(int t, const std::function<void(int)>& f) {
    const int n = hi_ - lo_ + 1;
    const int a = lo_ + static_cast<int>((static_cast<long long>(n) * t) / nthreads_);
    const int b = lo_ + static_cast<int>((static_cast<long long>(n) * (t + 1)) / nthreads_) - 1;
    for (int v = a; v <= b; ++v) f(v);
  }

  void loop(int t) {
    unsigned long long seen = 0;
    for (;;) {
      std::unique_lock<std::mutex> lk(m_);
      cv_.wait(lk, [&] { return stop_ || gen_ != seen; });
      if (stop_) return;
      seen = gen_;
      const std::function<void(int)>* f = job_;
      lk.unlock();
      chunk(t, *f);
      lk.lock();
      if (--pending_ == 0) done_cv_.notify_one();
    }
  }

  int nthreads_ = 1;
  std::vector<std::thread> workers_;
  std::mutex m_;
  std::condition_variable cv_, done_cv_;
  const std::function<void(int)>* job_ = nullptr;
  int lo_ = 0, hi_ = -1, pending_ = 0;
  unsigned long long gen_ = 0;
  bool stop_ = false;
};

template <class F>
inline void par_for(int lo, int hi, F&& f) {
  std::function<void(int)> fn(std::forward<F>(f));
  ThreadPool::instance().run(lo, hi, fn);
}

inline int oracle_threads() { return ThreadPool::instance().size(); }

}  // namespace streams_oracle
