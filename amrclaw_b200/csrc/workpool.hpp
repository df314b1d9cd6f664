// Small persistent host thread pool for the per-patch host work of a regrid
// (flag buffering and nesting masks, fill-program compilation). The reference
// runs the same per-grid loops under OpenMP (e.g. bufnst2.f, advanc.f:106).
#pragma once
#include <algorithm>
#include <atomic>
#include <condition_variable>
#include <cstdlib>
#include <exception>
#include <functional>
#include <mutex>
#include <thread>
#include <vector>

namespace amrb {

class WorkPool {
 public:
  // nthreads <= 0: AMRGPU_HOST_THREADS if set (a server running many contexts lowers it),
  // else up to 16 hardware threads
  explicit WorkPool(int nthreads = 0) {
    if (nthreads <= 0) {
      const char* e = std::getenv("AMRGPU_HOST_THREADS");
      nthreads = e ? std::atoi(e) : 0;
    }
    if (nthreads <= 0) nthreads = (int)std::min(16u, std::max(1u, std::thread::hardware_concurrency()));
    nthreads = std::min(nthreads, 64);
    for (int t = 1; t < nthreads; ++t) workers_.emplace_back([this] { loop(); });
  }
  ~WorkPool() {
    {
      std::lock_guard<std::mutex> g(mu_);
      stop_ = true;
    }
    cv_.notify_all();
    for (auto& w : workers_) w.join();
  }
  int size() const { return (int)workers_.size() + 1; }

  // Calls f(i) for i in [0, n) on all threads; rethrows the first exception.
  void run(int n, const std::function<void(int)>& f) {
    if (n <= 0) return;
    if (workers_.empty() || n == 1) { for (int i = 0; i < n; ++i) f(i); return; }
    {
      std::lock_guard<std::mutex> g(mu_);
      job_ = &f; n_ = n; next_.store(0); err_ = nullptr; active_ = (int)workers_.size(); ++gen_;
    }
    cv_.notify_all();
    work();
    std::unique_lock<std::mutex> lk(mu_);
    done_cv_.wait(lk, [this] { return active_ == 0; });
    job_ = nullptr;
    if (err_) std::rethrow_exception(err_);
  }

 private:
  void work() {
    while (true) {
      const int i = next_.fetch_add(1);
      if (i >= n_) break;
      try {
        (*job_)(i);
      } catch (...) {
        std::lock_guard<std::mutex> g(mu_);
        if (!err_) err_ = std::current_exception();
      }
    }
  }
  void loop() {
    unsigned seen = 0;
    while (true) {
      {
        std::unique_lock<std::mutex> lk(mu_);
        cv_.wait(lk, [&] { return stop_ || gen_ != seen; });
        if (stop_) return;
        seen = gen_;
      }
      work();
      {
        std::lock_guard<std::mutex> g(mu_);
        if (--active_ == 0) done_cv_.notify_all();
      }
    }
  }
  std::vector<std::thread> workers_;
  std::mutex mu_;
  std::condition_variable cv_, done_cv_;
  const std::function<void(int)>* job_ = nullptr;
  int n_ = 0, active_ = 0;
  std::atomic<int> next_{0};
  unsigned gen_ = 0;
  bool stop_ = false;
  std::exception_ptr err_;
};

}  // namespace amrb
