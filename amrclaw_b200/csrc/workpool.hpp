// Small persistent host thread pool for the per-patch host work of a regrid
// (flag buffering and nesting masks, fill-program compilation). The reference
// runs the same per-grid loops under OpenMP (e.g. bufnst2.f, advanc.f:106).
#pragma once
#include <algorithm>
#include <atomic>
#include <chrono>
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
      stop_.store(true);
    }
    cv_.notify_all();
    for (auto& w : workers_) w.join();
  }
  int size() const { return (int)workers_.size() + 1; }

  // Calls f(i) for i in [0, n) on the caller and up to n-1 helpers; rethrows the first
  // exception. A regrid makes many such calls in a row: idle workers poll for kSpinUs
  // microseconds before they sleep, so a call that follows soon finds them awake, and only
  // as many workers as there are items beyond the first join a call.
  void run(int n, const std::function<void(int)>& f) {
    if (n <= 0) return;
    const int helpers = std::min<int>((int)workers_.size(), n - 1);
    if (helpers == 0) { for (int i = 0; i < n; ++i) f(i); return; }
    {
      std::lock_guard<std::mutex> g(mu_);
      job_ = &f; n_ = n; next_.store(0); err_ = nullptr;
      active_.store(helpers);
      const unsigned long long gen = (state_.load() >> 32) + 1;
      state_.store((gen << 32) | (unsigned)helpers, std::memory_order_release);
    }
    cv_.notify_all();
    work();
    spin_while([this] { return active_.load(std::memory_order_acquire) != 0; });
    {
      std::unique_lock<std::mutex> lk(mu_);
      done_cv_.wait(lk, [this] { return active_.load() == 0; });
      job_ = nullptr;
    }
    if (err_) std::rethrow_exception(err_);
  }

 private:
  static constexpr int kSpinUs = 100;
  static void relax() {
#if defined(__x86_64__) || defined(__i386__)
    __builtin_ia32_pause();
#else
    std::this_thread::yield();
#endif
  }
  // polls cond() for at most kSpinUs microseconds and returns as soon as it is false;
  // after the first polls it yields between polls, so that with more threads than cores
  // the threads it waits for get to run
  template <class C>
  static void spin_while(C cond) {
    const auto t0 = std::chrono::steady_clock::now();
    for (int s = 0; cond(); ++s) {
      if (s < 256) relax();
      else std::this_thread::yield();
      if ((s & 31) == 31 && std::chrono::steady_clock::now() - t0 > std::chrono::microseconds(kSpinUs)) return;
    }
  }
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
  // state_ = (generation << 32) | free helper slots of that generation's call: a worker
  // takes at most one slot of each generation it sees, so every helper counted in
  // active_ belongs to the call that set it
  void loop() {
    // generation 0 is "no call yet": a worker that starts after the first call was posted
    // still joins it
    unsigned long long seen = 0;
    while (true) {
      spin_while([&] { return (state_.load(std::memory_order_acquire) >> 32) == seen && !stop_.load(); });
      if ((state_.load(std::memory_order_acquire) >> 32) == seen) {
        std::unique_lock<std::mutex> lk(mu_);
        cv_.wait(lk, [&] { return stop_.load() || (state_.load() >> 32) != seen; });
      }
      if (stop_.load()) return;
      unsigned long long v = state_.load(std::memory_order_acquire);
      bool took = false;
      while (true) {
        seen = v >> 32;
        if ((v & 0xffffffffull) == 0) break;
        if (state_.compare_exchange_weak(v, v - 1, std::memory_order_acq_rel)) { took = true; break; }
      }
      if (!took) continue;  // this call has its helpers
      work();
      if (active_.fetch_sub(1) == 1) {
        std::lock_guard<std::mutex> g(mu_);
        done_cv_.notify_all();
      }
    }
  }
  std::vector<std::thread> workers_;
  std::mutex mu_;
  std::condition_variable cv_, done_cv_;
  const std::function<void(int)>* job_ = nullptr;
  int n_ = 0;
  std::atomic<int> next_{0}, active_{0};
  std::atomic<unsigned long long> state_{0};
  std::atomic<bool> stop_{false};
  std::exception_ptr err_;
};

}  // namespace amrb
