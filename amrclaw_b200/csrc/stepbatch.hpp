// Cross-request batching of the 2D level step (the serving loop's "batches their level
// steps together"): solves that run concurrently in one process, each on its own host
// thread and CUDA stream, hand the patch step of a level substep to a process-wide
// batcher instead of launching it. Submissions of the same Riemann plugin and precision
// that arrive within a short window go out as ONE launch of step2_batch_kernel on the
// batcher's stream; each member's stream waits for the launch before its next work.
//
// Protocol of a submission (StepBatcher::submit, on the solve's host thread):
//   1. the member records `ready` on its own stream (its ghost fill, saveqc and qad are
//      queued before it) and appends itself to the pending list of its key;
//   2. the first member of a key to find no leader becomes the leader: it waits until as
//      many members have submitted as are registered for the key, or until the window has
//      passed, then takes up to STEP2_BATCH_MAX pending members, makes the batch stream
//      wait on their `ready` events, launches, records each member's `done` on the batch
//      stream and wakes them;
//   3. every member (leader included) makes its own stream wait on its `done` event.
// Each tile is stepped with its own solve's arguments, so a result does not depend on
// which solves shared its launches. A member whose launch failed gets the error.
#pragma once
#include <chrono>
#include <condition_variable>
#include <map>
#include <mutex>
#include <stdexcept>
#include <string>
#include <vector>

#include "kernels2d.cuh"

namespace amrb {

class StepBatcher {
 public:
  struct Member {
    int key = 0;
    cudaEvent_t ready = nullptr, done = nullptr;
    // filled per submission
    StepArgs args{};
    int grid = 0;
    bool launched = false;
    std::string error;
    int batch_size = 0;  // members of the launch this submission went out in
  };

  static StepBatcher& get() {
    static StepBatcher b;
    return b;
  }
  static int make_key(int solver, bool f32) { return solver * 2 + (f32 ? 1 : 0); }

  void join(Member& m, int key) {
    AMR_CUDA(cudaEventCreateWithFlags(&m.ready, cudaEventDisableTiming));
    AMR_CUDA(cudaEventCreateWithFlags(&m.done, cudaEventDisableTiming));
    m.key = key;
    std::lock_guard<std::mutex> lk(mu_);
    ++keys_[key].registered;
  }
  void leave(Member& m) {
    {
      std::lock_guard<std::mutex> lk(mu_);
      --keys_[m.key].registered;
    }
    cv_.notify_all();
    if (m.ready) cudaEventDestroy(m.ready);
    if (m.done) cudaEventDestroy(m.done);
    m.ready = m.done = nullptr;
  }

  // Queues member m's step (args, grid blocks) behind its stream's work and returns once the
  // shared launch is queued and `stream` waits for it. window_us: how long a leader waits
  // for the other registered members of its key.
  void submit(Member& m, const StepArgs& args, int grid, cudaStream_t stream, int window_us) {
    AMR_CUDA(cudaEventRecord(m.ready, stream));
    std::unique_lock<std::mutex> lk(mu_);
    Key& K = keys_[m.key];
    m.args = args; m.grid = grid; m.launched = false; m.error.clear(); m.batch_size = 0;
    K.pending.push_back(&m);
    cv_.notify_all();
    while (!m.launched) {
      if (!K.leader) {
        K.leader = true;
        const auto until = std::chrono::steady_clock::now() + std::chrono::microseconds(window_us);
        cv_.wait_until(lk, until, [&] { return (int)K.pending.size() >= std::max(1, K.registered); });
        const size_t n = std::min<size_t>(K.pending.size(), STEP2_BATCH_MAX);
        std::vector<Member*> take(K.pending.begin(), K.pending.begin() + n);
        K.pending.erase(K.pending.begin(), K.pending.begin() + n);
        K.leader = false;
        lk.unlock();
        std::string err;
        try {
          launch(take, m.key);
        } catch (std::exception& e) {
          err = e.what();
        }
        lk.lock();
        for (Member* x : take) { x->launched = true; x->error = err; x->batch_size = (int)n; }
        ++launches_;
        members_ += (long long)n;
        cv_.notify_all();
      } else {
        cv_.wait(lk);
      }
    }
    lk.unlock();
    if (!m.error.empty()) throw std::runtime_error("batched step launch: " + m.error);
    AMR_CUDA(cudaStreamWaitEvent(stream, m.done, 0));
  }

  // launches made and members they carried, over the process
  void stats(long long& launches, long long& members) {
    std::lock_guard<std::mutex> lk(mu_);
    launches = launches_;
    members = members_;
  }

 private:
  struct Key {
    int registered = 0;
    bool leader = false;
    std::vector<Member*> pending;
  };
  std::mutex mu_;
  std::condition_variable cv_;
  std::map<int, Key> keys_;
  std::mutex launch_mu_;
  cudaStream_t stream_ = nullptr;
  long long launches_ = 0, members_ = 0;

  void launch(const std::vector<Member*>& take, int key) {
    std::lock_guard<std::mutex> lk(launch_mu_);
    if (!stream_) AMR_CUDA(cudaStreamCreateWithFlags(&stream_, cudaStreamNonBlocking));
    StepBatch b{};
    b.n = (int)take.size();
    b.work0[0] = 0;
    int grid = 0;
    for (int k = 0; k < b.n; ++k) {
      b.m[k] = take[k]->args;
      b.work0[k + 1] = b.work0[k] + take[k]->args.nwork;
      grid += take[k]->grid;
      AMR_CUDA(cudaStreamWaitEvent(stream_, take[k]->ready, 0));
    }
    launch_step2_batch(key / 2, b, grid, stream_, (key & 1) != 0);
    for (Member* x : take) AMR_CUDA(cudaEventRecord(x->done, stream_));
  }
};

}  // namespace amrb
