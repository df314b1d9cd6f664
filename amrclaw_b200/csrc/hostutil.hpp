// Host-side utilities shared by the 2D and 3D orchestrators: the device pool
// allocator, device buffers with pinned upload staging, and section timers.
#pragma once
#include "common.cuh"
#include <algorithm>
#include <chrono>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <map>
#include <set>
#include <string>
#include <vector>

namespace amrb {

static const double RINF = (double)10.e32f;

// Device-buffer reallocations of this process (cudaFree + cudaMalloc: both wait for the
// device): count and host seconds, reported with the section timers.
inline long long g_dbuf_reallocs = 0;
inline double g_dbuf_realloc_s = 0;
// uploads through the pinned staging ring: bytes, ring wraps (each waits for the stream)
// and host seconds in the copy into the ring
inline double g_stage_bytes = 0, g_stage_copy_s = 0;
inline long long g_stage_wraps = 0;
// pool (Arena) growths: count, host seconds and bytes added
inline long long g_arena_grows = 0;
inline double g_arena_grow_s = 0, g_arena_grow_bytes = 0;

// Stream-ordered reallocation. While a context works on the calling thread its stream is
// set here, and device buffers that grow are freed and allocated in that stream's order
// (cudaFreeAsync / cudaMallocAsync) instead of cudaFree / cudaMalloc, which wait for the
// whole device. The device's default memory pool keeps freed memory for reuse
// (retain_pool_memory), so a grown buffer seldom maps new pages.
inline thread_local cudaStream_t t_alloc_stream = nullptr;
struct AllocStreamScope {
  cudaStream_t prev;
  explicit AllocStreamScope(cudaStream_t s) : prev(t_alloc_stream) { t_alloc_stream = s; }
  ~AllocStreamScope() { t_alloc_stream = prev; }
};
inline void retain_pool_memory() {
  int dev = 0;
  AMR_CUDA(cudaGetDevice(&dev));
  cudaMemPool_t mp;
  AMR_CUDA(cudaDeviceGetDefaultMemPool(&mp, dev));
  unsigned long long thr = ~0ull;
  AMR_CUDA(cudaMemPoolSetAttribute(mp, cudaMemPoolAttrReleaseThreshold, &thr));
}

// Host-side section timers, printed at context destruction when AMRB_PROF is set.
struct HostProf {
  std::map<std::string, std::pair<double, long long>> acc;
  bool on = std::getenv("AMRB_PROF") != nullptr;
  ~HostProf() {
    if (!on) return;
    for (auto& kv : acc) std::fprintf(stderr, "PROF %-22s %9.4f s %8lld calls\n", kv.first.c_str(), kv.second.first, kv.second.second);
    std::fprintf(stderr, "PROF %-22s %9.4f s %8lld calls\n", "dbuf_realloc", g_dbuf_realloc_s, g_dbuf_reallocs);
    std::fprintf(stderr, "PROF %-22s %9.4f s %8lld wraps %.1f MB\n", "staging_copy", g_stage_copy_s, g_stage_wraps, g_stage_bytes / 1e6);
    std::fprintf(stderr, "PROF %-22s %9.4f s %8lld grows %.1f MB\n", "arena_grow", g_arena_grow_s, g_arena_grows, g_arena_grow_bytes / 1e6);
  }
};
struct ScopedTimer {
  HostProf& P; const char* name; std::chrono::steady_clock::time_point t0;
  ScopedTimer(HostProf& p, const char* n) : P(p), name(n), t0(std::chrono::steady_clock::now()) {}
  ~ScopedTimer() {
    if (!P.on) return;
    auto& a = P.acc[name];
    a.first += std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    a.second += 1;
  }
};
// Consecutive phases of one scope: next() closes the running phase and opens another.
struct PhaseTimer {
  HostProf& P; const char* name = nullptr; std::chrono::steady_clock::time_point t0;
  explicit PhaseTimer(HostProf& p) : P(p) {}
  void close() {
    if (name && P.on) {
      auto& a = P.acc[name];
      a.first += std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
      a.second += 1;
    }
    name = nullptr;
  }
  void next(const char* n) { close(); name = n; t0 = std::chrono::steady_clock::now(); }
  ~PhaseTimer() { close(); }
};
#define HPROF(name) ScopedTimer _hp_##__LINE__(hprof, name)  // rinfinity of amr_module.f90 (a default-REAL literal)

// ------------------------------------------------------------------ device pool
// An allocation that would grow a capped pool past its limit (amrgpu_set_pool_limit).
struct PoolLimitError : std::runtime_error {
  using std::runtime_error::runtime_error;
};

struct Arena {
  double* d = nullptr;
  long long cap = 0;
  long long limit = 0;  // most doubles the pool may hold (0: no limit)
  // the context stream when one was set at init: the arena then lives in the device's
  // stream-ordered memory pool, and a new context reuses what an earlier one gave back
  // instead of mapping fresh pages
  cudaStream_t s = nullptr;
  // free blocks indexed both ways: by offset (for coalescing) and by size (best fit in
  // O(log n); a level with thousands of patches would make a first-fit scan quadratic)
  std::map<long long, long long> fr;              // offset -> length
  std::set<std::pair<long long, long long>> bysz;  // (length, offset)
  long long inuse = 0, peak = 0;
  static long long rnd(long long n) { return (n + 31) / 32 * 32; }
  void init(long long n) {
    n = rnd(std::max<long long>(n, 1 << 20));
    s = t_alloc_stream;
    if (s) AMR_CUDA(cudaMallocAsync((void**)&d, sizeof(double) * n, s));
    else AMR_CUDA(cudaMalloc(&d, sizeof(double) * n));
    cap = n;
    fr.clear(); bysz.clear();
    add_free(0, n);
  }
  void add_free(long long off, long long n) { fr[off] = n; bysz.emplace(n, off); }
  void del_free(std::map<long long, long long>::iterator it) { bysz.erase({it->second, it->first}); fr.erase(it); }
  void grow(long long need) {
    const auto t0 = std::chrono::steady_clock::now();
    // kernels on any stream may still use the pool: let them finish before it moves
    if (limit > 0 && cap + rnd(need) > limit)
      throw PoolLimitError("device pool limit reached: " + std::to_string(sizeof(double) * (cap + rnd(need))) +
                           " bytes needed, limit " + std::to_string(sizeof(double) * limit));
    AMR_CUDA(cudaDeviceSynchronize());
    long long ncap = std::max(cap * 2, cap + rnd(need) + (1 << 20));
    if (limit > 0) ncap = std::min(ncap, limit);
    double* nd = nullptr;
    if (s) {
      // in the context stream's order: later work on that stream sees the moved pool
      AMR_CUDA(cudaMallocAsync((void**)&nd, sizeof(double) * ncap, s));
      AMR_CUDA(cudaMemcpyAsync(nd, d, sizeof(double) * cap, cudaMemcpyDeviceToDevice, s));
      AMR_CUDA(cudaFreeAsync(d, s));
    } else {
      AMR_CUDA(cudaMalloc(&nd, sizeof(double) * ncap));
      AMR_CUDA(cudaMemcpy(nd, d, sizeof(double) * cap, cudaMemcpyDeviceToDevice));
      AMR_CUDA(cudaFree(d));
    }
    d = nd;
    release_raw(cap, ncap - cap);
    g_arena_grow_bytes += (double)sizeof(double) * (ncap - cap);
    cap = ncap;
    ++g_arena_grows;
    g_arena_grow_s += std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
  }
  void release_raw(long long off, long long n) {
    auto nx = fr.lower_bound(off);
    if (nx != fr.begin()) {
      auto pv = std::prev(nx);
      if (pv->first + pv->second == off) { off = pv->first; n += pv->second; del_free(pv); }
    }
    nx = fr.lower_bound(off);
    if (nx != fr.end() && off + n == nx->first) { n += nx->second; del_free(nx); }
    add_free(off, n);
  }
  long long alloc(long long n) {
    n = rnd(std::max<long long>(n, 1));
    for (int pass = 0; pass < 2; ++pass) {
      auto b = bysz.lower_bound({n, -1});  // smallest block that fits, lowest offset among equals
      if (b != bysz.end()) {
        const long long len = b->first, off = b->second;
        del_free(fr.find(off));
        if (len > n) add_free(off + n, len - n);
        inuse += n; peak = std::max(peak, inuse);
        return off;
      }
      grow(n);
    }
    throw std::runtime_error("device pool exhausted");
  }
  void release(long long off, long long n) {
    if (off < 0) return;
    n = rnd(std::max<long long>(n, 1));
    inuse -= n;
    release_raw(off, n);
  }
  void destroy() {
    if (d) {
      if (s) { cudaFreeAsync(d, s); cudaStreamSynchronize(s); }
      else cudaFree(d);
    }
    d = nullptr;
  }
};

// amrgpu_set_pool_limit: the patch pool and the register pool of a context share the cap,
// each limited to what it holds now plus the rest of the cap (0 removes it)
inline void set_arena_limits(Arena& pool, Arena& regs, long long bytes) {
  if (bytes < 0) throw std::invalid_argument("amrgpu_set_pool_limit: negative size");
  if (bytes == 0) { pool.limit = regs.limit = 0; return; }
  const long long held = (long long)sizeof(double) * (pool.cap + regs.cap);
  if (bytes < held)
    throw std::invalid_argument("amrgpu_set_pool_limit: the pools already hold " + std::to_string(held) + " bytes");
  const long long spare = (bytes - held) / (long long)sizeof(double);
  pool.limit = pool.cap + spare;
  regs.limit = regs.cap + spare;
}

// Pinned host staging for host-to-device uploads: a copy from pinned memory is
// queued without the driver's pageable bounce. Space is reused only after the
// stream has been synchronized (Staging::reset is called right after each sync).
struct Staging {
  char* h = nullptr;
  size_t cap = 0, used = 0;
  const void* put(const void* src, size_t n, cudaStream_t s) {
    const size_t n2 = (n + 255) & ~(size_t)255;
    if (used + n2 > cap) {
      ++g_stage_wraps;
      AMR_CUDA(cudaStreamSynchronize(s));
      used = 0;
      if (n2 > cap) {
        if (h) AMR_CUDA(cudaFreeHost(h));
        cap = std::max<size_t>({n2, cap * 2, (size_t)8 << 20});
        AMR_CUDA(cudaMallocHost((void**)&h, cap));
      }
    }
    char* dst = h + used;
    const auto t0 = std::chrono::steady_clock::now();
    std::memcpy(dst, src, n);
    g_stage_copy_s += std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    g_stage_bytes += (double)n;
    used += n2;
    return dst;
  }
  void reset() { used = 0; }
  // pin the ring once at start-up: growing it later (cudaFreeHost + cudaMallocHost) costs
  // milliseconds that vary with the host's memory state
  void reserve(size_t bytes) {
    if (bytes <= cap) return;
    if (h) AMR_CUDA(cudaFreeHost(h));
    cap = bytes; used = 0;
    AMR_CUDA(cudaMallocHost((void**)&h, cap));
  }
  void destroy() { if (h) cudaFreeHost(h); h = nullptr; cap = used = 0; }
};

template <class T> struct DBuf {
  T* d = nullptr; size_t cap = 0, n = 0;
  void realloc_to(size_t c) {
    const auto t0 = std::chrono::steady_clock::now();
    cap = c;
    if (t_alloc_stream) {
      if (d) AMR_CUDA(cudaFreeAsync(d, t_alloc_stream));
      AMR_CUDA(cudaMallocAsync((void**)&d, sizeof(T) * cap, t_alloc_stream));
    } else {
      if (d) AMR_CUDA(cudaFree(d));
      AMR_CUDA(cudaMalloc(&d, sizeof(T) * cap));
    }
    ++g_dbuf_reallocs;
    g_dbuf_realloc_s += std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
  }
  // smallest allocation (64 KiB): small per-level arrays then rarely reallocate
  static constexpr size_t kMin = (64 << 10) / sizeof(T) > 16 ? (64 << 10) / sizeof(T) : 16;
  void upload(const std::vector<T>& h, cudaStream_t s, Staging& stg) { upload(h.data(), h.size(), s, stg); }
  void upload(const T* h, size_t cnt, cudaStream_t s, Staging& stg) {
    n = cnt;
    if (n > cap) realloc_to(std::max<size_t>(n * 2, kMin));
    if (n) AMR_CUDA(cudaMemcpyAsync(d, stg.put(h, sizeof(T) * n, s), sizeof(T) * n, cudaMemcpyHostToDevice, s));
  }
  void ensure(size_t m) {
    if (m > cap) realloc_to(std::max<size_t>(m, 16) * 3 / 2);
    n = m;
  }
  // ensure() for large scratch that changes size with the hierarchy: grows to twice the
  // request, so a slowly growing level does not reallocate (and synchronise) every regrid
  void reserve(size_t m) {
    if (m > cap) realloc_to(std::max<size_t>(m * 2, kMin));
    n = m;
  }
  void free() { if (d) cudaFree(d); d = nullptr; cap = n = 0; }
};


}  // namespace amrb
