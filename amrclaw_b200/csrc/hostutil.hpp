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

// Host-side section timers, printed at context destruction when AMRB_PROF is set.
struct HostProf {
  std::map<std::string, std::pair<double, long long>> acc;
  bool on = std::getenv("AMRB_PROF") != nullptr;
  ~HostProf() {
    if (!on) return;
    for (auto& kv : acc) std::fprintf(stderr, "PROF %-22s %9.4f s %8lld calls\n", kv.first.c_str(), kv.second.first, kv.second.second);
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
struct Arena {
  double* d = nullptr;
  long long cap = 0;
  // free blocks indexed both ways: by offset (for coalescing) and by size (best fit in
  // O(log n); a level with thousands of patches would make a first-fit scan quadratic)
  std::map<long long, long long> fr;              // offset -> length
  std::set<std::pair<long long, long long>> bysz;  // (length, offset)
  long long inuse = 0, peak = 0;
  static long long rnd(long long n) { return (n + 31) / 32 * 32; }
  void init(long long n) {
    n = rnd(std::max<long long>(n, 1 << 20));
    AMR_CUDA(cudaMalloc(&d, sizeof(double) * n));
    cap = n;
    fr.clear(); bysz.clear();
    add_free(0, n);
  }
  void add_free(long long off, long long n) { fr[off] = n; bysz.emplace(n, off); }
  void del_free(std::map<long long, long long>::iterator it) { bysz.erase({it->second, it->first}); fr.erase(it); }
  void grow(long long need) {
    // kernels on any stream may still use the pool: let them finish before it moves
    AMR_CUDA(cudaDeviceSynchronize());
    long long ncap = std::max(cap * 2, cap + rnd(need) + (1 << 20));
    double* nd = nullptr;
    AMR_CUDA(cudaMalloc(&nd, sizeof(double) * ncap));
    AMR_CUDA(cudaMemcpy(nd, d, sizeof(double) * cap, cudaMemcpyDeviceToDevice));
    AMR_CUDA(cudaFree(d));
    d = nd;
    release_raw(cap, ncap - cap);
    cap = ncap;
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
  void destroy() { if (d) cudaFree(d); d = nullptr; }
};

// Pinned host staging for host-to-device uploads: a copy from pinned memory is
// queued without the driver's pageable bounce. Space is reused only after the
// stream has been synchronized (Staging::reset is called right after each sync).
struct Staging {
  char* h = nullptr;
  size_t cap = 0, used = 0;
  const void* put(const void* src, size_t n, cudaStream_t s) {
    const size_t n2 = (n + 255) & ~(size_t)255;
    if (used + n2 > cap) {
      AMR_CUDA(cudaStreamSynchronize(s));
      used = 0;
      if (n2 > cap) {
        if (h) AMR_CUDA(cudaFreeHost(h));
        cap = std::max<size_t>({n2, cap * 2, (size_t)8 << 20});
        AMR_CUDA(cudaMallocHost((void**)&h, cap));
      }
    }
    char* dst = h + used;
    std::memcpy(dst, src, n);
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
  // smallest allocation (64 KiB): small per-level arrays then rarely reallocate
  static constexpr size_t kMin = (64 << 10) / sizeof(T) > 16 ? (64 << 10) / sizeof(T) : 16;
  void upload(const std::vector<T>& h, cudaStream_t s, Staging& stg) { upload(h.data(), h.size(), s, stg); }
  void upload(const T* h, size_t cnt, cudaStream_t s, Staging& stg) {
    n = cnt;
    if (n > cap) {
      if (d) AMR_CUDA(cudaFree(d));
      cap = std::max<size_t>(n * 2, kMin);
      AMR_CUDA(cudaMalloc(&d, sizeof(T) * cap));
    }
    if (n) AMR_CUDA(cudaMemcpyAsync(d, stg.put(h, sizeof(T) * n, s), sizeof(T) * n, cudaMemcpyHostToDevice, s));
  }
  void ensure(size_t m) {
    if (m > cap) {
      if (d) AMR_CUDA(cudaFree(d));
      cap = std::max<size_t>(m, 16) * 3 / 2;
      AMR_CUDA(cudaMalloc(&d, sizeof(T) * cap));
    }
    n = m;
  }
  // ensure() for large scratch that changes size with the hierarchy: grows to twice the
  // request, so a slowly growing level does not reallocate (and synchronise) every regrid
  void reserve(size_t m) {
    if (m > cap) {
      if (d) AMR_CUDA(cudaFree(d));
      cap = std::max<size_t>(m * 2, kMin);
      AMR_CUDA(cudaMalloc(&d, sizeof(T) * cap));
    }
    n = m;
  }
  void free() { if (d) cudaFree(d); d = nullptr; cap = n = 0; }
};


}  // namespace amrb
