// host_copy.h -- host <-> device copies of pageable host memory through pinned
// staging buffers.
//
// A copy from or to pageable memory cannot be a DMA: the driver bounces it
// through its own pinned buffer on the calling thread.  Here the bounce is done
// by the library instead, in chunks through a small ring of pinned buffers per
// context, so that the host-side copy of one chunk overlaps the DMA of the
// previous one, and each host-side copy is split over a process-wide pool of
// threads (one thread alone moves ~10 GB/s, well under a PCIe Gen5 x16 link).
#pragma once

#include <cuda_runtime.h>

#include <algorithm>
#include <condition_variable>
#include <cstring>
#include <mutex>
#include <thread>
#include <vector>

namespace srcu {

// A fixed pool of threads that splits one memcpy at a time into equal parts;
// the calling thread does a part too.  Jobs from several threads take turns.
class HostCopyPool {
 public:
  static HostCopyPool &get() {
    static HostCopyPool pool;
    return pool;
  }

  void copy(void *dst, const void *src, size_t bytes) {
    if (bytes < kMinSplit || workers_.empty()) {
      std::memcpy(dst, src, bytes);
      return;
    }
    std::lock_guard<std::mutex> turn(job_mu_);
    const size_t parts = workers_.size() + 1;
    {
      std::lock_guard<std::mutex> lock(mu_);
      dst_ = static_cast<char *>(dst);
      src_ = static_cast<const char *>(src);
      bytes_ = bytes;
      parts_ = parts;
      remaining_ = workers_.size();
      ++generation_;
    }
    cv_.notify_all();
    run_part(0);
    std::unique_lock<std::mutex> lock(mu_);
    done_cv_.wait(lock, [&] { return remaining_ == 0; });
  }

  ~HostCopyPool() {
    {
      std::lock_guard<std::mutex> lock(mu_);
      stop_ = true;
      ++generation_;
    }
    cv_.notify_all();
    for (auto &t : workers_) t.join();
  }

 private:
  static constexpr size_t kMinSplit = size_t(1) << 20;  // smaller copies stay on the caller

  HostCopyPool() {
    const unsigned hw = std::thread::hardware_concurrency();
    const unsigned n = std::min(7u, hw > 1 ? hw / 2 : 0u);
    for (unsigned k = 0; k < n; ++k) workers_.emplace_back([this, k] { worker(k + 1); });
  }

  void run_part(size_t part) {
    // parts of equal size, on 64-byte boundaries
    const size_t step = ((bytes_ + parts_ - 1) / parts_ + 63) & ~size_t(63);
    const size_t lo = std::min(bytes_, part * step), hi = std::min(bytes_, lo + step);
    if (hi > lo) std::memcpy(dst_ + lo, src_ + lo, hi - lo);
  }

  void worker(size_t part) {
    unsigned long long seen = 0;
    for (;;) {
      {
        std::unique_lock<std::mutex> lock(mu_);
        cv_.wait(lock, [&] { return generation_ != seen; });
        seen = generation_;
        if (stop_) return;
      }
      run_part(part);
      std::lock_guard<std::mutex> lock(mu_);
      if (--remaining_ == 0) done_cv_.notify_one();
    }
  }

  std::vector<std::thread> workers_;
  std::mutex job_mu_, mu_;
  std::condition_variable cv_, done_cv_;
  char *dst_ = nullptr;
  const char *src_ = nullptr;
  size_t bytes_ = 0, parts_ = 1, remaining_ = 0;
  unsigned long long generation_ = 0;
  bool stop_ = false;
};

// Whether a host pointer is ordinary pageable memory (not pinned or registered).
inline bool is_pageable(const void *p) {
  cudaPointerAttributes a;
  if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
    cudaGetLastError();
    return true;
  }
  return a.type == cudaMemoryTypeUnregistered;
}

}  // namespace srcu
