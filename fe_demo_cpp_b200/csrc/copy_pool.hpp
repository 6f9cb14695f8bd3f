// A small pool of host threads for large memcpy's between pageable and
// page-locked host memory (the host-vector apply's staging).  One thread
// copies 8-12 GB/s; the pool splits each copy over its workers and the
// caller.  Several callers may use it at once (the copy in and the copy out
// of one apply run on two threads).
#pragma once
#include <algorithm>
#include <condition_variable>
#include <cstddef>
#include <cstring>
#include <deque>
#include <mutex>
#include <thread>
#include <vector>

namespace fem_b200 {

class CopyPool {
 public:
  explicit CopyPool(int workers) {
    for (int i = 0; i < workers; ++i) th_.emplace_back([this] { loop(); });
  }
  ~CopyPool() {
    {
      std::lock_guard<std::mutex> lock(mu_);
      stop_ = true;
    }
    cv_.notify_all();
    for (std::thread& t : th_) t.join();
  }
  CopyPool(const CopyPool&) = delete;
  CopyPool& operator=(const CopyPool&) = delete;

  int workers() const { return int(th_.size()); }

  // dst[0, bytes) = src[0, bytes); returns when every part is copied.
  void copy(void* dst, const void* src, size_t bytes) {
    constexpr size_t kMinPart = size_t(256) << 10;
    const size_t parts = std::min<size_t>(th_.size() + 1, std::max<size_t>(1, bytes / kMinPart));
    char* d = static_cast<char*>(dst);
    const char* s = static_cast<const char*>(src);
    if (parts <= 1) {
      std::memcpy(d, s, bytes);
      return;
    }
    const size_t step = ((bytes + parts - 1) / parts + 63) & ~size_t(63);
    Batch b;
    {
      std::lock_guard<std::mutex> lock(mu_);
      for (size_t off = step; off < bytes; off += step) {
        q_.push_back({d + off, s + off, std::min(step, bytes - off), &b});
        ++b.left;
      }
    }
    cv_.notify_all();
    std::memcpy(d, s, std::min(step, bytes));
    std::unique_lock<std::mutex> lock(b.m);
    b.cv.wait(lock, [&] { return b.left == 0; });
  }

 private:
  struct Batch {
    std::mutex m;
    std::condition_variable cv;
    int left = 0;
  };
  struct Job {
    char* dst;
    const char* src;
    size_t n;
    Batch* b;
  };

  void loop() {
    for (;;) {
      Job j;
      {
        std::unique_lock<std::mutex> lock(mu_);
        cv_.wait(lock, [&] { return stop_ || !q_.empty(); });
        if (q_.empty()) return;  // stopping
        j = q_.front();
        q_.pop_front();
      }
      std::memcpy(j.dst, j.src, j.n);
      std::lock_guard<std::mutex> lock(j.b->m);
      if (--j.b->left == 0) j.b->cv.notify_one();
    }
  }

  std::vector<std::thread> th_;
  std::mutex mu_;
  std::condition_variable cv_;
  std::deque<Job> q_;
  bool stop_ = false;
};

}  // namespace fem_b200
