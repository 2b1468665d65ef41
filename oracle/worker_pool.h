// worker_pool.h -- TEST INFRASTRUCTURE: the thread pool of the CPU oracles'
// batched render (vko_render_jobs).  Threads are created once; run(fn) makes
// every worker call fn(worker) and returns when all have finished, with the
// wall time from the release of the workers to the last one's return.
#pragma once

#include <chrono>
#include <condition_variable>
#include <cstdint>
#include <functional>
#include <mutex>
#include <thread>
#include <vector>

namespace vko {

class WorkerPool {
 public:
  explicit WorkerPool(uint32_t n) {
    threads_.reserve(n);
    for (uint32_t w = 0; w < n; ++w) threads_.emplace_back([this, w] { loop(w); });
  }
  ~WorkerPool() {
    {
      std::lock_guard<std::mutex> lk(m_);
      stop_ = true;
      ++generation_;
    }
    go_.notify_all();
    for (auto& t : threads_) t.join();
  }
  WorkerPool(const WorkerPool&) = delete;
  WorkerPool& operator=(const WorkerPool&) = delete;

  uint32_t size() const { return static_cast<uint32_t>(threads_.size()); }

  // Runs fn(worker) on every worker; returns the wall time in milliseconds.
  double run(const std::function<void(uint32_t)>& fn) {
    std::unique_lock<std::mutex> lk(m_);
    fn_ = &fn;
    pending_ = size();
    const auto t0 = std::chrono::steady_clock::now();
    ++generation_;
    go_.notify_all();
    done_.wait(lk, [this] { return pending_ == 0; });
    const auto t1 = std::chrono::steady_clock::now();
    fn_ = nullptr;
    return std::chrono::duration<double, std::milli>(t1 - t0).count();
  }

 private:
  void loop(uint32_t w) {
    uint64_t seen = 0;
    for (;;) {
      const std::function<void(uint32_t)>* fn = nullptr;
      {
        std::unique_lock<std::mutex> lk(m_);
        go_.wait(lk, [&] { return generation_ != seen; });
        seen = generation_;
        if (stop_) return;
        fn = fn_;
      }
      (*fn)(w);
      {
        std::lock_guard<std::mutex> lk(m_);
        if (--pending_ == 0) done_.notify_one();
      }
    }
  }

  std::vector<std::thread> threads_;
  std::mutex m_;
  std::condition_variable go_, done_;
  const std::function<void(uint32_t)>* fn_ = nullptr;
  uint64_t generation_ = 0;
  uint32_t pending_ = 0;
  bool stop_ = false;
};

// About eight chunks per worker, at most 64 pixels each, at least one.
inline uint32_t chunk_pixels(uint32_t pixel_count, uint32_t workers) {
  const uint64_t per = (static_cast<uint64_t>(pixel_count) + 8ull * workers - 1) / (8ull * workers);
  return static_cast<uint32_t>(per < 1 ? 1 : (per > 64 ? 64 : per));
}

}  // namespace vko
