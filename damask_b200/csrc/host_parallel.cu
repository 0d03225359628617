// Host thread pool for the per-member work of a batch (see host_parallel.h).
#include "host_parallel.h"

#include <cuda_runtime.h>

#include "../../include/damask_b200.h"

namespace dmk {

HostPool::HostPool(int n_threads, int device) {
  for (int t = 0; t < n_threads; ++t) threads_.emplace_back([this, device] { work(device); });
}

HostPool::~HostPool() {
  {
    std::lock_guard<std::mutex> lk(m_);
    stop_ = true;
  }
  start_.notify_all();
  for (auto& t : threads_) t.join();
}

// takes indices until none are left; records each failure with this thread's error message
void HostPool::drain() {
  for (int k = next_.fetch_add(1); k < n_; k = next_.fetch_add(1)) {
    const int rc = (*job_)(k);
    if (rc) {
      rc_[k] = rc;
      const char* m = dmk_last_error();
      msg_[k] = m ? m : "";
    }
  }
}

void HostPool::work(int device) {
  cudaSetDevice(device);
  uint64_t seen = 0;
  for (;;) {
    {
      std::unique_lock<std::mutex> lk(m_);
      start_.wait(lk, [&] { return stop_ || generation_ != seen; });
      if (stop_) return;
      seen = generation_;
    }
    drain();
    {
      std::lock_guard<std::mutex> lk(m_);
      if (--busy_ == 0) done_.notify_all();
    }
  }
}

int HostPool::run(int n, const std::function<int(int)>& f, std::string* msg) {
  if (n <= 0) return 0;
  rc_.assign(n, 0);
  msg_.assign(n, std::string());
  {
    std::lock_guard<std::mutex> lk(m_);
    job_ = &f;
    n_ = n;
    next_.store(0);
    busy_ = int(threads_.size());
    ++generation_;
  }
  start_.notify_all();
  drain();
  {
    std::unique_lock<std::mutex> lk(m_);
    done_.wait(lk, [&] { return busy_ == 0; });
    job_ = nullptr;
  }
  for (int k = 0; k < n; ++k)
    if (rc_[k]) {
      if (msg) *msg = msg_[k];
      return rc_[k];
    }
  return 0;
}

}  // namespace dmk
